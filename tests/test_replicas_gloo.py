"""The N>1 path of bench.py on CPU: two gloo ranks (world size 2).

Each rank of a multi-GPU run advances its own replica; the only collective
is the max of the ranks' times, and the job value counts every rank's cells
over that slowest time.  Two spawned processes check the collective, the
arithmetic and that the ranks' replicas are different realisations of the
same configuration."""
import os
import socket

import numpy as np
import pytest

from cm1_b200.replicas import job_value, max_over_ranks, replica_seed


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def _worker(rank, world, port, out):
    import torch.distributed as dist
    from cm1_b200.cases import make_case
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), WORLD_SIZE=str(world), RANK=str(rank))
    import datetime
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        ms = 10.0 * (rank + 1)                       # rank 1 is the slow one
        ms_max = max_over_ranks(ms, dist, device="cpu")
        case = make_case("dry_bubble", seed=replica_seed(rank), ni=16, nj=12, nk=8)
        cells = case.cfg.ni * case.cfg.nj * case.cfg.nk
        out[rank] = (ms_max, job_value(world, cells, 5, ms_max), float(case.state["th3d"].sum()),
                     (case.cfg.ni, case.cfg.nj, case.cfg.nk))
        dist.barrier()
    finally:
        dist.destroy_process_group()


def test_two_gloo_ranks():
    import torch.multiprocessing as mp
    world = 2
    port = _free_port()
    mgr = mp.get_context("spawn").Manager()
    out = mgr.dict()
    mp.start_processes(_worker, args=(world, port, out), nprocs=world, join=True, start_method="spawn")
    r0, r1 = out[0], out[1]
    assert r0[0] == r1[0] == 20.0                     # the max over ranks, on every rank
    cells = 16 * 12 * 8
    assert r0[1] == pytest.approx(2 * cells * 5 / 0.020)
    assert r0[3] == r1[3]                            # same configuration
    assert r0[2] != r1[2]                            # different realisations


def test_single_rank_helpers():
    assert max_over_ranks(3.5) == 3.5
    assert job_value(1, 100, 2, 1.0) == pytest.approx(2e5)
    with pytest.raises(ValueError):
        job_value(1, 100, 2, 0.0)
    assert replica_seed(0) != replica_seed(1)
    assert np.isfinite(job_value(8, 5_242_880, 20, 9.7))
