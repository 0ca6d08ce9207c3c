"""Regenerates the oracle regression fixture in this folder.

The reference has no golden vectors for the large step, so this fixture is
the oracle's own output for a small seeded moist, open-boundary case (one
complete time step: solve2 + pdefq + solve3).  tests/test_oracle_kat.py checks
the oracle reproduces it bit for bit; the GPU tests compare against the same
case within the parity tolerance (1e-5 of each field's range).

    python tests/golden/make_golden.py
"""
import os
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)

from cm1_b200.cases import make_case  # noqa: E402
from oracle import oracle  # noqa: E402


def main():
    case = make_case("supercell", ni=12, nj=10, nk=8, seed=42)
    st, m2, cfl = oracle.step(case)
    keep = {k: v for k, v in st.items() if k not in ("uten1", "vten1", "wten1", "ppten", "thten1", "qten", "ptten")}
    out = os.path.join(os.path.dirname(os.path.abspath(__file__)), "supercell_12x10x8_step1.npz")
    np.savez_compressed(out, mass2=np.float64(m2), cflmax=np.float32(cfl), **keep)
    print("wrote", out, os.path.getsize(out), "bytes")


if __name__ == "__main__":
    main()
