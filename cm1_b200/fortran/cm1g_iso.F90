!-----------------------------------------------------------------------
!  cm1g_iso -- ISO_C_BINDING interface to libcm1g.so for CM1's Fortran.
!
!  Drop-in use from solve2.F / cm1.F:
!
!    use cm1g_iso
!    ...  (once, after param/base/init3d)
!    call cm1g_setup( cm1g_ctx )
!    ...  (in the time loop, instead of solve2 + pdefq or mp_driver + solve3)
!    call cm1g_large_step( cm1g_ctx, nstep, dt, mtime, mass1, mass2, cflmax, &
!                          ua,u3d,uten1, va,v3d,vten1, wa,w3d,wten1,       &
!                          ppi,pp3d,ppx,ppten, tha,th3d,thten1, rho,prs,   &
!                          qa,q3d,qten, pta,pt3d,ptten,                    &
!                          radbcw,radbce,radbcs,radbcn, rain,prate )
!
!  The arrays are the model's own (ib:ie,jb:je,kb:ke ...) arrays; the
!  library copies them to the GPU and back each call.  Fortran `real` is
!  C float, `double precision` is C double, `integer` is int32_t.
!-----------------------------------------------------------------------
module cm1g_iso
  use iso_c_binding
  implicit none
  private
  public :: cm1g_config_t, cm1g_grid_t, cm1g_state_t
  public :: cm1g_init, cm1g_finalize, cm1g_step, cm1g_solve2, cm1g_solve3, cm1g_pdefq
  public :: cm1g_bcs, cm1g_bcp, cm1g_bcu, cm1g_bcv, cm1g_bcw, cm1g_last_error_f
  public :: cm1g_calcmass, cm1g_calcener, cm1g_dtsmall, cm1g_tendency_init
  public :: cm1g_setup, cm1g_large_step
  public :: cm1g_tune_t, cm1g_set_tune, cm1g_get_tune, cm1g_autotune

  integer(c_int32_t), parameter :: CM1G_MAXQ = 8

  type, bind(C) :: cm1g_config_t
    integer(c_int32_t) :: ni, nj, nk, ngxy
    real(c_float)      :: dx, dy, dz
    integer(c_int32_t) :: wbc, ebc, sbc, nbc
    integer(c_int32_t) :: hadvordrs, vadvordrs, hadvordrv, vadvordrv
    integer(c_int32_t) :: advwenos, advwenov, weno_order
    integer(c_int32_t) :: nsound
    real(c_float)      :: alph, kdiv
    integer(c_int32_t) :: imoist, eqtset, numq, nqv
    integer(c_int32_t) :: iptra, npt, pdtra
    integer(c_int32_t) :: apmasscon
    integer(c_int32_t) :: irbc
    real(c_float)      :: cstar
    integer(c_int32_t) :: roflux
    real(c_float)      :: smeps
    integer(c_int32_t) :: testcase, psolver, terrain_flag, axisymm, icor
    real(c_float)      :: qmag(CM1G_MAXQ)
    integer(c_int32_t) :: idiff, difforder, mdiff
    real(c_float)      :: kdiff6
    integer(c_int32_t) :: ptype, nql1, nql2, efall
    real(c_float)      :: tsmall, qsmall
  end type

  type, bind(C) :: cm1g_grid_t
    type(c_ptr) :: uh, ruh, uf, ruf, vh, rvh, vf, rvf
    type(c_ptr) :: mh, rmh, c1, c2, mf, rmf
    type(c_ptr) :: pi0, rho0, rr0, rf0, rrf0, th0, rth0, qv0, qc0, qi0, prs0
    type(c_ptr) :: u0, v0, dtu0, dtv0
  end type

  type, bind(C) :: cm1g_state_t
    type(c_ptr) :: ua, u3d, uten1, va, v3d, vten1, wa, w3d, wten1
    type(c_ptr) :: ppi, pp3d, ppx, ppten, tha, th3d, thten1, rho, prs
    type(c_ptr) :: qa, q3d, qten, pta, pt3d, ptten
    type(c_ptr) :: radbcw, radbce, radbcs, radbcn
    type(c_ptr) :: rain, prate
  end type

  ! launch shapes of the large step (cm1g_set_tune / cm1g_autotune)
  type, bind(C) :: cm1g_tune_t
    integer(c_int32_t) :: adv_shape, mom_shape, sound_form
    real(c_float)      :: step_ms
  end type

  ! switches of namelist param9 and host values of the statistics package
  ! (cm1g_stat_setup); fill from module input after param
  type, bind(C) :: cm1g_stat_opts_t
    integer(c_int32_t) :: stat_w, stat_wlevs, stat_u, stat_v, stat_rmw, stat_pipert, stat_prspert, &
                          stat_thpert, stat_q, stat_tke, stat_km, stat_kh, stat_div, stat_rh, stat_rhi, &
                          stat_the, stat_cloud, stat_sfcprs, stat_wsp, stat_cfl, stat_vort, stat_tmass, &
                          stat_tmois, stat_qmass, stat_tenerg, stat_mo, stat_tmf, stat_pcn, stat_qsrc
    integer(c_int32_t) :: adapt_dt, bbc, ptype, iice
    integer(c_int32_t) :: nql1, nql2
    integer(c_int32_t) :: cloudvar(CM1G_MAXQ)
    integer(c_int32_t) :: nbudget
    real(c_float)      :: maxz, cgs1, cgs2, cgs3
    type(c_ptr)        :: zh, zf
    character(kind=c_char) :: qname(4, CM1G_MAXQ)
    type(c_ptr)        :: budname
  end type

  ! writeout's output switches for the fields the library advances
  type, bind(C) :: cm1g_writeout_opts_t
    integer(c_int32_t) :: output_rain, output_prate, output_th, output_thpert, output_prs, output_prspert, &
                          output_pi, output_pipert, output_rho, output_rhopert, output_qv, output_qvpert, &
                          output_q, output_u, output_upert, output_v, output_vpert, output_w
    character(kind=c_char) :: qname(4, CM1G_MAXQ)
  end type

  ! scalars of a restart file (cm1g_restart_write / cm1g_restart_read)
  type, bind(C) :: cm1g_restart_t
    integer(c_int32_t) :: nstep
    real(c_double)     :: mtime
    real(c_float)      :: dt, dtlast
    real(c_double)     :: mass1
  end type

  interface
    integer(c_int) function cm1g_init(cfg, grid, ctx) bind(C, name="cm1g_init")
      import :: c_int, c_ptr, cm1g_config_t, cm1g_grid_t
      type(cm1g_config_t), intent(in) :: cfg
      type(cm1g_grid_t), intent(in) :: grid
      type(c_ptr), intent(out) :: ctx
    end function
    integer(c_int) function cm1g_finalize(ctx) bind(C, name="cm1g_finalize")
      import :: c_int, c_ptr
      type(c_ptr), value :: ctx
    end function
    integer(c_int) function cm1g_solve2(ctx, nstep, dt, mtime, mass1, mass2, cflmax, st) bind(C, name="cm1g_solve2")
      import :: c_int, c_int32_t, c_float, c_double, c_ptr, cm1g_state_t
      type(c_ptr), value :: ctx
      integer(c_int32_t), value :: nstep
      real(c_float), value :: dt
      real(c_double), value :: mtime, mass1
      real(c_double), intent(out) :: mass2
      real(c_float), intent(out) :: cflmax
      type(cm1g_state_t), intent(inout) :: st
    end function
    integer(c_int) function cm1g_step(ctx, nstep, dt, mtime, mass1, mass2, cflmax, st, use_graph) &
        bind(C, name="cm1g_step")
      import :: c_int, c_int32_t, c_float, c_double, c_ptr, cm1g_state_t
      type(c_ptr), value :: ctx
      integer(c_int32_t), value :: nstep
      real(c_float), value :: dt
      real(c_double), value :: mtime, mass1
      real(c_double), intent(out) :: mass2
      real(c_float), intent(out) :: cflmax
      type(cm1g_state_t), intent(inout) :: st
      integer(c_int32_t), value :: use_graph
    end function
    integer(c_int) function cm1g_solve3(ctx, st) bind(C, name="cm1g_solve3")
      import :: c_int, c_ptr, cm1g_state_t
      type(c_ptr), value :: ctx
      type(cm1g_state_t), intent(inout) :: st
    end function
    integer(c_int) function cm1g_pdefq(ctx, rmax, asq, rho, q3d) bind(C, name="cm1g_pdefq")
      import :: c_int, c_float, c_double, c_ptr
      type(c_ptr), value :: ctx
      real(c_float), value :: rmax
      real(c_double), intent(inout) :: asq
      real(c_float), intent(in) :: rho(*)
      real(c_float), intent(inout) :: q3d(*)
    end function
    integer(c_int) function cm1g_bcs(ctx, s) bind(C, name="cm1g_bcs")
      import :: c_int, c_float, c_ptr
      type(c_ptr), value :: ctx
      real(c_float), intent(inout) :: s(*)
    end function
    integer(c_int) function cm1g_bcp(ctx, p) bind(C, name="cm1g_bcp")
      import :: c_int, c_float, c_ptr
      type(c_ptr), value :: ctx
      real(c_float), intent(inout) :: p(*)
    end function
    integer(c_int) function cm1g_bcu(ctx, u) bind(C, name="cm1g_bcu")
      import :: c_int, c_float, c_ptr
      type(c_ptr), value :: ctx
      real(c_float), intent(inout) :: u(*)
    end function
    integer(c_int) function cm1g_bcv(ctx, v) bind(C, name="cm1g_bcv")
      import :: c_int, c_float, c_ptr
      type(c_ptr), value :: ctx
      real(c_float), intent(inout) :: v(*)
    end function
    integer(c_int) function cm1g_bcw(ctx, w, flag) bind(C, name="cm1g_bcw")
      import :: c_int, c_int32_t, c_float, c_ptr
      type(c_ptr), value :: ctx
      real(c_float), intent(inout) :: w(*)
      integer(c_int32_t), value :: flag
    end function
    ! advs (adv.F:14-19): the arguments kept, in advs's order
    integer(c_int) function cm1g_advs(ctx, nrk, wflag, divx, rru, rrv, rrw, s0, s, sten, pdef, pdefweno, &
                                      dt, weps) bind(C, name="cm1g_advs")
      import :: c_int, c_int32_t, c_float, c_double, c_ptr
      type(c_ptr), value :: ctx
      integer(c_int32_t), value :: nrk, wflag, pdef, pdefweno
      real(c_float), intent(in) :: divx(*), rru(*), rrv(*), rrw(*), s0(*), s(*)
      real(c_float), intent(inout) :: sten(*)
      real(c_float), value :: dt
      real(c_double), value :: weps
    end function
    ! advu, advv, advw (adv.F:911-912, 1847-1848, 2778-2781): the arguments
    ! kept, in each routine's order; rru/rrv/rrw/divx are formed on the device
    integer(c_int) function cm1g_advu(ctx, nrk, u3d, uten, v3d, w3d) bind(C, name="cm1g_advu")
      import :: c_int, c_int32_t, c_float, c_ptr
      type(c_ptr), value :: ctx
      integer(c_int32_t), value :: nrk
      real(c_float), intent(in) :: u3d(*), v3d(*), w3d(*)
      real(c_float), intent(inout) :: uten(*)
    end function
    integer(c_int) function cm1g_advv(ctx, nrk, v3d, vten, u3d, w3d) bind(C, name="cm1g_advv")
      import :: c_int, c_int32_t, c_float, c_ptr
      type(c_ptr), value :: ctx
      integer(c_int32_t), value :: nrk
      real(c_float), intent(in) :: v3d(*), u3d(*), w3d(*)
      real(c_float), intent(inout) :: vten(*)
    end function
    integer(c_int) function cm1g_advw(ctx, nrk, w3d, wten, u3d, v3d) bind(C, name="cm1g_advw")
      import :: c_int, c_int32_t, c_float, c_ptr
      type(c_ptr), value :: ctx
      integer(c_int32_t), value :: nrk
      real(c_float), intent(in) :: w3d(*), u3d(*), v3d(*)
      real(c_float), intent(inout) :: wten(*)
    end function
    ! solve2.F:883-893's three calls in one
    integer(c_int) function cm1g_advuvw(ctx, nrk, u3d, v3d, w3d, uten, vten, wten) bind(C, name="cm1g_advuvw")
      import :: c_int, c_int32_t, c_float, c_ptr
      type(c_ptr), value :: ctx
      integer(c_int32_t), value :: nrk
      real(c_float), intent(in) :: u3d(*), v3d(*), w3d(*)
      real(c_float), intent(inout) :: uten(*), vten(*), wten(*)
    end function
    ! sound (sound.F:10-24): the arguments kept, in sound's order
    integer(c_int) function cm1g_sound(ctx, dt, radbcw, radbce, radbcs, radbcn, &
                                       rru, ua, u3d, uten, rrv, va, v3d, vten, rrw, wa, w3d, wten, &
                                       ppi, pp3d, piadv, ppten, ppx, thv, ppterm, nrk, dttmp) &
        bind(C, name="cm1g_sound")
      import :: c_int, c_int32_t, c_float, c_ptr
      type(c_ptr), value :: ctx
      real(c_float), value :: dt, dttmp
      real(c_float), intent(inout) :: radbcw(*), radbce(*), radbcs(*), radbcn(*)
      real(c_float), intent(inout) :: rru(*), ua(*), u3d(*), rrv(*), va(*), v3d(*), rrw(*), wa(*), w3d(*)
      real(c_float), intent(in) :: uten(*), vten(*), wten(*), piadv(*), ppten(*), thv(*), ppterm(*)
      real(c_float), intent(inout) :: ppi(*), pp3d(*), ppx(*)
      integer(c_int32_t), value :: nrk
    end function
    ! calcmass (misclibs.F:3134) and calcener (misclibs.F:3343): FP64 budgets
    integer(c_int) function cm1g_calcmass(ctx, rho, tmass) bind(C, name="cm1g_calcmass")
      import :: c_int, c_float, c_double, c_ptr
      type(c_ptr), value :: ctx
      real(c_float), intent(in) :: rho(*)
      real(c_double), intent(out) :: tmass
    end function
    integer(c_int) function cm1g_calcener(ctx, zh, rho, ua, va, wa, ppi, tha, qv, ql, qi, vr, energy) &
        bind(C, name="cm1g_calcener")
      import :: c_int, c_float, c_double, c_ptr
      type(c_ptr), value :: ctx
      real(c_float), intent(in) :: zh(*), rho(*), ua(*), va(*), wa(*), ppi(*), tha(*), qv(*), ql(*), qi(*), vr(*)
      real(c_double), intent(out) :: energy(5)
    end function
    ! dtsmall (misclibs.F:817): the module values it reads are arguments here
    integer(c_int) function cm1g_dtsmall(psolver, nx, ny, min_dx, min_dy, min_dz, adapt_dt, dt, dbldt, nsound) &
        bind(C, name="cm1g_dtsmall")
      import :: c_int, c_int32_t, c_float, c_double
      integer(c_int32_t), value :: psolver, nx, ny, adapt_dt
      real(c_float), value :: min_dx, min_dy, min_dz
      real(c_float), intent(inout) :: dt
      real(c_double), intent(inout) :: dbldt
      integer(c_int32_t), intent(out) :: nsound
    end function
    ! Rayleigh damping / zeroing of the pre-RK tendencies (solve1.F:414-486)
    integer(c_int) function cm1g_tendency_init(ctx, irdamp, rdalpha, tauh, taus, tauf, uavg, vavg, thavg, &
        ua, va, wa, tha, uten1, vten1, wten1, thten1, qten, ptten) bind(C, name="cm1g_tendency_init")
      import :: c_int, c_int32_t, c_float, c_ptr
      type(c_ptr), value :: ctx
      integer(c_int32_t), value :: irdamp
      real(c_float), value :: rdalpha
      real(c_float), intent(in) :: tauh(*), taus(*), tauf(*), uavg(*), vavg(*), thavg(*), ua(*), va(*), wa(*), tha(*)
      real(c_float), intent(inout) :: uten1(*), vten1(*), wten1(*), thten1(*), qten(*), ptten(*)
    end function
    type(c_ptr) function cm1g_last_error() bind(C, name="cm1g_last_error")
      import :: c_ptr
    end function
    ! 2nd-order diffusion: diff2def + diff2u/v/w/s of solve1 (difforder=2)
    integer(c_int) function cm1g_diff2(ctx, kdiff2, idiff, bbc, tbc, cgs, cgt, ua, va, wa, rho, tha, qa, pta, &
                                       uten1, vten1, wten1, thten1, qten, ptten) bind(C, name="cm1g_diff2")
      import :: c_int, c_int32_t, c_float, c_ptr
      type(c_ptr), value :: ctx
      real(c_float), value :: kdiff2
      integer(c_int32_t), value :: idiff, bbc, tbc
      real(c_float), intent(in) :: cgs(3), cgt(3)
      type(c_ptr), value :: ua, va, wa, rho, tha, qa, pta, uten1, vten1, wten1, thten1, qten, ptten
    end function
    ! Smagorinsky LES (sgsmodel=2): sfc_and_turb's closure + solve1's turb* tendencies
    integer(c_int) function cm1g_turbsmag(ctx, csm, tconfig, bcturbs, bbc, tbc, cgs, cgt, ua, va, wa, rho, tha, &
                                          qa, pta, uten1, vten1, wten1, thten1, qten, ptten, kmh, kmv) &
                                          bind(C, name="cm1g_turbsmag")
      import :: c_int, c_int32_t, c_float, c_ptr
      type(c_ptr), value :: ctx
      real(c_float), value :: csm
      integer(c_int32_t), value :: tconfig, bcturbs, bbc, tbc
      real(c_float), intent(in) :: cgs(3), cgt(3)
      type(c_ptr), value :: ua, va, wa, rho, tha, qa, pta, uten1, vten1, wten1, thten1, qten, ptten, kmh, kmv
    end function
    ! mp_driver's Kessler branch alone (ptype=1) and its FP64 budgets
    integer(c_int) function cm1g_mp_driver(ctx, dt, st) bind(C, name="cm1g_mp_driver")
      import :: c_int, c_float, c_ptr, cm1g_state_t
      type(c_ptr), value :: ctx
      real(c_float), value :: dt
      type(cm1g_state_t), intent(inout) :: st
    end function
    integer(c_int) function cm1g_mp_budget(ctx, qbudget, asq, reset) bind(C, name="cm1g_mp_budget")
      import :: c_int, c_int32_t, c_double, c_ptr
      type(c_ptr), value :: ctx
      real(c_double), intent(out) :: qbudget(7), asq(3)
      integer(c_int32_t), value :: reset
    end function
    ! records of output files (level by level, i fastest) and restart files
    integer(c_int) function cm1g_pack_records(ctx, n, fields, stag, k1, k2, out) bind(C, name="cm1g_pack_records")
      import :: c_int, c_int32_t, c_float, c_ptr
      type(c_ptr), value :: ctx
      integer(c_int32_t), value :: n
      type(c_ptr), intent(in) :: fields(*)
      integer(c_int32_t), intent(in) :: stag(*), k1(*), k2(*)
      real(c_float), intent(out) :: out(*)
    end function
    integer(c_int) function cm1g_writeout(ctx, prefix, nwrite, mtime, opts, st) bind(C, name="cm1g_writeout")
      import :: c_int, c_int32_t, c_double, c_char, c_ptr, cm1g_writeout_opts_t, cm1g_state_t
      type(c_ptr), value :: ctx
      character(kind=c_char), intent(in) :: prefix(*)
      integer(c_int32_t), value :: nwrite
      real(c_double), value :: mtime
      type(cm1g_writeout_opts_t), intent(in) :: opts
      type(cm1g_state_t), intent(in) :: st
    end function
    integer(c_int) function cm1g_restart_write(ctx, path, hdr, st) bind(C, name="cm1g_restart_write")
      import :: c_int, c_char, c_ptr, cm1g_restart_t, cm1g_state_t
      type(c_ptr), value :: ctx
      character(kind=c_char), intent(in) :: path(*)
      type(cm1g_restart_t), intent(in) :: hdr
      type(cm1g_state_t), intent(in) :: st
    end function
    integer(c_int) function cm1g_restart_read(ctx, path, hdr, st) bind(C, name="cm1g_restart_read")
      import :: c_int, c_char, c_ptr, cm1g_restart_t, cm1g_state_t
      type(c_ptr), value :: ctx
      character(kind=c_char), intent(in) :: path(*)
      type(cm1g_restart_t), intent(out) :: hdr
      type(cm1g_state_t), intent(inout) :: st
    end function
    ! statpack (statpack.F:10-658): set-up once, then one call per statfrq
    integer(c_int) function cm1g_stat_setup(ctx, opts, stat_out) bind(C, name="cm1g_stat_setup")
      import :: c_int, c_int32_t, c_ptr, cm1g_stat_opts_t
      type(c_ptr), value :: ctx
      type(cm1g_stat_opts_t), intent(in) :: opts
      integer(c_int32_t), intent(out) :: stat_out
    end function
    integer(c_int) function cm1g_statpack(ctx, mtime, dt, ua, va, wa, ppi, tha, prs, rho, qa, pta, prate, &
                                          qbudget, asq, bsq, rstat) bind(C, name="cm1g_statpack")
      import :: c_int, c_float, c_double, c_ptr
      type(c_ptr), value :: ctx
      real(c_double), value :: mtime
      real(c_float), value :: dt
      type(c_ptr), value :: ua, va, wa, ppi, tha, prs, rho, qa, pta, prate, qbudget, asq, bsq
      real(c_float), intent(out) :: rstat(*)
    end function
    integer(c_int) function cm1g_stat_write(path, nrec, rstat, nstat) bind(C, name="cm1g_stat_write")
      import :: c_int, c_int32_t, c_float, c_char
      character(kind=c_char), intent(in) :: path(*)
      integer(c_int32_t), value :: nrec, nstat
      real(c_float), intent(in) :: rstat(*)
    end function
    integer(c_int) function cm1g_set_tune(ctx, tune) bind(C, name="cm1g_set_tune")
      import :: c_int, c_ptr, cm1g_tune_t
      type(c_ptr), value :: ctx
      type(cm1g_tune_t), intent(in) :: tune
    end function
    integer(c_int) function cm1g_get_tune(ctx, tune) bind(C, name="cm1g_get_tune")
      import :: c_int, c_ptr, cm1g_tune_t
      type(c_ptr), value :: ctx
      type(cm1g_tune_t), intent(out) :: tune
    end function
    ! times the candidate launch shapes on a copy of st; cache_path: a
    ! NUL-terminated file name (c_loc of a character array) or c_null_ptr
    integer(c_int) function cm1g_autotune(ctx, dt, mass1, st, reps, cache_path, tune) bind(C, name="cm1g_autotune")
      import :: c_int, c_int32_t, c_float, c_double, c_ptr, cm1g_state_t, cm1g_tune_t
      type(c_ptr), value :: ctx
      real(c_float), value :: dt
      real(c_double), value :: mass1
      type(cm1g_state_t), intent(in) :: st
      integer(c_int32_t), value :: reps
      type(c_ptr), value :: cache_path
      type(cm1g_tune_t), intent(out) :: tune
    end function
  end interface

contains

  ! Message of the last failed call, as a Fortran string.
  function cm1g_last_error_f() result(msg)
    character(len=256) :: msg
    character(kind=c_char), pointer :: p(:)
    integer :: i
    msg = ' '
    call c_f_pointer(cm1g_last_error(), p, [256])
    do i = 1, 256
      if (p(i) == c_null_char) exit
      msg(i:i) = p(i)
    enddo
  end function

  ! Fill the configuration from module `input` and create the context
  ! (run once after param, base and init3d have set the base state).
  subroutine cm1g_setup(ctx, uh,ruh,uf,ruf,vh,rvh,vf,rvf, mh,rmh,c1,c2,mf,rmf, &
                        pi0,rho0,rr0,rf0,rrf0,th0,rth0,qv0,qc0,qi0,prs0, u0,v0, dtu0,dtv0, qmag)
    use input
    use constants, only : epsilon
    type(c_ptr), intent(out) :: ctx
    real, target, intent(in) :: uh(ib:ie),ruh(ib:ie),uf(ib:ie+1),ruf(ib:ie+1)
    real, target, intent(in) :: vh(jb:je),rvh(jb:je),vf(jb:je+1),rvf(jb:je+1)
    real, target, intent(in), dimension(ib:ie,jb:je,kb:ke) :: mh,rmh,c1,c2
    real, target, intent(in), dimension(ib:ie,jb:je,kb:ke+1) :: mf,rmf
    real, target, intent(in), dimension(ib:ie,jb:je,kb:ke) :: pi0,rho0,rr0,rf0,rrf0,th0,rth0,qv0,qc0,qi0,prs0
    real, target, intent(in) :: u0(ib:ie+1,jb:je,kb:ke), v0(ib:ie,jb:je+1,kb:ke)
    real, target, intent(in) :: dtu0(ib:ie,jb:je), dtv0(ib:ie,jb:je)
    real, intent(in) :: qmag(:)
    type(cm1g_config_t) :: cfg
    type(cm1g_grid_t) :: g
    integer :: rc, n
    cfg%ni = ni; cfg%nj = nj; cfg%nk = nk; cfg%ngxy = ngxy
    cfg%dx = dx; cfg%dy = dy; cfg%dz = dz
    cfg%wbc = wbc; cfg%ebc = ebc; cfg%sbc = sbc; cfg%nbc = nbc
    cfg%hadvordrs = hadvordrs; cfg%vadvordrs = vadvordrs
    cfg%hadvordrv = hadvordrv; cfg%vadvordrv = vadvordrv
    cfg%advwenos = advwenos; cfg%advwenov = advwenov; cfg%weno_order = weno_order
    cfg%nsound = nsound; cfg%alph = alph; cfg%kdiv = kdiv
    cfg%imoist = imoist; cfg%eqtset = eqtset; cfg%numq = numq; cfg%nqv = nqv
    cfg%iptra = iptra; cfg%npt = npt; cfg%pdtra = pdtra
    cfg%apmasscon = apmasscon; cfg%irbc = irbc; cfg%cstar = cstar; cfg%roflux = roflux
    cfg%smeps = smeps; cfg%testcase = testcase; cfg%psolver = psolver
    cfg%terrain_flag = merge(1, 0, terrain_flag); cfg%axisymm = axisymm; cfg%icor = icor
    cfg%idiff = idiff; cfg%difforder = difforder; cfg%mdiff = mdiff; cfg%kdiff6 = kdiff6
    cfg%ptype = ptype; cfg%nql1 = nql1; cfg%nql2 = nql2; cfg%efall = efall
    cfg%tsmall = tsmall; cfg%qsmall = qsmall
    cfg%qmag = 0.0
    do n = 1, min(size(qmag), int(CM1G_MAXQ))
      cfg%qmag(n) = qmag(n)
    enddo
    g%uh = c_loc(uh); g%ruh = c_loc(ruh); g%uf = c_loc(uf); g%ruf = c_loc(ruf)
    g%vh = c_loc(vh); g%rvh = c_loc(rvh); g%vf = c_loc(vf); g%rvf = c_loc(rvf)
    g%mh = c_loc(mh); g%rmh = c_loc(rmh); g%c1 = c_loc(c1); g%c2 = c_loc(c2)
    g%mf = c_loc(mf); g%rmf = c_loc(rmf)
    g%pi0 = c_loc(pi0); g%rho0 = c_loc(rho0); g%rr0 = c_loc(rr0); g%rf0 = c_loc(rf0)
    g%rrf0 = c_loc(rrf0); g%th0 = c_loc(th0); g%rth0 = c_loc(rth0); g%qv0 = c_loc(qv0)
    g%qc0 = c_loc(qc0); g%qi0 = c_loc(qi0); g%prs0 = c_loc(prs0)
    g%u0 = c_loc(u0); g%v0 = c_loc(v0); g%dtu0 = c_loc(dtu0); g%dtv0 = c_loc(dtv0)
    rc = cm1g_init(cfg, g, ctx)
    if (rc /= 0) then
      print *, ' cm1g_init failed: ', trim(cm1g_last_error_f())
      call stopcm1
    endif
  end subroutine

  ! One large step (solve2, then pdefq for qv (ptype=0) or mp_driver's
  ! Kessler branch (ptype=1), then solve3's dynamical-core part).
  subroutine cm1g_large_step(ctx, nstep, dt, mtime, mass1, mass2, cflmax, &
                             ua,u3d,uten1, va,v3d,vten1, wa,w3d,wten1,   &
                             ppi,pp3d,ppx,ppten, tha,th3d,thten1, rho,prs, &
                             qa,q3d,qten, pta,pt3d,ptten, radbcw,radbce,radbcs,radbcn, &
                             rain,prate)
    type(c_ptr), intent(in) :: ctx
    integer, intent(in) :: nstep
    real, intent(in) :: dt
    double precision, intent(in) :: mtime, mass1
    double precision, intent(out) :: mass2
    real, intent(out) :: cflmax
    real, target, intent(inout) :: ua(*),u3d(*),uten1(*),va(*),v3d(*),vten1(*),wa(*),w3d(*),wten1(*)
    real, target, intent(inout) :: ppi(*),pp3d(*),ppx(*),ppten(*),tha(*),th3d(*),thten1(*),rho(*),prs(*)
    real, target, intent(inout) :: qa(*),q3d(*),qten(*),pta(*),pt3d(*),ptten(*)
    real, target, intent(inout) :: radbcw(*),radbce(*),radbcs(*),radbcn(*)
    real, target, intent(inout) :: rain(*),prate(*)
    type(cm1g_state_t) :: s
    integer :: rc
    s%ua = c_loc(ua); s%u3d = c_loc(u3d); s%uten1 = c_loc(uten1)
    s%va = c_loc(va); s%v3d = c_loc(v3d); s%vten1 = c_loc(vten1)
    s%wa = c_loc(wa); s%w3d = c_loc(w3d); s%wten1 = c_loc(wten1)
    s%ppi = c_loc(ppi); s%pp3d = c_loc(pp3d); s%ppx = c_loc(ppx); s%ppten = c_loc(ppten)
    s%tha = c_loc(tha); s%th3d = c_loc(th3d); s%thten1 = c_loc(thten1)
    s%rho = c_loc(rho); s%prs = c_loc(prs)
    s%qa = c_loc(qa); s%q3d = c_loc(q3d); s%qten = c_loc(qten)
    s%pta = c_loc(pta); s%pt3d = c_loc(pt3d); s%ptten = c_loc(ptten)
    s%radbcw = c_loc(radbcw); s%radbce = c_loc(radbce); s%radbcs = c_loc(radbcs); s%radbcn = c_loc(radbcn)
    s%rain = c_loc(rain); s%prate = c_loc(prate)
    rc = cm1g_step(ctx, int(nstep, c_int32_t), dt, mtime, mass1, mass2, cflmax, s, 0_c_int32_t)
    if (rc /= 0) then
      print *, ' cm1g_step failed: ', trim(cm1g_last_error_f())
      call stopcm1
    endif
  end subroutine

end module cm1g_iso
