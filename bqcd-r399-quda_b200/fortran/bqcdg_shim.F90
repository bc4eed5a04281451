!===============================================================================
!
! bqcdg_shim.F90 - the Fortran side of the drop-in boundary between BQCD's
! HMC driver and libbqcdg.so (include/bqcdg.h), through iso_c_binding.
!
! Build: compile this file with BQCD's own flags and preprocessor (it
! includes defs.h) in place of invert_quda.F90 (Makefile:77), keep
! QUDA_SOLVER defined (defs.h:30), and link with
!   -L<repo>/bqcd-r399-quda_b200/lib -lbqcdg
! The five solver call sites (dsf1.F90:66, dsf2.F90:64, hmc_init_phi.F90:68,
! action.F90:55, traces.F90:142) then reach the B200 solver unchanged.
!
! Contents
!   module bqcdg_f      bind(c) mirrors of the structs of bqcdg.h and
!                       interface blocks of the entry points used here; the
!                       context (one per process, created on first use)
!   quda_solver         drop-in for invert_quda.F90:96 (same name, arguments)
!   bqcdg_f_cg          cg(matrix_mult, x, b, para, conf, iterations) of
!                       cg.F90:51 in FP64 on the device; the operator is
!                       w_dagger_w or mtdagmt, told apart by procedure
!                       association
!   bqcdg_f_dsf         dsf(p, conf, step, para, a, b) of dsf.F90:28
!   bqcdg_f_mtil ...    mtil, mtil_dag (m_tilde.F90:43,80), mtdagmt
!                       (mtdagmt.F90:28), w_mult, w_mult_dag, w_dagger_w
!                       (w_mult.F90:28,46,64) with their (out, in, para, conf)
!                       arguments, usable as matrix_mult
!
! Every bind(c) type below must match its C struct member for member; the
! CPU test tests/test_fortran_shim.py compares them with the compiled
! header's offsets and sizes.
!
! Links: BQCD calls every fermion routine on links bracketed by flip_bc()
! (flip_bc.F90:97-121), so they are uploaded with flipped = 1.  Like the
! QUDA hook (invert_quda.F90:134-138), links and clover are uploaded on every
! call.  Status codes are turned into die()/warn() as the reference does:
! no convergence dies unless cg_para%log == 2 (cg.F90:121-124).
!
!===============================================================================
# include "defs.h"

module bqcdg_f

  use iso_c_binding
  implicit none

  integer(c_int), parameter :: BQCDG_OK = 0
  integer(c_int), parameter :: BQCDG_ENOCONV = 3
  integer(c_int), parameter :: BQCDG_EUNSUPPORTED = 8
  integer(c_int), parameter :: BQCDG_PREC_DOUBLE = 0
  integer(c_int), parameter :: BQCDG_PREC_HALF = 2

  ! bqcdg_params
  type, bind(c) :: bqcdg_params
     real(c_double) :: kappa
     real(c_double) :: csw_kappa
     real(c_double) :: h
     real(c_double) :: rho
  end type bqcdg_params

  ! bqcdg_cg_para (type_cg_para of cg.F90:30-34)
  type, bind(c) :: bqcdg_cg_para
     real(c_float)  :: rest
     integer(c_int) :: maxiter
     integer(c_int) :: log
  end type bqcdg_cg_para

  ! bqcdg_solver_opts
  type, bind(c) :: bqcdg_solver_opts
     integer(c_int) :: precision
     integer(c_int) :: maxiter
     integer(c_int) :: relative
     real(c_double) :: tol
     real(c_double) :: delta
     integer(c_int) :: check_true_residual
     integer(c_int) :: time_kernels
     integer(c_int) :: rhs_per_thread
  end type bqcdg_solver_opts

  ! bqcdg_solve_info
  type, bind(c) :: bqcdg_solve_info
     integer(c_int) :: niter
     integer(c_int) :: reliable_updates
     real(c_double) :: rtr
     real(c_double) :: true_rtr
     real(c_double) :: b2
     real(c_double) :: seconds
     real(c_double) :: stencil_ms
     integer(c_int) :: stencil_launches
     integer(c_int) :: converged
     integer(c_int) :: kernel_launches
  end type bqcdg_solve_info

  ! bqcdg_conf_meta (the ConfInfoHeader fields of conf_info.F90:28-63)
  type, bind(c) :: bqcdg_conf_meta
     integer(c_int) :: run
     integer(c_int) :: traj
     integer(c_int) :: ensemble(2)
     real(c_double) :: beta(2)
     real(c_double) :: kappa(2)
     real(c_double) :: csw(2)
     real(c_double) :: csw_kappa(2)
     real(c_double) :: h(2)
     real(c_double) :: plaq_energy
     integer(c_int) :: L(4)
     integer(c_int) :: bc(4)
  end type bqcdg_conf_meta

  type(c_ptr), save :: bqcdg_context = c_null_ptr

  interface
     integer(c_int) function bqcdg_create(ctx, L, bc, device) bind(c, name = "bqcdg_create")
       import :: c_ptr, c_int
       type(c_ptr), intent(out) :: ctx
       integer(c_int), intent(in) :: L(4), bc(4)
       integer(c_int), value :: device
     end function bqcdg_create

     integer(c_int) function bqcdg_load_gauge(ctx, u, flipped) bind(c, name = "bqcdg_load_gauge")
       import :: c_ptr, c_int
       type(c_ptr), value :: ctx, u
       integer(c_int), value :: flipped
     end function bqcdg_load_gauge

     integer(c_int) function bqcdg_load_clover(ctx, a, ainv, b) bind(c, name = "bqcdg_load_clover")
       import :: c_ptr, c_int
       type(c_ptr), value :: ctx, a, ainv, b
     end function bqcdg_load_clover

     integer(c_int) function bqcdg_load_clover_solver(ctx, a, ainv) bind(c, name = "bqcdg_load_clover_solver")
       import :: c_ptr, c_int
       type(c_ptr), value :: ctx, a, ainv
     end function bqcdg_load_clover_solver

     integer(c_int) function bqcdg_quda_solver(ctx, x, b, p, cgp, iterations, info) &
          bind(c, name = "bqcdg_quda_solver")
       import :: c_ptr, c_int, bqcdg_params, bqcdg_cg_para, bqcdg_solve_info
       type(c_ptr), value :: ctx, x, b
       type(bqcdg_params), intent(in) :: p
       type(bqcdg_cg_para), intent(in) :: cgp
       integer(c_int), intent(out) :: iterations
       type(bqcdg_solve_info), intent(out) :: info
     end function bqcdg_quda_solver

     integer(c_int) function bqcdg_cg(ctx, x, b, p, cgp, iterations, info) bind(c, name = "bqcdg_cg")
       import :: c_ptr, c_int, bqcdg_params, bqcdg_cg_para, bqcdg_solve_info
       type(c_ptr), value :: ctx, x, b
       type(bqcdg_params), intent(in) :: p
       type(bqcdg_cg_para), intent(in) :: cgp
       integer(c_int), intent(out) :: iterations
       type(bqcdg_solve_info), intent(out) :: info
     end function bqcdg_cg

     integer(c_int) function bqcdg_solve(ctx, x, b, p, o, info) bind(c, name = "bqcdg_solve")
       import :: c_ptr, c_int, bqcdg_params, bqcdg_solver_opts, bqcdg_solve_info
       type(c_ptr), value :: ctx, x, b
       type(bqcdg_params), intent(in) :: p
       type(bqcdg_solver_opts), intent(in) :: o
       type(bqcdg_solve_info), intent(out) :: info
     end function bqcdg_solve

     integer(c_int) function bqcdg_dsf(ctx, p, step, par, a, b) bind(c, name = "bqcdg_dsf")
       import :: c_ptr, c_int, c_double, bqcdg_params
       type(c_ptr), value :: ctx, p, a, b
       real(c_double), value :: step
       type(bqcdg_params), intent(in) :: par
     end function bqcdg_dsf

     ! the six operators share one argument list
     integer(c_int) function bqcdg_mtil(ctx, out, in, p) bind(c, name = "bqcdg_mtil")
       import :: c_ptr, c_int, bqcdg_params
       type(c_ptr), value :: ctx, out, in
       type(bqcdg_params), intent(in) :: p
     end function bqcdg_mtil
     integer(c_int) function bqcdg_mtil_dag(ctx, out, in, p) bind(c, name = "bqcdg_mtil_dag")
       import :: c_ptr, c_int, bqcdg_params
       type(c_ptr), value :: ctx, out, in
       type(bqcdg_params), intent(in) :: p
     end function bqcdg_mtil_dag
     integer(c_int) function bqcdg_mtdagmt(ctx, out, in, p) bind(c, name = "bqcdg_mtdagmt")
       import :: c_ptr, c_int, bqcdg_params
       type(c_ptr), value :: ctx, out, in
       type(bqcdg_params), intent(in) :: p
     end function bqcdg_mtdagmt
     integer(c_int) function bqcdg_w_mult(ctx, out, in, p) bind(c, name = "bqcdg_w_mult")
       import :: c_ptr, c_int, bqcdg_params
       type(c_ptr), value :: ctx, out, in
       type(bqcdg_params), intent(in) :: p
     end function bqcdg_w_mult
     integer(c_int) function bqcdg_w_mult_dag(ctx, out, in, p) bind(c, name = "bqcdg_w_mult_dag")
       import :: c_ptr, c_int, bqcdg_params
       type(c_ptr), value :: ctx, out, in
       type(bqcdg_params), intent(in) :: p
     end function bqcdg_w_mult_dag
     integer(c_int) function bqcdg_w_dagger_w(ctx, out, in, p) bind(c, name = "bqcdg_w_dagger_w")
       import :: c_ptr, c_int, bqcdg_params
       type(c_ptr), value :: ctx, out, in
       type(bqcdg_params), intent(in) :: p
     end function bqcdg_w_dagger_w

     integer(c_int) function bqcdg_conf_write(ctx, base, meta) bind(c, name = "bqcdg_conf_write")
       import :: c_ptr, c_int, c_char, bqcdg_conf_meta
       type(c_ptr), value :: ctx
       character(kind = c_char), intent(in) :: base(*)
       type(bqcdg_conf_meta), intent(inout) :: meta
     end function bqcdg_conf_write
     integer(c_int) function bqcdg_conf_read(ctx, info, meta) bind(c, name = "bqcdg_conf_read")
       import :: c_ptr, c_int, c_char, bqcdg_conf_meta
       type(c_ptr), value :: ctx
       character(kind = c_char), intent(in) :: info(*)
       type(bqcdg_conf_meta), intent(inout) :: meta
     end function bqcdg_conf_read
  end interface

contains

  ! the process's context, created on first use (device 0 of the process's
  ! visible devices; one process per GPU)
  subroutine bqcdg_f_context()
    use module_lattice
    integer(c_int) :: st
    if (c_associated(bqcdg_context)) return
    st = bqcdg_create(bqcdg_context, int(L, c_int), int(bc_fermions, c_int), 0_c_int)
    call bqcdg_f_check(st, "bqcdg_create")
  end subroutine bqcdg_f_context

  subroutine bqcdg_f_check(st, routine)
    integer(c_int), intent(in) :: st
    character(len = *), intent(in) :: routine
    character(len = 100) :: msg
    if (st == BQCDG_OK) return
    write(msg, "(a, a, i3)") routine, "(): libbqcdg status ", st
    call die(msg)
  end subroutine bqcdg_f_check

  ! conf%u (flipped by the caller) and the clover parts the call reads
  subroutine bqcdg_f_upload(para, conf, solver_only)
    use typedef_hmc
    type(hmc_para), intent(in) :: para
    type(hmc_conf), intent(in) :: conf
    logical, intent(in) :: solver_only
    integer(c_int) :: st
    call bqcdg_f_context()
    st = bqcdg_load_gauge(bqcdg_context, c_loc(conf%u(1, 1, 1, 0, 1)), 1_c_int)
    call bqcdg_f_check(st, "bqcdg_load_gauge")
    if (para%csw_kappa /= ZERO) then
       if (solver_only) then
          st = bqcdg_load_clover_solver(bqcdg_context, c_loc(conf%a(1, 1, 0)), c_loc(conf%i(1, 1, 0)))
       else
          st = bqcdg_load_clover(bqcdg_context, c_loc(conf%a(1, 1, 0)), c_loc(conf%i(1, 1, 0)), &
                                 c_loc(conf%b(1, 1, 0)))
       endif
       call bqcdg_f_check(st, "bqcdg_load_clover")
    endif
  end subroutine bqcdg_f_upload

  ! statistics exactly as cg.F90:128-132 and invert_quda.F90:178-186
  subroutine bqcdg_f_count(niter)
    use module_cg
    integer, intent(in) :: niter
    cg_stat%ncall = cg_stat%ncall + 1
    cg_stat%niter = niter
    cg_stat%niter_max = max(cg_stat%niter_max, niter)
    cg_stat%niter_tot = cg_stat%niter_tot + niter
    cg_iterations_total = cg_iterations_total + niter
  end subroutine bqcdg_f_count

end module bqcdg_f

!-------------------------------------------------------------------------------
! drop-in for invert_quda.F90:96: mixed-precision CG on the device (int16
! sloppy fields, FP64 reliable updates), absolute stop rtr <= cg_para%rest,
! FP64 true residual checked on the device (invert_quda.F90:155-168 checks it
! on the host with matrix_mult).  rho selects the operator: (M~+rho)^+(M~+rho),
! mtdagmt for rho = 0.  h /= 0 is refused as by the QUDA hook
! (invert_quda.F90:298-301).
!-------------------------------------------------------------------------------
subroutine quda_solver(matrix_mult, x, b, para, conf, iterations, rho)

  use bqcdg_f
  use module_cg
  use typedef_hmc
  implicit none

  external                                  :: matrix_mult
  SPINCOL_OVERINDEXED, intent(out), target  :: x
  SPINCOL_OVERINDEXED, intent(in),  target  :: b
  type(hmc_para),       intent(in)          :: para
  type(hmc_conf),       intent(in)          :: conf
  integer,              intent(out)         :: iterations
  REAL,                 intent(in)          :: rho

  type(bqcdg_params)     :: p
  type(bqcdg_cg_para)    :: cgp
  type(bqcdg_solve_info) :: info
  integer(c_int)         :: st, it
  character(len = 72)    :: msg

  call bqcdg_f_upload(para, conf, .true.)
  p = bqcdg_params(para%kappa, para%csw_kappa, para%h, rho)
  cgp = bqcdg_cg_para(real(cg_para%rest, c_float), int(cg_para%maxiter, c_int), int(cg_para%log, c_int))
  st = bqcdg_quda_solver(bqcdg_context, c_loc(x), c_loc(b), p, cgp, it, info)
  if (st == BQCDG_ENOCONV) then
     write(msg, *) "cg(): no convergence; rtr = ", info%true_rtr
     call die(msg)
  endif
  if (st == BQCDG_EUNSUPPORTED) call die("quda_solver(): h /= 0 is not supported")
  call bqcdg_f_check(st, "quda_solver")
  iterations = it
  call bqcdg_f_count(iterations)

end subroutine quda_solver

!-------------------------------------------------------------------------------
! cg.F90:51 on the device, all FP64 with the reference's iterates: x is the
! initial guess on entry; matrix_mult is w_dagger_w (rho = para%rho) or
! mtdagmt (rho = 0).
!-------------------------------------------------------------------------------
subroutine bqcdg_f_cg(matrix_mult, x, b, para, conf, iterations)

  use bqcdg_f
  use module_cg
  use typedef_hmc
  implicit none

  external                                  :: matrix_mult
  SPINCOL_OVERINDEXED, intent(inout), target :: x
  SPINCOL_OVERINDEXED, intent(in),  target  :: b
  type(hmc_para),       intent(in)          :: para
  type(hmc_conf),       intent(in)          :: conf
  integer,              intent(out)         :: iterations

  external                  :: w_dagger_w
  procedure(), pointer      :: mm
  type(bqcdg_params)        :: p
  type(bqcdg_cg_para)       :: cgp
  type(bqcdg_solve_info)    :: info
  integer(c_int)            :: st, it
  REAL                      :: rho
  character(len = 72)       :: msg

  mm => matrix_mult
  rho = ZERO
  if (associated(mm, w_dagger_w)) rho = para%rho

  call bqcdg_f_upload(para, conf, .true.)
  p = bqcdg_params(para%kappa, para%csw_kappa, para%h, rho)
  cgp = bqcdg_cg_para(real(cg_para%rest, c_float), int(cg_para%maxiter, c_int), int(cg_para%log, c_int))
  st = bqcdg_cg(bqcdg_context, c_loc(x), c_loc(b), p, cgp, it, info)
  if (st == BQCDG_ENOCONV) then
     write(msg, *) "cg(): no convergence; rtr = ", info%rtr
     call die(msg)
  endif
  call bqcdg_f_check(st, "cg")
  iterations = it
  call bqcdg_f_count(iterations)

end subroutine bqcdg_f_cg

!-------------------------------------------------------------------------------
! dsf.F90:28: p += the pseudofermion force of the even fields a, b (hopping
! part and, for csw /= 0, the clover part), links flipped by the caller.
!-------------------------------------------------------------------------------
subroutine bqcdg_f_dsf(p, conf, step, para, a, b)

  use bqcdg_f
  use typedef_hmc
  implicit none

  type(hmc_para),  intent(in)            :: para
  type(hmc_conf),  intent(in)            :: conf
  GENERATOR_FIELD, intent(inout), target :: p
  REAL,            intent(in)            :: step
  SPINCOL_FIELD,   intent(in), target    :: a
  SPINCOL_FIELD,   intent(in), target    :: b

  type(bqcdg_params) :: par
  integer(c_int)     :: st

  call bqcdg_f_upload(para, conf, .false.)
  par = bqcdg_params(para%kappa, para%csw_kappa, para%h, para%rho)
  st = bqcdg_dsf(bqcdg_context, c_loc(p), real(step, c_double), par, c_loc(a), c_loc(b))
  call bqcdg_f_check(st, "dsf")

end subroutine bqcdg_f_dsf

!-------------------------------------------------------------------------------
! the operators with the reference's (out, in, para, conf) arguments
!-------------------------------------------------------------------------------
! mtil, m_tilde.F90:43
subroutine bqcdg_f_mtil(out, in, para, conf)

  use bqcdg_f
  use typedef_hmc
  implicit none

  SPINCOL_FIELD,  intent(out), target :: out
  SPINCOL_FIELD,  intent(in),  target :: in
  type(hmc_para), intent(in)          :: para
  type(hmc_conf), intent(in)          :: conf
  integer(c_int)                      :: st

  call bqcdg_f_upload(para, conf, .true.)
  st = bqcdg_mtil(bqcdg_context, c_loc(out), c_loc(in), &
       bqcdg_params(para%kappa, para%csw_kappa, para%h, para%rho))
  call bqcdg_f_check(st, "mtil")

end subroutine bqcdg_f_mtil

! mtil_dag, m_tilde.F90:80
subroutine bqcdg_f_mtil_dag(out, in, para, conf)

  use bqcdg_f
  use typedef_hmc
  implicit none

  SPINCOL_FIELD,  intent(out), target :: out
  SPINCOL_FIELD,  intent(in),  target :: in
  type(hmc_para), intent(in)          :: para
  type(hmc_conf), intent(in)          :: conf
  integer(c_int)                      :: st

  call bqcdg_f_upload(para, conf, .true.)
  st = bqcdg_mtil_dag(bqcdg_context, c_loc(out), c_loc(in), &
       bqcdg_params(para%kappa, para%csw_kappa, para%h, para%rho))
  call bqcdg_f_check(st, "mtil_dag")

end subroutine bqcdg_f_mtil_dag

! mtdagmt, mtdagmt.F90:28
subroutine bqcdg_f_mtdagmt(out, in, para, conf)

  use bqcdg_f
  use typedef_hmc
  implicit none

  SPINCOL_FIELD,  intent(out), target :: out
  SPINCOL_FIELD,  intent(in),  target :: in
  type(hmc_para), intent(in)          :: para
  type(hmc_conf), intent(in)          :: conf
  integer(c_int)                      :: st

  call bqcdg_f_upload(para, conf, .true.)
  st = bqcdg_mtdagmt(bqcdg_context, c_loc(out), c_loc(in), &
       bqcdg_params(para%kappa, para%csw_kappa, para%h, para%rho))
  call bqcdg_f_check(st, "mtdagmt")

end subroutine bqcdg_f_mtdagmt

! w_mult, w_mult.F90:28
subroutine bqcdg_f_w_mult(out, in, para, conf)

  use bqcdg_f
  use typedef_hmc
  implicit none

  SPINCOL_FIELD,  intent(out), target :: out
  SPINCOL_FIELD,  intent(in),  target :: in
  type(hmc_para), intent(in)          :: para
  type(hmc_conf), intent(in)          :: conf
  integer(c_int)                      :: st

  call bqcdg_f_upload(para, conf, .true.)
  st = bqcdg_w_mult(bqcdg_context, c_loc(out), c_loc(in), &
       bqcdg_params(para%kappa, para%csw_kappa, para%h, para%rho))
  call bqcdg_f_check(st, "w_mult")

end subroutine bqcdg_f_w_mult

! w_mult_dag, w_mult.F90:46
subroutine bqcdg_f_w_mult_dag(out, in, para, conf)

  use bqcdg_f
  use typedef_hmc
  implicit none

  SPINCOL_FIELD,  intent(out), target :: out
  SPINCOL_FIELD,  intent(in),  target :: in
  type(hmc_para), intent(in)          :: para
  type(hmc_conf), intent(in)          :: conf
  integer(c_int)                      :: st

  call bqcdg_f_upload(para, conf, .true.)
  st = bqcdg_w_mult_dag(bqcdg_context, c_loc(out), c_loc(in), &
       bqcdg_params(para%kappa, para%csw_kappa, para%h, para%rho))
  call bqcdg_f_check(st, "w_mult_dag")

end subroutine bqcdg_f_w_mult_dag

! w_dagger_w, w_mult.F90:64
subroutine bqcdg_f_w_dagger_w(out, in, para, conf)

  use bqcdg_f
  use typedef_hmc
  implicit none

  SPINCOL_FIELD,  intent(out), target :: out
  SPINCOL_FIELD,  intent(in),  target :: in
  type(hmc_para), intent(in)          :: para
  type(hmc_conf), intent(in)          :: conf
  integer(c_int)                      :: st

  call bqcdg_f_upload(para, conf, .true.)
  st = bqcdg_w_dagger_w(bqcdg_context, c_loc(out), c_loc(in), &
       bqcdg_params(para%kappa, para%csw_kappa, para%h, para%rho))
  call bqcdg_f_check(st, "w_dagger_w")

end subroutine bqcdg_f_w_dagger_w
