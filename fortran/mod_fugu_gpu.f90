! ==============================================================================
! mod_fugu_gpu -- ISO_C_BINDING bridge from the FUGU-2D Fortran code to the
! B200 library libfugu_gpu.so (C ABI: include/fugu_gpu.h).
!
! It goes beside the reference's modules in src/ and is wired in by
! use_gpu.patch (this directory):
!   * main.f90 gains the namelist key use_gpu (default .false.) and releases
!     the device context at the end of the run;
!   * advance_coupled_step (src/mod_solver_coupled.f90:137) starts with a
!     branch that, when use_gpu is set, hands the whole step to
!     gpu_advance_coupled_step below and returns.
!
! gpu_advance_coupled_step takes exactly advance_coupled_step's dummy
! arguments (same names, shapes, optional arguments), so the branch forwards
! its own arguments unchanged; absent optional arguments stay absent.  The
! device context is created by the first call from the module globals of
! mod_params and mod_mpi (one MPI rank: the whole domain stays on one GPU).
! Later calls refresh its parameters when those globals have changed.
! Extension knobs of the library (mixed precision, flexible GMRES, ...) are
! set in gpu_knobs after "call gpu_defaults()" and before the first step;
! fields that mirror reference globals are always overwritten from them.
!
! Arrays pass by the address of their lower-bound element, column-major with
! nh = 2 ghost layers, as the C ABI expects; the dummies carry the target
! attribute so that c_loc is valid for the duration of the call.
! ==============================================================================
module mod_fugu_gpu
  use, intrinsic :: iso_c_binding
  use mod_precision, only: dp, ip
  use mod_params,    only: rho1, rho2, mu1, mu2, sigma, gx, gy, cfl_target, alpha_penalty, &
                           time_order, tol_bicgstab2, max_iter_bicgstab2
  use mod_mpi,       only: dx_grid, dy_grid, periods, dims
  implicit none
  private

  public :: use_gpu, gpu_device, gpu_knobs, gpu_defaults, gpu_advance_coupled_step, gpu_finalize
  public :: fugu_params, fugu_step_opts, fugu_stats

  ! fugu_params (include/fugu_gpu.h) -- field order must match the C struct
  type, bind(C) :: fugu_params
    integer(c_int)  :: nx, ny
    real(c_double)  :: dx, dy
    integer(c_int)  :: periodic_x, periodic_y
    real(c_double)  :: rho1, rho2, mu1, mu2, sigma, gx, gy
    real(c_double)  :: cfl_target, alpha_penalty
    integer(c_int)  :: time_order
    real(c_double)  :: tol_bicgstab2
    integer(c_int)  :: max_iter_bicgstab2
    real(c_double)  :: pcg_tol
    integer(c_int)  :: pcg_max_iter, pcd_sweeps
    real(c_double)  :: jacobi_omega, svof_delta_h
    integer(c_int)  :: svof_max_iter
    real(c_double)  :: svof_tol
    integer(c_int)  :: limiter, free_slip_x, krylov_bc_fix, refine
    real(c_double)  :: refine_inner_tol
    integer(c_int)  :: refine_max_inner, refine_max_outer, precision, pcg_cap_start, &
                       pcd_sweeps_max, pcd_smoother
    real(c_double)  :: pcd_sor_omega
    integer(c_int)  :: graphs
    real(c_double)  :: pcd_visc_scale
    integer(c_int)  :: vec_rows
  end type
  ! fugu_step_opts: advance_coupled_step's optional arguments, has_* = present()
  type, bind(C) :: fugu_step_opts
    integer(c_int) :: use_bicgstab2, has_lid
    real(c_double) :: u_top_lid
    integer(c_int) :: has_tol
    real(c_double) :: tol
    integer(c_int) :: has_max_iter, max_iter, consistent_amp, has_penalty, has_u_solid
    real(c_double) :: u_solid
    integer(c_int) :: has_v_solid
    real(c_double) :: v_solid
  end type
  type, bind(C) :: fugu_stats
    integer(c_int)       :: iter
    real(c_double)       :: res
    integer(c_long_long) :: pcg_iters
    integer(c_int)       :: pcg_calls, svof_iters, matvecs, outer, status
  end type

  interface
    subroutine fugu_params_default(p) bind(C, name="fugu_params_default")
      import :: fugu_params
      type(fugu_params), intent(out) :: p
    end subroutine
    integer(c_int) function fugu_create(p, device, ctx) bind(C, name="fugu_create")
      import :: c_int, c_ptr, fugu_params
      type(fugu_params), intent(in) :: p
      integer(c_int), value :: device
      type(c_ptr), intent(out) :: ctx
    end function
    integer(c_int) function fugu_set_params(ctx, p) bind(C, name="fugu_set_params")
      import :: c_int, c_ptr, fugu_params
      type(c_ptr), value :: ctx
      type(fugu_params), intent(in) :: p
    end function
    subroutine fugu_destroy(ctx) bind(C, name="fugu_destroy")
      import :: c_ptr
      type(c_ptr), value :: ctx
    end subroutine
    type(c_ptr) function fugu_last_error(ctx) bind(C, name="fugu_last_error")
      import :: c_ptr
      type(c_ptr), value :: ctx
    end function
    integer(c_int) function fugu_advance_coupled_step(ctx, u_vel, v_vel, p_field, c_field, &
        u_prev, v_prev, rho_c, rho_u, rho_v, kappa, zeta, eta, kappa_curv, f_sigma_u, &
        f_sigma_v, phi_s_u, phi_s_v, dt, step_idx, opts, stats) bind(C, name="fugu_advance_coupled_step")
      import :: c_int, c_ptr, c_double, fugu_step_opts, fugu_stats
      type(c_ptr), value :: ctx, u_vel, v_vel, p_field, c_field, u_prev, v_prev, rho_c, rho_u, rho_v
      type(c_ptr), value :: kappa, zeta, eta, kappa_curv, f_sigma_u, f_sigma_v, phi_s_u, phi_s_v
      real(c_double), value :: dt
      integer(c_int), value :: step_idx
      type(fugu_step_opts), intent(in) :: opts
      type(fugu_stats), intent(out) :: stats
    end function
  end interface

  logical, save            :: use_gpu = .false.   ! namelist key of main.f90
  integer(c_int), save     :: gpu_device = 0      ! CUDA device of the context
  type(fugu_params), save  :: gpu_knobs           ! extension knobs (gpu_defaults first)
  logical, save            :: knobs_ready = .false.
  type(c_ptr), save        :: gpu_ctx = c_null_ptr
  type(fugu_params), save  :: ctx_params           ! parameters the context holds

contains

  ! The library's defaults in gpu_knobs (the reference's module defaults and
  ! call-site constants, every extension off).  Idempotent.
  subroutine gpu_defaults()
    if (.not. knobs_ready) then
      call fugu_params_default(gpu_knobs)
      knobs_ready = .true.
    end if
  end subroutine gpu_defaults

  ! gpu_knobs with the reference's globals written over their mirrors
  subroutine current_params(nx, ny, p)
    integer(ip), intent(in) :: nx, ny
    type(fugu_params), intent(out) :: p
    call gpu_defaults()
    p = gpu_knobs
    p%nx = nx
    p%ny = ny
    p%dx = dx_grid
    p%dy = dy_grid
    p%periodic_x = merge(1_c_int, 0_c_int, periods(1))
    p%periodic_y = merge(1_c_int, 0_c_int, periods(2))
    p%rho1 = rho1
    p%rho2 = rho2
    p%mu1 = mu1
    p%mu2 = mu2
    p%sigma = sigma
    p%gx = gx
    p%gy = gy
    p%cfl_target = cfl_target
    p%alpha_penalty = alpha_penalty
    p%time_order = time_order
    p%tol_bicgstab2 = tol_bicgstab2
    p%max_iter_bicgstab2 = max_iter_bicgstab2
  end subroutine current_params

  ! stop with the library's message when a call failed
  subroutine check(rc, what)
    integer(c_int), intent(in) :: rc
    character(len=*), intent(in) :: what
    character(kind=c_char), pointer :: msg(:)
    character(len=512) :: text
    integer :: k
    if (rc == 0) return
    text = ''
    if (c_associated(gpu_ctx)) then
      call c_f_pointer(fugu_last_error(gpu_ctx), msg, [512])
      do k = 1, 512
        if (msg(k) == c_null_char) exit
        text(k:k) = msg(k)
      end do
    end if
    write(*, '(A,A,I0,A,A)') what, ' failed (status ', rc, '): ', trim(text)
    error stop 'mod_fugu_gpu: GPU call failed'
  end subroutine check

  ! advance_coupled_step (src/mod_solver_coupled.f90:137-380) on the GPU: the
  ! same dummy arguments; the state is uploaded, stepped and downloaded by
  ! fugu_advance_coupled_step.
  subroutine gpu_advance_coupled_step(u_vel, v_vel, p_field, c_field, &
                                      u_prev, v_prev, &
                                      rho_c, rho_u, rho_v, kappa, zeta, eta, &
                                      kappa_curv, f_sigma_u, f_sigma_v, &
                                      dt_step, step_idx, nx, ny, nh, &
                                      iter_out, res_out, use_bicgstab2, u_top_lid, &
                                      tol_in, max_iter_in, &
                                      consistent_amp, phi_s_u, phi_s_v, u_solid_in, v_solid_in)
    integer(ip), intent(in) :: step_idx, nx, ny, nh
    real(dp), intent(in) :: dt_step
    real(dp), dimension(0-nh:nx+nh, 1-nh:ny+nh), intent(inout), target :: u_vel, u_prev
    real(dp), dimension(1-nh:nx+nh, 0-nh:ny+nh), intent(inout), target :: v_vel, v_prev
    real(dp), dimension(1-nh:nx+nh, 1-nh:ny+nh), intent(inout), target :: p_field, c_field
    real(dp), dimension(1-nh:nx+nh, 1-nh:ny+nh), intent(inout), target :: rho_c, kappa, kappa_curv
    real(dp), dimension(0-nh:nx+nh, 1-nh:ny+nh), intent(inout), target :: rho_u, f_sigma_u
    real(dp), dimension(1-nh:nx+nh, 0-nh:ny+nh), intent(inout), target :: rho_v, f_sigma_v
    real(dp), dimension(0-nh:nx+nh, 0-nh:ny+nh), intent(inout), target :: zeta, eta
    integer(ip), optional, intent(out) :: iter_out
    real(dp), optional, intent(out)    :: res_out
    logical, optional, intent(in)      :: use_bicgstab2, consistent_amp
    real(dp), optional, intent(in)     :: u_top_lid, tol_in, u_solid_in, v_solid_in
    integer(ip), optional, intent(in)  :: max_iter_in
    real(dp), dimension(0-nh:nx+nh, 1-nh:ny+nh), optional, intent(in), target :: phi_s_u
    real(dp), dimension(1-nh:nx+nh, 0-nh:ny+nh), optional, intent(in), target :: phi_s_v

    type(fugu_params) :: p
    type(fugu_step_opts) :: opts
    type(fugu_stats) :: stats
    type(c_ptr) :: pen_u, pen_v
    integer(c_signed_char) :: mold(1)

    if (nh /= 2) error stop 'mod_fugu_gpu: the GPU path needs nh = 2 ghost layers'
    if (product(dims) /= 1) error stop 'mod_fugu_gpu: the GPU path runs the whole domain on one rank'
    call current_params(nx, ny, p)
    if (.not. c_associated(gpu_ctx)) then
      call check(fugu_create(p, gpu_device, gpu_ctx), 'fugu_create')
      ctx_params = p
    else if (any(transfer(p, mold) /= transfer(ctx_params, mold))) then
      call check(fugu_set_params(gpu_ctx, p), 'fugu_set_params')
      ctx_params = p
    end if

    ! optional arguments: has_* mirrors present() (mod_solver_coupled.f90:175-194)
    opts%use_bicgstab2 = 1
    if (present(use_bicgstab2)) opts%use_bicgstab2 = merge(1_c_int, 0_c_int, use_bicgstab2)
    opts%has_lid = merge(1_c_int, 0_c_int, present(u_top_lid))
    opts%u_top_lid = 0.0_c_double
    if (present(u_top_lid)) opts%u_top_lid = u_top_lid
    opts%has_tol = merge(1_c_int, 0_c_int, present(tol_in))
    opts%tol = 0.0_c_double
    if (present(tol_in)) opts%tol = tol_in
    opts%has_max_iter = merge(1_c_int, 0_c_int, present(max_iter_in))
    opts%max_iter = 0
    if (present(max_iter_in)) opts%max_iter = max_iter_in
    opts%consistent_amp = 0
    if (present(consistent_amp)) opts%consistent_amp = merge(1_c_int, 0_c_int, consistent_amp)
    opts%has_penalty = merge(1_c_int, 0_c_int, present(phi_s_u) .and. present(phi_s_v))
    opts%has_u_solid = merge(1_c_int, 0_c_int, present(u_solid_in))
    opts%u_solid = 0.0_c_double
    if (present(u_solid_in)) opts%u_solid = u_solid_in
    opts%has_v_solid = merge(1_c_int, 0_c_int, present(v_solid_in))
    opts%v_solid = 0.0_c_double
    if (present(v_solid_in)) opts%v_solid = v_solid_in
    pen_u = c_null_ptr
    pen_v = c_null_ptr
    if (opts%has_penalty == 1) then
      pen_u = c_loc(phi_s_u(0-nh, 1-nh))
      pen_v = c_loc(phi_s_v(1-nh, 0-nh))
    end if

    call check(fugu_advance_coupled_step(gpu_ctx, &
               c_loc(u_vel(0-nh, 1-nh)), c_loc(v_vel(1-nh, 0-nh)), &
               c_loc(p_field(1-nh, 1-nh)), c_loc(c_field(1-nh, 1-nh)), &
               c_loc(u_prev(0-nh, 1-nh)), c_loc(v_prev(1-nh, 0-nh)), &
               c_loc(rho_c(1-nh, 1-nh)), c_loc(rho_u(0-nh, 1-nh)), c_loc(rho_v(1-nh, 0-nh)), &
               c_loc(kappa(1-nh, 1-nh)), c_loc(zeta(0-nh, 0-nh)), c_loc(eta(0-nh, 0-nh)), &
               c_loc(kappa_curv(1-nh, 1-nh)), c_loc(f_sigma_u(0-nh, 1-nh)), &
               c_loc(f_sigma_v(1-nh, 0-nh)), pen_u, pen_v, &
               real(dt_step, c_double), int(step_idx, c_int), opts, stats), &
               'fugu_advance_coupled_step')
    if (present(iter_out)) iter_out = stats%iter
    if (present(res_out))  res_out  = stats%res
  end subroutine gpu_advance_coupled_step

  ! release the device context (end of run); a later step creates a new one
  subroutine gpu_finalize()
    if (c_associated(gpu_ctx)) call fugu_destroy(gpu_ctx)
    gpu_ctx = c_null_ptr
  end subroutine gpu_finalize

end module mod_fugu_gpu
