! iso_c_binding interface to libdiablo_gpu (include/diablo_gpu.h) for the
! reference's Fortran driver.  Every entry point of the header is bound here
! under its C name; the diablo_params type matches the C struct field by
! field (kinds and order), and the constants match the header's enums.
!
! Argument conventions:
!   - a context or ensemble handle is type(c_ptr), passed by value;
!   - arrays that may live on the host or the device (state buffers, the
!     transforms' v and vv) are type(c_ptr) by value, so a caller passes
!     c_loc(array) for a host array or a device address it holds;
!   - host-only inputs and outputs (the grid gy, statistics, times, tiles) are
!     plain Fortran arguments by reference.
! Drop-in use (the reference's for/fft.f90:247,319 and for/diablo.f90:104-107)
! is shown in INTEGRATION.md.
module diablo_gpu
  use, intrinsic :: iso_c_binding
  implicit none

  integer(c_int), parameter :: DIABLO_ABI_VERSION = 1
  integer(c_int), parameter :: DIABLO_MAX_TH = 8

  ! status codes (enum diablo_status)
  integer(c_int), parameter :: DIABLO_OK = 0
  integer(c_int), parameter :: DIABLO_ERR_ARG = -1
  integer(c_int), parameter :: DIABLO_ERR_SIZE = -2
  integer(c_int), parameter :: DIABLO_ERR_CUDA = -3
  integer(c_int), parameter :: DIABLO_ERR_NONFINITE = -4
  integer(c_int), parameter :: DIABLO_ERR_TIMEOUT = -5
  integer(c_int), parameter :: DIABLO_ERR_UNSUPPORTED = -6
  integer(c_int), parameter :: DIABLO_ERR_STATE = -7
  integer(c_int), parameter :: DIABLO_ERR_NOMEM = -8

  ! precision (enum diablo_precision)
  integer(c_int), parameter :: DIABLO_FP64 = 0
  integer(c_int), parameter :: DIABLO_MIXED = 1

  ! fields (enum diablo_field): scalar n is DIABLO_TH + n
  integer(c_int), parameter :: DIABLO_U1 = 0
  integer(c_int), parameter :: DIABLO_U2 = 1
  integer(c_int), parameter :: DIABLO_U3 = 2
  integer(c_int), parameter :: DIABLO_P = 3
  integer(c_int), parameter :: DIABLO_TH = 4

  ! buffer layouts (enum diablo_layout)
  integer(c_int), parameter :: DIABLO_LAYOUT_FOURIER = 0
  integer(c_int), parameter :: DIABLO_LAYOUT_PHYSICAL = 1
  ! ensemble stepping modes
  integer(c_int), parameter :: DIABLO_ENSEMBLE_BRANCHES = 0
  integer(c_int), parameter :: DIABLO_ENSEMBLE_PERSISTENT = 1

  ! Run parameters: field order and kinds exactly as struct diablo_params.
  type, bind(C) :: diablo_params
    integer(c_int) :: struct_size
    integer(c_int) :: nx, ny, nz, n_th
    real(c_double) :: lx, ly, lz
    real(c_double) :: re, nu_v_scale, beta, ro, delta
    real(c_double) :: grav_x, grav_y, grav_z
    real(c_double) :: delta_t
    integer(c_int) :: f_type
    real(c_double) :: ubulk0, px0, omega0, amp_omega0, force_start
    integer(c_int) :: u_bc_ymin, v_bc_ymin, w_bc_ymin, u_bc_ymax, v_bc_ymax, w_bc_ymax
    real(c_double) :: u_bc_ymin_c1, v_bc_ymin_c1, w_bc_ymin_c1
    real(c_double) :: u_bc_ymax_c1, v_bc_ymax_c1, w_bc_ymax_c1
    real(c_double) :: pr(DIABLO_MAX_TH), ri(DIABLO_MAX_TH)
    integer(c_int) :: th_bc_ymin(DIABLO_MAX_TH), th_bc_ymax(DIABLO_MAX_TH)
    real(c_double) :: th_bc_ymin_c1(DIABLO_MAX_TH), th_bc_ymax_c1(DIABLO_MAX_TH)
    real(c_double) :: dthdx(DIABLO_MAX_TH), dthdz(DIABLO_MAX_TH)
    integer(c_int) :: use_les, les_model_type, create_new_flow
    integer(c_int) :: variable_dt
    real(c_double) :: cfl
    integer(c_int) :: update_dt
    real(c_double) :: max_dt
    integer(c_int) :: precision
    integer(c_int) :: flavor_front
    integer(c_int) :: filter_th(DIABLO_MAX_TH)
    integer(c_int) :: filter_int(DIABLO_MAX_TH)
  end type diablo_params

  interface
    ! ---- context lifetime (read_inputs, init_mpi, create_grid_chan, init_flow, init_fft)
    function diablo_create(p, gy, status) bind(C, name="diablo_create")
      import :: c_ptr, c_double, c_int, diablo_params
      type(diablo_params), intent(in) :: p
      real(c_double), intent(in) :: gy(*)
      integer(c_int), intent(out) :: status
      type(c_ptr) :: diablo_create
    end function diablo_create
    function diablo_destroy(ctx) bind(C, name="diablo_destroy")
      import :: c_ptr, c_int
      type(c_ptr), value :: ctx
      integer(c_int) :: diablo_destroy
    end function diablo_destroy

    ! ---- state in the reference layout (host or device buffers)
    function diablo_upload_state(ctx, field, buf, layout) bind(C, name="diablo_upload_state")
      import :: c_ptr, c_int
      type(c_ptr), value :: ctx, buf
      integer(c_int), value :: field, layout
      integer(c_int) :: diablo_upload_state
    end function diablo_upload_state
    function diablo_download_state(ctx, field, buf, layout) bind(C, name="diablo_download_state")
      import :: c_ptr, c_int
      type(c_ptr), value :: ctx, buf
      integer(c_int), value :: field, layout
      integer(c_int) :: diablo_download_state
    end function diablo_download_state
    function diablo_download_nu_t(ctx, buf) bind(C, name="diablo_download_nu_t")
      import :: c_ptr, c_int
      type(c_ptr), value :: ctx, buf
      integer(c_int) :: diablo_download_nu_t
    end function diablo_download_nu_t

    ! ---- for/fft.f90:247 and :319 (v == vv allowed)
    function diablo_fft_xz_to_fourier(ctx, v, vv) bind(C, name="diablo_fft_xz_to_fourier")
      import :: c_ptr, c_int
      type(c_ptr), value :: ctx, v, vv
      integer(c_int) :: diablo_fft_xz_to_fourier
    end function diablo_fft_xz_to_fourier
    function diablo_fft_xz_to_physical(ctx, vv, v) bind(C, name="diablo_fft_xz_to_physical")
      import :: c_ptr, c_int
      type(c_ptr), value :: ctx, vv, v
      integer(c_int) :: diablo_fft_xz_to_physical
    end function diablo_fft_xz_to_physical
    ! the forward transform without a context, for callers that cannot
    ! allocate device memory (device arrays only)
    function diablo_fft_xz_to_fourier_noalloc(nx, ny, nz, v, vv, stream) &
        bind(C, name="diablo_fft_xz_to_fourier_noalloc")
      import :: c_ptr, c_int
      integer(c_int), value :: nx, ny, nz
      type(c_ptr), value :: v, vv, stream
      integer(c_int) :: diablo_fft_xz_to_fourier_noalloc
    end function diablo_fft_xz_to_fourier_noalloc

    ! ---- the step (for/channel.f90:10, for/diablo.f90:98-108, for/advance.f90:17)
    function diablo_rk_substep(ctx, rk_step) bind(C, name="diablo_rk_substep")
      import :: c_ptr, c_int
      type(c_ptr), value :: ctx
      integer(c_int), value :: rk_step
      integer(c_int) :: diablo_rk_substep
    end function diablo_rk_substep
    function diablo_step(ctx, nsteps) bind(C, name="diablo_step")
      import :: c_ptr, c_int
      type(c_ptr), value :: ctx
      integer(c_int), value :: nsteps
      integer(c_int) :: diablo_step
    end function diablo_step
    function diablo_pre_first_step(ctx, compute_pressure) bind(C, name="diablo_pre_first_step")
      import :: c_ptr, c_int
      type(c_ptr), value :: ctx
      integer(c_int), value :: compute_pressure
      integer(c_int) :: diablo_pre_first_step
    end function diablo_pre_first_step
    function diablo_apply_bc_post(ctx) bind(C, name="diablo_apply_bc_post")
      import :: c_ptr, c_int
      type(c_ptr), value :: ctx
      integer(c_int) :: diablo_apply_bc_post
    end function diablo_apply_bc_post
    function diablo_filter_chan(ctx, n) bind(C, name="diablo_filter_chan")
      import :: c_ptr, c_int
      type(c_ptr), value :: ctx
      integer(c_int), value :: n
      integer(c_int) :: diablo_filter_chan
    end function diablo_filter_chan

    ! ---- statistics (save_stats_chan, for/statistics.f90:44-712)
    function diablo_stats_size(ctx) bind(C, name="diablo_stats_size")
      import :: c_ptr, c_int
      type(c_ptr), value :: ctx
      integer(c_int) :: diablo_stats_size
    end function diablo_stats_size
    function diablo_stats(ctx, homogeneous_x, out, len) bind(C, name="diablo_stats")
      import :: c_ptr, c_int, c_double
      type(c_ptr), value :: ctx
      integer(c_int), value :: homogeneous_x
      real(c_double), intent(out) :: out(*)
      integer(c_int), value :: len
      integer(c_int) :: diablo_stats
    end function diablo_stats
    ! eps_sgs1 of les_chan (for/les.f90:924-1068), formed at the step after a
    ! diablo_stats call on an LES context
    function diablo_les_eps_sgs1(ctx, out, len) bind(C, name="diablo_les_eps_sgs1")
      import :: c_ptr, c_int, c_double
      type(c_ptr), value :: ctx
      real(c_double), intent(out) :: out(*)
      integer(c_int), value :: len
      integer(c_int) :: diablo_les_eps_sgs1
    end function diablo_les_eps_sgs1

    ! ---- run control
    function diablo_set_precision(ctx, precision) bind(C, name="diablo_set_precision")
      import :: c_ptr, c_int
      type(c_ptr), value :: ctx
      integer(c_int), value :: precision
      integer(c_int) :: diablo_set_precision
    end function diablo_set_precision
    function diablo_get_time(ctx, time, time_step, delta_t) bind(C, name="diablo_get_time")
      import :: c_ptr, c_int, c_double
      type(c_ptr), value :: ctx
      real(c_double), intent(out) :: time
      integer(c_int), intent(out) :: time_step
      real(c_double), intent(out) :: delta_t
      integer(c_int) :: diablo_get_time
    end function diablo_get_time
    function diablo_set_time(ctx, time, time_step, delta_t) bind(C, name="diablo_set_time")
      import :: c_ptr, c_int, c_double
      type(c_ptr), value :: ctx
      real(c_double), value :: time
      integer(c_int), value :: time_step
      real(c_double), value :: delta_t
      integer(c_int) :: diablo_set_time
    end function diablo_set_time
    function diablo_set_stream(ctx, stream) bind(C, name="diablo_set_stream")
      import :: c_ptr, c_int
      type(c_ptr), value :: ctx, stream
      integer(c_int) :: diablo_set_stream
    end function diablo_set_stream
    function diablo_synchronize(ctx) bind(C, name="diablo_synchronize")
      import :: c_ptr, c_int
      type(c_ptr), value :: ctx
      integer(c_int) :: diablo_synchronize
    end function diablo_synchronize
    function diablo_check_finite(ctx) bind(C, name="diablo_check_finite")
      import :: c_ptr, c_int
      type(c_ptr), value :: ctx
      integer(c_int) :: diablo_check_finite
    end function diablo_check_finite
    function diablo_set_wait_bound(ctx, max_spins, withheld_arrivals) bind(C, name="diablo_set_wait_bound")
      import :: c_ptr, c_int, c_long_long
      type(c_ptr), value :: ctx
      integer(c_long_long), value :: max_spins
      integer(c_int), value :: withheld_arrivals
      integer(c_int) :: diablo_set_wait_bound
    end function diablo_set_wait_bound

    ! ---- tracing and status text
    function diablo_kernel_launches(ctx) bind(C, name="diablo_kernel_launches")
      import :: c_ptr, c_long_long
      type(c_ptr), value :: ctx
      integer(c_long_long) :: diablo_kernel_launches
    end function diablo_kernel_launches
    function diablo_set_profiling(ctx, enable) bind(C, name="diablo_set_profiling")
      import :: c_ptr, c_int
      type(c_ptr), value :: ctx
      integer(c_int), value :: enable
      integer(c_int) :: diablo_set_profiling
    end function diablo_set_profiling
    function diablo_kernel_times(ctx, slot, total_ms, launches) bind(C, name="diablo_kernel_times")
      import :: c_ptr, c_int, c_double, c_long_long
      type(c_ptr), value :: ctx
      integer(c_int), value :: slot
      real(c_double), intent(out) :: total_ms
      integer(c_long_long), intent(out) :: launches
      integer(c_int) :: diablo_kernel_times
    end function diablo_kernel_times
    function diablo_kernel_slots() bind(C, name="diablo_kernel_slots")
      import :: c_int
      integer(c_int) :: diablo_kernel_slots
    end function diablo_kernel_slots
    function diablo_kernel_name(slot) bind(C, name="diablo_kernel_name")
      import :: c_ptr, c_int
      integer(c_int), value :: slot
      type(c_ptr) :: diablo_kernel_name
    end function diablo_kernel_name
    function diablo_status_string(status) bind(C, name="diablo_status_string")
      import :: c_ptr, c_int
      integer(c_int), value :: status
      type(c_ptr) :: diablo_status_string
    end function diablo_status_string
    function diablo_abi_version() bind(C, name="diablo_abi_version")
      import :: c_int
      integer(c_int) :: diablo_abi_version
    end function diablo_abi_version

    ! ---- discrete adjoint; lam(1:4+N_th) hold the addresses of the Fourier
    ! arrays dJ/d(u1, u2, u3, p, th_1, ..)
    function diablo_adjoint_record(ctx, nsteps, every) bind(C, name="diablo_adjoint_record")
      import :: c_ptr, c_int
      type(c_ptr), value :: ctx
      integer(c_int), value :: nsteps, every
      integer(c_int) :: diablo_adjoint_record
    end function diablo_adjoint_record
    function diablo_adjoint_run(ctx, lam) bind(C, name="diablo_adjoint_run")
      import :: c_ptr, c_int
      type(c_ptr), value :: ctx
      type(c_ptr), intent(in) :: lam(*)
      integer(c_int) :: diablo_adjoint_run
    end function diablo_adjoint_run

    ! ---- transform tiles
    function diablo_autotune(ctx, tiles) bind(C, name="diablo_autotune")
      import :: c_ptr, c_int
      type(c_ptr), value :: ctx
      integer(c_int), intent(out) :: tiles(4)
      integer(c_int) :: diablo_autotune
    end function diablo_autotune
    function diablo_tiles(ctx, tiles) bind(C, name="diablo_tiles")
      import :: c_ptr, c_int
      type(c_ptr), value :: ctx
      integer(c_int), intent(out) :: tiles(4)
      integer(c_int) :: diablo_tiles
    end function diablo_tiles

    ! ---- the host round trip: bufs(1:4+N_th) hold the addresses of the
    ! host Fourier arrays u1, u2, u3, p, th_1, ..
    function diablo_step_host(ctx, bufs, nsteps) bind(C, name="diablo_step_host")
      import :: c_ptr, c_int
      type(c_ptr), value :: ctx
      type(c_ptr), intent(in) :: bufs(*)
      integer(c_int), value :: nsteps
      integer(c_int) :: diablo_step_host
    end function diablo_step_host
    ! ---- ensembles of independent channels
    function diablo_ensemble_create(members, n, status) bind(C, name="diablo_ensemble_create")
      import :: c_ptr, c_int
      type(c_ptr), intent(in) :: members(*)
      integer(c_int), value :: n
      integer(c_int), intent(out) :: status
      type(c_ptr) :: diablo_ensemble_create
    end function diablo_ensemble_create
    function diablo_ensemble_step(e, nsteps) bind(C, name="diablo_ensemble_step")
      import :: c_ptr, c_int
      type(c_ptr), value :: e
      integer(c_int), value :: nsteps
      integer(c_int) :: diablo_ensemble_step
    end function diablo_ensemble_step
    function diablo_ensemble_synchronize(e) bind(C, name="diablo_ensemble_synchronize")
      import :: c_ptr, c_int
      type(c_ptr), value :: e
      integer(c_int) :: diablo_ensemble_synchronize
    end function diablo_ensemble_synchronize
    function diablo_ensemble_stream(e) bind(C, name="diablo_ensemble_stream")
      import :: c_ptr
      type(c_ptr), value :: e
      type(c_ptr) :: diablo_ensemble_stream
    end function diablo_ensemble_stream
    function diablo_ensemble_destroy(e) bind(C, name="diablo_ensemble_destroy")
      import :: c_ptr, c_int
      type(c_ptr), value :: e
      integer(c_int) :: diablo_ensemble_destroy
    end function diablo_ensemble_destroy
    function diablo_ensemble_set_mode(e, mode) bind(C, name="diablo_ensemble_set_mode")
      import :: c_ptr, c_int
      type(c_ptr), value :: e
      integer(c_int), value :: mode
      integer(c_int) :: diablo_ensemble_set_mode
    end function diablo_ensemble_set_mode
    function diablo_ensemble_mode(e) bind(C, name="diablo_ensemble_mode")
      import :: c_ptr, c_int
      type(c_ptr), value :: e
      integer(c_int) :: diablo_ensemble_mode
    end function diablo_ensemble_mode
    function diablo_ensemble_autotune(e, steps_per_trial) bind(C, name="diablo_ensemble_autotune")
      import :: c_ptr, c_int
      type(c_ptr), value :: e
      integer(c_int), value :: steps_per_trial
      integer(c_int) :: diablo_ensemble_autotune
    end function diablo_ensemble_autotune
  end interface

contains

  ! Stop with the library's status text when a call failed, as the
  ! reference's own error paths stop (for/advance.f90:113-117).
  subroutine diablo_check(status, what)
    integer(c_int), intent(in) :: status
    character(len=*), intent(in) :: what
    if (status /= DIABLO_OK) then
      write (*, '(a, a, i0)') trim(what), ' failed: status ', status
      stop 'libdiablo_gpu error'
    end if
  end subroutine diablo_check

end module diablo_gpu
