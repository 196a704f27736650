! psdns_gpu_mod.f90 -- Fortran 2003 interface to libpsdns_gpu (include/psdns_gpu.h).
!
! A PSDNS driver USEs this module and calls the C-ABI through iso_c_binding;
! no Fortran compiler exists in the build container, so this file is shipped
! for the driver build (link with -lpsdns_gpu).
module psdns_gpu_mod
  use iso_c_binding
  implicit none

  integer(c_int32_t), parameter :: PSDNS_PREC_FP32 = 0, PSDNS_PREC_FP64 = 1
  integer(c_int32_t), parameter :: PSDNS_DFT_FP32 = 0, PSDNS_DFT_TC_BF16X3 = 1
  integer(c_int32_t), parameter :: PSDNS_LAYOUT_YCYL = 0
  integer(c_int32_t), parameter :: PSDNS_LAYOUT_FULL = 1
  integer(c_int32_t), parameter :: PSDNS_FIELD_U = 0, PSDNS_FIELD_UN = 1

  type, bind(c) :: psdns_params
    integer(c_int32_t) :: nx, ny, nz, nc, precision, kshift, ksran, seed_input
    integer(c_int32_t) :: kranf1, kranf2
    integer(c_int32_t) :: dft, rkmethod
    integer(c_int32_t) :: reserved_i(4)
    real(c_double) :: viscos, beta1, beta2, beta3, cfl, dt
    real(c_double) :: kforce, tforce, epsfor, tfiuo, pr
    real(c_double) :: grad(3)
    real(c_double) :: reserved_d(8)
  end type psdns_params

  interface
    integer(c_int) function psdns_gpu_default_params(p) bind(c, name='psdns_gpu_default_params')
      import :: c_int, psdns_params
      type(psdns_params), intent(inout) :: p
    end function
    integer(c_int) function psdns_gpu_init(p, ctx) bind(c, name='psdns_gpu_init')
      import :: c_int, c_ptr, psdns_params
      type(psdns_params), intent(in) :: p
      type(c_ptr), intent(out) :: ctx
    end function
    integer(c_int) function psdns_gpu_finalize(ctx) bind(c, name='psdns_gpu_finalize')
      import :: c_int, c_ptr
      type(c_ptr), value :: ctx
    end function
    integer(c_int) function psdns_gpu_set_state(ctx, un, layout) bind(c, name='psdns_gpu_set_state')
      import :: c_int, c_ptr, c_double_complex, c_int32_t
      type(c_ptr), value :: ctx
      complex(c_double_complex), intent(in) :: un(*)
      integer(c_int32_t), value :: layout
    end function
    integer(c_int) function psdns_gpu_get_state(ctx, out, which, layout) bind(c, name='psdns_gpu_get_state')
      import :: c_int, c_ptr, c_double_complex, c_int32_t
      type(c_ptr), value :: ctx
      complex(c_double_complex), intent(out) :: out(*)
      integer(c_int32_t), value :: which, layout
    end function
    integer(c_int) function psdns_gpu_step(ctx, info) bind(c, name='psdns_gpu_step')
      import :: c_int, c_ptr, c_double
      type(c_ptr), value :: ctx
      real(c_double), intent(out) :: info(8)
    end function
    integer(c_int) function psdns_gpu_rk_stage(ctx, kstep, gsh, dt, forcing, velmax) bind(c, name='psdns_gpu_rk_stage')
      import :: c_int, c_ptr, c_double, c_int32_t
      type(c_ptr), value :: ctx
      integer(c_int32_t), value :: kstep
      real(c_double), intent(in) :: gsh(3, 2)
      real(c_double), intent(in) :: dt
      type(c_ptr), value :: forcing       ! c_loc(for) or c_null_ptr
      real(c_double), intent(out) :: velmax
    end function
    integer(c_int) function psdns_gpu_spectra(ctx, which, ek, dk, eijk, stats) bind(c, name='psdns_gpu_spectra')
      import :: c_int, c_ptr, c_double, c_int32_t
      type(c_ptr), value :: ctx
      integer(c_int32_t), value :: which
      real(c_double), intent(out) :: ek(*), dk(*), eijk(*), stats(7)
    end function
    integer(c_int) function psdns_gpu_particles_set(ctx, np, pos) bind(c, name='psdns_gpu_particles_set')
      import :: c_int, c_ptr, c_double, c_int64_t
      type(c_ptr), value :: ctx
      integer(c_int64_t), value :: np
      real(c_double), intent(in) :: pos(*)
    end function
    integer(c_int) function psdns_gpu_particles_get(ctx, pos, vel) bind(c, name='psdns_gpu_particles_get')
      import :: c_int, c_ptr, c_double
      type(c_ptr), value :: ctx
      real(c_double), intent(out) :: pos(*), vel(*)
    end function
    integer(c_int) function psdns_gpu_particles_write(ctx, prefix, ngp, istep, append) &
        bind(c, name='psdns_gpu_particles_write')
      import :: c_int, c_ptr, c_char, c_int32_t
      type(c_ptr), value :: ctx
      character(kind=c_char), intent(in) :: prefix(*)
      integer(c_int32_t), value :: ngp, istep, append
    end function
    integer(c_int) function psdns_gpu_set_state_async(ctx, un, layout) bind(c, name='psdns_gpu_set_state_async')
      import :: c_int, c_ptr, c_int32_t
      type(c_ptr), value :: ctx
      type(c_ptr), value :: un        ! c_loc of a pinned (page-locked) array
      integer(c_int32_t), value :: layout
    end function
    integer(c_int) function psdns_gpu_get_state_async(ctx, out, which, layout) &
        bind(c, name='psdns_gpu_get_state_async')
      import :: c_int, c_ptr, c_int32_t
      type(c_ptr), value :: ctx
      type(c_ptr), value :: out
      integer(c_int32_t), value :: which, layout
    end function
    ! pinned host arrays (c_loc of a cudaHostRegister'ed or cudaHostAlloc'ed uy)
    integer(c_int) function psdns_gpu_set_state_sphere_async(ctx, un) &
        bind(c, name='psdns_gpu_set_state_sphere_async')
      import :: c_int, c_ptr
      type(c_ptr), value :: ctx
      type(c_ptr), value :: un
    end function
    integer(c_int) function psdns_gpu_get_state_sphere_async(ctx, out, which) &
        bind(c, name='psdns_gpu_get_state_sphere_async')
      import :: c_int, c_ptr, c_int32_t
      type(c_ptr), value :: ctx
      type(c_ptr), value :: out
      integer(c_int32_t), value :: which
    end function
    integer(c_int) function psdns_gpu_particles_advance(ctx, gsh1, dt_prev) &
        bind(c, name='psdns_gpu_particles_advance')
      import :: c_int, c_ptr, c_double
      type(c_ptr), value :: ctx
      real(c_double), intent(in) :: gsh1(3)
      real(c_double), value :: dt_prev
    end function
    integer(c_int) function psdns_gpu_host_register(ptr, bytes) bind(c, name='psdns_gpu_host_register')
      import :: c_int, c_ptr, c_size_t
      type(c_ptr), value :: ptr
      integer(c_size_t), value :: bytes
    end function
    integer(c_int) function psdns_gpu_host_unregister(ptr) bind(c, name='psdns_gpu_host_unregister')
      import :: c_int, c_ptr
      type(c_ptr), value :: ptr
    end function
    integer(c_int) function psdns_gpu_sync(ctx) bind(c, name='psdns_gpu_sync')
      import :: c_int, c_ptr
      type(c_ptr), value :: ctx
    end function
    integer(c_int) function psdns_gpu_field_sinusoidal(ctx, au, av) bind(c, name='psdns_gpu_field_sinusoidal')
      import :: c_int, c_ptr, c_double
      type(c_ptr), value :: ctx
      real(c_double), value :: au, av
    end function
    integer(c_int) function psdns_gpu_particles_init(ctx, nop, pstart, kipran) bind(c, name='psdns_gpu_particles_init')
      import :: c_int, c_ptr, c_int32_t, c_int64_t
      type(c_ptr), value :: ctx
      integer(c_int64_t), value :: nop
      integer(c_int32_t), value :: pstart, kipran
    end function
    integer(c_int) function psdns_gpu_write_checkpoint(ctx, path, which) bind(c, name='psdns_gpu_write_checkpoint')
      import :: c_int, c_ptr, c_int32_t, c_char
      type(c_ptr), value :: ctx
      character(kind=c_char), intent(in) :: path(*)   ! terminated by c_null_char
      integer(c_int32_t), value :: which
    end function
    integer(c_int) function psdns_gpu_write_checkpoint_set(ctx, prefix, iproc, jproc, which) &
        bind(c, name='psdns_gpu_write_checkpoint_set')
      import :: c_int, c_ptr, c_char, c_int32_t
      type(c_ptr), value :: ctx
      character(kind=c_char), intent(in) :: prefix(*)
      integer(c_int32_t), value :: iproc, jproc, which
    end function
    integer(c_int) function psdns_gpu_read_checkpoint_set(ctx, paths, nfiles) &
        bind(c, name='psdns_gpu_read_checkpoint_set')
      import :: c_int, c_ptr, c_int32_t
      type(c_ptr), value :: ctx
      type(c_ptr), value :: paths        ! c_loc of an array of c_loc(path(1)) pointers
      integer(c_int32_t), value :: nfiles
    end function
    integer(c_int) function psdns_gpu_write_chkptou(ctx, path, istep, iostep) bind(c, name='psdns_gpu_write_chkptou')
      import :: c_int, c_ptr, c_char, c_int32_t
      type(c_ptr), value :: ctx
      character(kind=c_char), intent(in) :: path(*)
      integer(c_int32_t), value :: istep, iostep
    end function
    integer(c_int) function psdns_gpu_read_chkptou(ctx, path, strict, istep) bind(c, name='psdns_gpu_read_chkptou')
      import :: c_int, c_ptr, c_char, c_int32_t
      type(c_ptr), value :: ctx
      character(kind=c_char), intent(in) :: path(*)
      integer(c_int32_t), value :: strict
      integer(c_int32_t), intent(out) :: istep
    end function
    integer(c_int) function psdns_gpu_write_ranout(ctx, path) bind(c, name='psdns_gpu_write_ranout')
      import :: c_int, c_ptr, c_char
      type(c_ptr), value :: ctx
      character(kind=c_char), intent(in) :: path(*)
    end function
    integer(c_int) function psdns_gpu_read_ranin(ctx, path) bind(c, name='psdns_gpu_read_ranin')
      import :: c_int, c_ptr, c_char
      type(c_ptr), value :: ctx
      character(kind=c_char), intent(in) :: path(*)
    end function
    integer(c_int) function psdns_gpu_read_checkpoint(ctx, path) bind(c, name='psdns_gpu_read_checkpoint')
      import :: c_int, c_ptr, c_char
      type(c_ptr), value :: ctx
      character(kind=c_char), intent(in) :: path(*)
    end function
    integer(c_int) function psdns_gpu_transfer_spectrum(ctx, gsh, tk) bind(c, name='psdns_gpu_transfer_spectrum')
      import :: c_int, c_ptr, c_double
      type(c_ptr), value :: ctx
      real(c_double), intent(in) :: gsh(3)
      real(c_double), intent(out) :: tk(*)
    end function
    integer(c_int) function psdns_gpu_spectra_scales(ctx, which, xr, yr, zr, stats) &
        bind(c, name='psdns_gpu_spectra_scales')
      import :: c_int, c_ptr, c_int32_t, c_double
      type(c_ptr), value :: ctx
      integer(c_int32_t), value :: which
      real(c_double), intent(out) :: xr(*), yr(*), zr(*), stats(55)
    end function
    integer(c_int) function psdns_gpu_gradient_moments(ctx, which, gsh, out) &
        bind(c, name='psdns_gpu_gradient_moments')
      import :: c_int, c_ptr, c_int32_t, c_double
      type(c_ptr), value :: ctx
      integer(c_int32_t), value :: which
      real(c_double), intent(in) :: gsh(3)
      real(c_double), intent(out) :: out(16)
    end function
    ! ensembles of independent boxes (params(count): one psdns_params per box)
    integer(c_int) function psdns_gpu_ensemble_create(params, count, ens) bind(c, name='psdns_gpu_ensemble_create')
      import :: c_int, c_ptr, c_int32_t, psdns_params
      type(psdns_params), intent(in) :: params(*)
      integer(c_int32_t), value :: count
      type(c_ptr), intent(out) :: ens
    end function
    integer(c_int) function psdns_gpu_ensemble_destroy(ens) bind(c, name='psdns_gpu_ensemble_destroy')
      import :: c_int, c_ptr
      type(c_ptr), value :: ens
    end function
    integer(c_int) function psdns_gpu_ensemble_field_init(ens, seeds) bind(c, name='psdns_gpu_ensemble_field_init')
      import :: c_int, c_ptr, c_int32_t
      type(c_ptr), value :: ens
      integer(c_int32_t), intent(in) :: seeds(*)
    end function
    integer(c_int) function psdns_gpu_ensemble_set_state(ens, box, un, layout) &
        bind(c, name='psdns_gpu_ensemble_set_state')
      import :: c_int, c_ptr, c_int32_t, c_double
      type(c_ptr), value :: ens
      integer(c_int32_t), value :: box, layout
      real(c_double), intent(in) :: un(*)
    end function
    integer(c_int) function psdns_gpu_ensemble_get_state(ens, box, out, which, layout) &
        bind(c, name='psdns_gpu_ensemble_get_state')
      import :: c_int, c_ptr, c_int32_t, c_double
      type(c_ptr), value :: ens
      integer(c_int32_t), value :: box, which, layout
      real(c_double), intent(out) :: out(*)
    end function
    integer(c_int) function psdns_gpu_ensemble_step(ens, nsteps, info) bind(c, name='psdns_gpu_ensemble_step')
      import :: c_int, c_ptr, c_int32_t, c_double
      type(c_ptr), value :: ens
      integer(c_int32_t), value :: nsteps
      real(c_double), intent(out) :: info(*)
    end function
    integer(c_int) function psdns_gpu_ensemble_tuning(ens, cap, out, nclasses) bind(c, name='psdns_gpu_ensemble_tuning')
      import :: c_int, c_ptr, c_int32_t, c_double
      type(c_ptr), value :: ens
      integer(c_int32_t), value :: cap
      real(c_double), intent(out) :: out(*)
      integer(c_int32_t), intent(out) :: nclasses
    end function
    integer(c_int) function psdns_gpu_ensemble_spectra(ens, box, which, ek, dk, eijk, stats) &
        bind(c, name='psdns_gpu_ensemble_spectra')
      import :: c_int, c_ptr, c_int32_t, c_double
      type(c_ptr), value :: ens
      integer(c_int32_t), value :: box, which
      real(c_double), intent(out) :: ek(*), dk(*), eijk(*), stats(7)
    end function
    integer(c_int) function psdns_gpu_last_error(buf, len) bind(c, name='psdns_gpu_last_error')
      import :: c_int, c_char, c_int32_t
      character(kind=c_char), intent(out) :: buf(*)
      integer(c_int32_t), value :: len
    end function
    integer(c_int) function psdns_gpu_geometry(n, kxn, xz_tot, cut_z, colstart) bind(c, name='psdns_gpu_geometry')
      import :: c_int, c_int32_t
      integer(c_int32_t), value :: n
      integer(c_int32_t) :: kxn, xz_tot
      integer(c_int32_t) :: cut_z(*), colstart(*)
    end function
    integer(c_int) function psdns_gpu_kymax(n, kymax) bind(c, name='psdns_gpu_kymax')
      import :: c_int, c_int32_t
      integer(c_int32_t), value :: n
      integer(c_int32_t) :: kymax(*)
    end function
    integer(c_int) function psdns_gpu_field_init(ctx, seed) bind(c, name='psdns_gpu_field_init')
      import :: c_int, c_ptr, c_int32_t
      type(c_ptr), value :: ctx
      integer(c_int32_t), value :: seed
    end function
    integer(c_int) function psdns_gpu_forcing_stats(ctx, efk, eirate, erate) bind(c, name='psdns_gpu_forcing_stats')
      import :: c_int, c_ptr, c_double
      type(c_ptr), value :: ctx
      real(c_double) :: efk(*), eirate(3), erate
    end function
    integer(c_int) function psdns_gpu_forcing_table(ctx, table, kfor, k2fo) bind(c, name='psdns_gpu_forcing_table')
      import :: c_int, c_ptr, c_double, c_int32_t
      type(c_ptr), value :: ctx
      real(c_double) :: table(*)
      integer(c_int32_t) :: kfor, k2fo
    end function
    integer(c_int) function psdns_gpu_get_time(ctx, out4) bind(c, name='psdns_gpu_get_time')
      import :: c_int, c_ptr, c_double
      type(c_ptr), value :: ctx
      real(c_double) :: out4(4)
    end function
    integer(c_int) function psdns_gpu_get_stream(ctx, stream) bind(c, name='psdns_gpu_get_stream')
      import :: c_int, c_ptr
      type(c_ptr), value :: ctx
      type(c_ptr) :: stream
    end function
    integer(c_int) function psdns_gpu_profile(ctx, enable) bind(c, name='psdns_gpu_profile')
      import :: c_int, c_ptr, c_int32_t
      type(c_ptr), value :: ctx
      integer(c_int32_t), value :: enable
    end function
    integer(c_int) function psdns_gpu_kernel_times(ctx, ms, launches) bind(c, name='psdns_gpu_kernel_times')
      import :: c_int, c_ptr, c_double, c_int64_t
      type(c_ptr), value :: ctx
      real(c_double) :: ms(6)
      integer(c_int64_t) :: launches(6)
    end function
    ! device arrays u_dev, un_dev and the stream are device/CUDA handles
    ! learned coarse solver: filter, shell damping, features and the correction network
    integer(c_int) function psdns_gpu_filter_state(fine, coarse) bind(c, name='psdns_gpu_filter_state')
      import :: c_int, c_ptr
      type(c_ptr), value :: fine, coarse
    end function
    integer(c_int) function psdns_gpu_shell_factor(ctx, nshell, f) bind(c, name='psdns_gpu_shell_factor')
      import :: c_int, c_ptr, c_int32_t, c_double
      type(c_ptr), value :: ctx
      integer(c_int32_t), value :: nshell
      real(c_double), intent(in) :: f(0:*)
    end function
    integer(c_int) function psdns_gpu_corrector_features(ctx, which, nshell, x) &
        bind(c, name='psdns_gpu_corrector_features')
      import :: c_int, c_ptr, c_int32_t, c_float
      type(c_ptr), value :: ctx
      integer(c_int32_t), value :: which, nshell
      real(c_float), intent(out) :: x(*)
    end function
    integer(c_int) function psdns_gpu_corrector_apply(corr, ctx, info) bind(c, name='psdns_gpu_corrector_apply')
      import :: c_int, c_ptr, c_double
      type(c_ptr), value :: corr, ctx
      real(c_double), intent(out) :: info(2)
    end function
    integer(c_int) function psdns_gpu_corrector_create(seed, corr) bind(c, name='psdns_gpu_corrector_create')
      import :: c_int, c_ptr, c_int32_t
      integer(c_int32_t), value :: seed
      type(c_ptr), intent(out) :: corr
    end function
    integer(c_int) function psdns_gpu_corrector_destroy(corr) bind(c, name='psdns_gpu_corrector_destroy')
      import :: c_int, c_ptr
      type(c_ptr), value :: corr
    end function
    integer(c_int) function psdns_gpu_corrector_params(corr, get, w) bind(c, name='psdns_gpu_corrector_params')
      import :: c_int, c_ptr, c_int32_t, c_float
      type(c_ptr), value :: corr
      integer(c_int32_t), value :: get
      real(c_float), intent(inout) :: w(*)
    end function
    integer(c_int) function psdns_gpu_corrector_forward(corr, nb, x, g) bind(c, name='psdns_gpu_corrector_forward')
      import :: c_int, c_ptr, c_int64_t, c_float
      type(c_ptr), value :: corr
      integer(c_int64_t), value :: nb
      real(c_float), intent(in) :: x(*)
      real(c_float), intent(out) :: g(*)
    end function
    integer(c_int) function psdns_gpu_corrector_grad(corr, nb, x, a, tau, wt, grad, loss) &
        bind(c, name='psdns_gpu_corrector_grad')
      import :: c_int, c_ptr, c_int64_t, c_float, c_double
      type(c_ptr), value :: corr
      integer(c_int64_t), value :: nb
      real(c_float), intent(in) :: x(*), a(*), tau(*), wt(*)
      real(c_float), intent(out) :: grad(*)
      real(c_double), intent(out) :: loss
    end function
    integer(c_int) function psdns_gpu_corrector_train(corr, nb, x, a, tau, wt, iters, lr, loss_hist) &
        bind(c, name='psdns_gpu_corrector_train')
      import :: c_int, c_ptr, c_int64_t, c_int32_t, c_float, c_double
      type(c_ptr), value :: corr
      integer(c_int64_t), value :: nb
      real(c_float), intent(in) :: x(*), a(*), tau(*), wt(*)
      integer(c_int32_t), value :: iters
      real(c_double), value :: lr
      real(c_double), intent(out) :: loss_hist(*)
    end function
    ! batched 1024-point DFT of lines (mode 0: FP32, 1: split-BF16 tensor cores)
    integer(c_int) function psdns_gpu_dft_lines(n, nlines, mode, in, out) bind(c, name='psdns_gpu_dft_lines')
      import :: c_int, c_int32_t, c_int64_t, c_double_complex
      integer(c_int32_t), value :: n
      integer(c_int64_t), value :: nlines
      integer(c_int32_t), value :: mode
      complex(c_double_complex), intent(in) :: in(*)
      complex(c_double_complex), intent(out) :: out(*)
    end function
    integer(c_int) function psdns_gpu_tc_gemm_check(a_mn_major, a, b, d) bind(c, name='psdns_gpu_tc_gemm_check')
      import :: c_int, c_int32_t, c_ptr
      integer(c_int32_t), value :: a_mn_major
      type(c_ptr), value :: a, b, d
    end function
    integer(c_int) function psdns_gpu_rk_stage_noalloc(p, kstep, gsh, dt, u_dev, un_dev, velmax_out, stream) &
        bind(c, name='psdns_gpu_rk_stage_noalloc')
      import :: c_int, c_ptr, c_double, c_int32_t, psdns_params
      type(psdns_params), intent(in) :: p
      integer(c_int32_t), value :: kstep
      real(c_double), intent(in) :: gsh(6), dt(*)
      type(c_ptr), value :: u_dev, un_dev, stream
      real(c_double) :: velmax_out
    end function
  end interface
end module psdns_gpu_mod
