! ISO_C_BINDING interface to libmhit_b200.so (include/mhit_b200.h) for a Fortran host.
!
! Replaces the body of the timestep loop of multi/main.f90:456-1042 (aroccon/MHIT36_mixedp) on one
! GPU.  Arrays are the reference's interior fields: real(8) u(nx,ny,nz) without halo planes,
! i.e. u(1:nx, 1+halo_ext:ny+halo_ext, 1+halo_ext:nz+halo_ext) of the reference copied to a
! contiguous array (the layout of its field files, multi/readwrite.f90:28-46).
!
! No Fortran compiler is present on the build image; this module is compiled by the host
! application's own build (nvfortran or gfortran):  gfortran -c mhit_gpu.f90
module mhit_gpu
  use iso_c_binding
  implicit none

  integer(c_int), parameter :: MHIT_OK = 0, MHIT_ERR_ARG = -1, MHIT_ERR_CUDA = -2, MHIT_ERR_NAN = -3
  integer(c_int), parameter :: MHIT_ERR_CFL = -4, MHIT_ERR_IO = -5, MHIT_ERR_STATE = -6, MHIT_ERR_TIMEOUT = -7
  integer(c_int), parameter :: MHIT_POISSON_FP64 = 0, MHIT_POISSON_FP32 = 1, MHIT_POISSON_FP32_REFINED = 2, &
                                MHIT_POISSON_FP32_INCREMENTAL = 3
  integer(c_int), parameter :: MHIT_LAP_EXACT = 0, MHIT_LAP_MODIFIED = 1
  integer(c_int), parameter :: MHIT_INTERP_LINEAR1D = 0, MHIT_INTERP_TRILINEAR = 1

  type, bind(C) :: mhit_params
    integer(c_int) :: nx, ny, nz
    real(c_double) :: dt, mu, rho
    real(c_double) :: f1, f2, f3, k0
    real(c_double) :: radius, sigma, epsr
    integer(c_int) :: phiflag, partflag, npart
    integer(c_int) :: poisson, laplacian, interp, yz_shift, use_graph, device
    integer(c_int) :: acdi_clamp
    integer(c_int) :: zsolve_tc
  end type mhit_params

  type, bind(C) :: mhit_run
    integer(c_int) :: restart, tstart, tfin, dump, inflow, inphi, inpart
  end type mhit_run

  ! one drop of mhit_label_drops (post/unionfind_periodic/main.f90:425-436)
  type, bind(C) :: mhit_drop
    integer(c_long_long) :: cells
    real(c_double) :: volume
    real(c_double) :: x, y, z
    real(c_double) :: u, v, w
  end type mhit_drop

  type, bind(C) :: mhit_diag
    integer(c_long_long) :: nstep
    real(c_double) :: gumax, cfl
    real(c_double) :: mean(3)
    real(c_double) :: maxdiv, ke, dissipation
    integer(c_int) :: flags
  end type mhit_diag

  interface
    integer(c_int) function mhit_abi_version() bind(C, name="mhit_abi_version")
      import :: c_int
    end function

    type(c_ptr) function mhit_last_error() bind(C, name="mhit_last_error")
      import :: c_ptr
    end function

    integer(c_int) function mhit_params_default(p) bind(C, name="mhit_params_default")
      import :: c_int, mhit_params
      type(mhit_params), intent(out) :: p
    end function

    ! readinput (multi/readinput.f90:4-81)
    integer(c_int) function mhit_read_input(path, p, run) bind(C, name="mhit_read_input")
      import :: c_int, c_char, mhit_params, mhit_run
      character(kind=c_char), dimension(*), intent(in) :: path
      type(mhit_params), intent(inout) :: p
      type(mhit_run), intent(out) :: run
    end function

    integer(c_int) function mhit_init(p, ctx) bind(C, name="mhit_init")
      import :: c_int, c_ptr, mhit_params
      type(mhit_params), intent(in) :: p
      type(c_ptr), intent(out) :: ctx
    end function

    subroutine mhit_destroy(ctx) bind(C, name="mhit_destroy")
      import :: c_ptr
      type(c_ptr), value :: ctx
    end subroutine

    ! initial fields (multi/main.f90:322-415); phi may be c_null_ptr when phiflag = 0
    integer(c_int) function mhit_upload_fields(ctx, u, v, w, phi) bind(C, name="mhit_upload_fields")
      import :: c_int, c_ptr, c_double
      type(c_ptr), value :: ctx
      real(c_double), dimension(*), intent(in) :: u, v, w
      type(c_ptr), value :: phi
    end function

    ! initial conditions built on the device (multi/main.f90:322-415 and the seeded fields)
    integer(c_int) function mhit_init_taylor_green(ctx) bind(C, name="mhit_init_taylor_green")
      import :: c_int, c_ptr
      type(c_ptr), value :: ctx
    end function

    ! modes: 3*(2*kmax+1)**3 complex amplitudes, [component][kz][ky][kx] with k from -kmax
    integer(c_int) function mhit_init_velocity_modes(ctx, kmax, modes, rms) bind(C, name="mhit_init_velocity_modes")
      import :: c_int, c_ptr, c_double
      type(c_ptr), value :: ctx
      integer(c_int), value :: kmax
      real(c_double), dimension(*), intent(in) :: modes
      real(c_double), value :: rms
    end function

    ! centres(3,ndrops): x, y, z of each drop
    integer(c_int) function mhit_init_drops(ctx, ndrops, centres, radius) bind(C, name="mhit_init_drops")
      import :: c_int, c_ptr, c_double
      type(c_ptr), value :: ctx
      integer(c_int), value :: ndrops
      real(c_double), dimension(*), intent(in) :: centres
      real(c_double), value :: radius
    end function

    ! tracer table built on the device: tags, seeded uniform positions, zero velocities
    integer(c_int) function mhit_init_particles(ctx, npart, seed) bind(C, name="mhit_init_particles")
      import :: c_int, c_ptr, c_long_long
      type(c_ptr), value :: ctx
      integer(c_int), value :: npart
      integer(c_long_long), value :: seed
    end function

    ! E(0:nbins-1): shell-summed kinetic-energy spectrum of the current velocity
    integer(c_int) function mhit_energy_spectrum(ctx, E, nbins) bind(C, name="mhit_energy_spectrum")
      import :: c_int, c_ptr, c_double
      type(c_ptr), value :: ctx
      real(c_double), dimension(*), intent(out) :: E
      integer(c_int), value :: nbins
    end function

    ! part(npart,12): tag, x, y, z, u, v, w, phi, u1, v1, w1, phi1 (multi/particles.f90:15-22)
    integer(c_int) function mhit_upload_particles(ctx, part, npart) bind(C, name="mhit_upload_particles")
      import :: c_int, c_ptr, c_double
      type(c_ptr), value :: ctx
      real(c_double), dimension(*), intent(in) :: part
      integer(c_int), value :: npart
    end function

    integer(c_int) function mhit_download_particles(ctx, part, npart) bind(C, name="mhit_download_particles")
      import :: c_int, c_ptr, c_double
      type(c_ptr), value :: ctx
      real(c_double), dimension(*), intent(out) :: part
      integer(c_int), value :: npart
    end function

    ! nsteps passes of the loop body multi/main.f90:456-1007
    integer(c_int) function mhit_step(ctx, nsteps) bind(C, name="mhit_step")
      import :: c_int, c_ptr
      type(c_ptr), value :: ctx
      integer(c_int), value :: nsteps
    end function

    ! any argument may be c_null_ptr
    integer(c_int) function mhit_download_fields(ctx, u, v, w, p, phi) bind(C, name="mhit_download_fields")
      import :: c_int, c_ptr
      type(c_ptr), value :: ctx, u, v, w, p, phi
    end function

    integer(c_int) function mhit_diagnostics(ctx, d) bind(C, name="mhit_diagnostics")
      import :: c_int, c_ptr, mhit_diag
      type(c_ptr), value :: ctx
      type(mhit_diag), intent(out) :: d
    end function

    ! writefield / readfield (multi/readwrite.f90)
    integer(c_int) function mhit_write_field(ctx, dir, t, fieldn) bind(C, name="mhit_write_field")
      import :: c_int, c_ptr, c_char
      type(c_ptr), value :: ctx
      character(kind=c_char), dimension(*), intent(in) :: dir
      integer(c_int), value :: t, fieldn
    end function

    integer(c_int) function mhit_read_field(ctx, path, fieldn) bind(C, name="mhit_read_field")
      import :: c_int, c_ptr, c_char
      type(c_ptr), value :: ctx
      character(kind=c_char), dimension(*), intent(in) :: path
      integer(c_int), value :: fieldn
    end function

    ! exact-resume checkpoint: fields, rhs_o history, device scalars, step count, tracers
    integer(c_int) function mhit_write_checkpoint(ctx, path) bind(C, name="mhit_write_checkpoint")
      import :: c_int, c_ptr, c_char
      type(c_ptr), value :: ctx
      character(kind=c_char), dimension(*), intent(in) :: path
    end function

    integer(c_int) function mhit_read_checkpoint(ctx, path) bind(C, name="mhit_read_checkpoint")
      import :: c_int, c_ptr, c_char
      type(c_ptr), value :: ctx
      character(kind=c_char), dimension(*), intent(in) :: path
    end function

    ! connected components of phi >= thresh (connectivity 6 or 26), statistics per drop;
    ! labels may be c_null_ptr or c_loc of an integer(c_int) array (nx, ny, nz)
    integer(c_int) function mhit_label_drops(ctx, thresh, connectivity, drops, maxdrops, ndrops, labels) &
        bind(C, name="mhit_label_drops")
      import :: c_int, c_ptr, c_double, mhit_drop
      type(c_ptr), value :: ctx
      real(c_double), value :: thresh
      integer(c_int), value :: connectivity, maxdrops
      type(mhit_drop), intent(out) :: drops(*)
      integer(c_int), intent(out) :: ndrops
      type(c_ptr), value :: labels
    end function

    integer(c_int) function mhit_time_steps(ctx, nsteps, ms) bind(C, name="mhit_time_steps")
      import :: c_int, c_ptr, c_double
      type(c_ptr), value :: ctx
      integer(c_int), value :: nsteps
      real(c_double), intent(out) :: ms
    end function

    ! ensemble of nbox independent boxes (params(1:nbox), any sizes) stepped together
    integer(c_int) function mhit_ensemble_create(params, nbox, ens) bind(C, name="mhit_ensemble_create")
      import :: c_int, c_ptr, mhit_params
      type(mhit_params), intent(in) :: params(*)
      integer(c_int), value :: nbox
      type(c_ptr), intent(out) :: ens
    end function

    subroutine mhit_ensemble_destroy(ens) bind(C, name="mhit_ensemble_destroy")
      import :: c_ptr
      type(c_ptr), value :: ens
    end subroutine

    ! context of box b (0-based): upload, download, diagnostics and field files per box
    integer(c_int) function mhit_ensemble_box(ens, b, ctx) bind(C, name="mhit_ensemble_box")
      import :: c_int, c_ptr
      type(c_ptr), value :: ens
      integer(c_int), value :: b
      type(c_ptr), intent(out) :: ctx
    end function

    integer(c_int) function mhit_ensemble_step(ens, nsteps) bind(C, name="mhit_ensemble_step")
      import :: c_int, c_ptr
      type(c_ptr), value :: ens
      integer(c_int), value :: nsteps
    end function

    integer(c_int) function mhit_ensemble_autotune(ens, trials, nlanes) bind(C, name="mhit_ensemble_autotune")
      import :: c_int, c_ptr
      type(c_ptr), value :: ens
      integer(c_int), value :: trials
      integer(c_int), intent(out) :: nlanes
    end function
  end interface

contains

  ! Fortran string of the last library error of this thread.
  function mhit_error_string() result(s)
    character(len=:), allocatable :: s
    type(c_ptr) :: p
    character(kind=c_char), pointer :: chars(:)
    integer :: n
    interface
      integer(c_size_t) function c_strlen(str) bind(C, name="strlen")
        import :: c_ptr, c_size_t
        type(c_ptr), value :: str
      end function
    end interface
    p = mhit_last_error()
    n = int(c_strlen(p))
    call c_f_pointer(p, chars, [n])
    allocate(character(len=n) :: s)
    s = transfer(chars(1:n), s)
  end function mhit_error_string

end module mhit_gpu
