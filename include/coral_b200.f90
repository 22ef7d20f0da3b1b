! coral_b200.f90 -- ISO_C_BINDING interfaces of every entry point declared in
! coral_b200.h, for a Fortran driver (Coral's plane_layer_main.f90 binds its C
! text readers the same way, src/text_parsing/cwraps.f90:1-23).
!
! Conventions: strings are passed NUL-terminated ('file'//c_null_char); a NULL
! char pointer is c_null_ptr through the *_ptr variants or an empty string
! (c_null_char) where the C side accepts one; handles, ensembles, networks and
! CUDA streams are type(c_ptr); device buffers (the no-allocation transform,
! the closure's data) are type(c_ptr) holding device addresses.  Every integer
! function returns 0 or a negative CORAL_E* code (coral_b200.h); the text of the
! last error comes back as a C string from coral_last_error.
module coral_b200_c
  use, intrinsic :: iso_c_binding
  implicit none

  integer(c_int), parameter :: CORAL_OK = 0, CORAL_EBADARG = -1, CORAL_ENOMEM = -2, CORAL_ECUDA = -3, &
                               CORAL_ESINGULAR = -4, CORAL_ENONFINITE = -5, CORAL_EPARSE = -6, CORAL_EIO = -7, &
                               CORAL_EUNSUPPORTED = -8, CORAL_ENODEV = -9

  ! the device solver of a plane_layer run built with the replacement include
  ! PL_IMEX_timestepping_marching_b200.f90 (created by its first march_forward)
  type(c_ptr), save :: coral_b200_handle = c_null_ptr

  interface
    ! ---- creation and queries -------------------------------------------------
    integer(c_int) function coral_create(eqs_text, pars_text, scheme, device, h) bind(C, name="coral_create")
      import :: c_int, c_char, c_ptr
      character(kind=c_char), dimension(*), intent(in) :: eqs_text, pars_text, scheme
      integer(c_int), value :: device
      type(c_ptr), intent(out) :: h
    end function
    integer(c_int) function coral_create_from_files(eqs, pars, scheme, device, h) &
        bind(C, name="coral_create_from_files")
      import :: c_int, c_char, c_ptr
      character(kind=c_char), dimension(*), intent(in) :: eqs, pars, scheme
      integer(c_int), value :: device
      type(c_ptr), intent(out) :: h
    end function
    integer(c_int) function coral_create_with_args(eqs_text, pars_text, scheme, device, args, h) &
        bind(C, name="coral_create_with_args")
      import :: c_int, c_char, c_ptr
      character(kind=c_char), dimension(*), intent(in) :: eqs_text, pars_text, scheme, args
      integer(c_int), value :: device
      type(c_ptr), intent(out) :: h
    end function
    subroutine coral_destroy(h) bind(C, name="coral_destroy")
      import :: c_ptr
      type(c_ptr), value :: h
    end subroutine
    type(c_ptr) function coral_last_error(h) bind(C, name="coral_last_error")
      import :: c_ptr
      type(c_ptr), value :: h
    end function
    integer(c_int) function coral_query(h, what, val) bind(C, name="coral_query")
      import :: c_int, c_ptr, c_long_long
      type(c_ptr), value :: h
      integer(c_int), value :: what
      integer(c_long_long), intent(out) :: val
    end function
    integer(c_int) function coral_var_positions(h, isys, ivar, positions, n, sz) bind(C, name="coral_var_positions")
      import :: c_int, c_ptr
      type(c_ptr), value :: h
      integer(c_int), value :: isys, ivar, n
      integer(c_int), dimension(*) :: positions
      integer(c_int), intent(out) :: sz
    end function
    ! ---- factorisation and time stepping ------------------------------------------
    integer(c_int) function coral_factorize(h, dt) bind(C, name="coral_factorize")
      import :: c_int, c_ptr, c_double
      type(c_ptr), value :: h
      real(c_double), value :: dt
    end function
    integer(c_int) function coral_march(h, dt, nsteps) bind(C, name="coral_march")
      import :: c_int, c_ptr, c_double
      type(c_ptr), value :: h
      real(c_double), value :: dt
      integer(c_int), value :: nsteps
    end function
    integer(c_int) function coral_synchronize(h) bind(C, name="coral_synchronize")
      import :: c_int, c_ptr
      type(c_ptr), value :: h
    end function
    integer(c_int) function coral_diagnostics(h, out3) bind(C, name="coral_diagnostics")
      import :: c_int, c_ptr, c_double
      type(c_ptr), value :: h
      real(c_double), dimension(3) :: out3
    end function
    integer(c_int) function coral_profile_step(h, dt, ms, n) bind(C, name="coral_profile_step")
      import :: c_int, c_ptr, c_double
      type(c_ptr), value :: h
      real(c_double), value :: dt
      real(c_double), dimension(*) :: ms
      integer(c_int), value :: n
    end function
    integer(c_int) function coral_stream(h, stream) bind(C, name="coral_stream")
      import :: c_int, c_ptr
      type(c_ptr), value :: h
      type(c_ptr), intent(out) :: stream
    end function
    ! ---- the time loop, timeseries, time keeping --------------------------------------
    integer(c_int) function coral_run(h, nsteps, outdir) bind(C, name="coral_run")
      import :: c_int, c_ptr, c_char
      type(c_ptr), value :: h
      integer(c_int), value :: nsteps
      character(kind=c_char), dimension(*), intent(in) :: outdir
    end function
    integer(c_int) function coral_set_timeseries(h, text) bind(C, name="coral_set_timeseries")
      import :: c_int, c_ptr, c_char
      type(c_ptr), value :: h
      character(kind=c_char), dimension(*), intent(in) :: text
    end function
    integer(c_int) function coral_set_timeseries_from_file(h, path) bind(C, name="coral_set_timeseries_from_file")
      import :: c_int, c_ptr, c_char
      type(c_ptr), value :: h
      character(kind=c_char), dimension(*), intent(in) :: path
    end function
    integer(c_int) function coral_set_usr_output(h, text) bind(C, name="coral_set_usr_output")
      import :: c_int, c_ptr, c_char
      type(c_ptr), value :: h
      character(kind=c_char), dimension(*), intent(in) :: text
    end function
    integer(c_int) function coral_set_usr_output_from_file(h, path) bind(C, name="coral_set_usr_output_from_file")
      import :: c_int, c_ptr, c_char
      type(c_ptr), value :: h
      character(kind=c_char), dimension(*), intent(in) :: path
    end function
    integer(c_int) function coral_export_usr_output(h, dir, time_integer) bind(C, name="coral_export_usr_output")
      import :: c_int, c_ptr, c_char, c_long_long
      type(c_ptr), value :: h
      character(kind=c_char), dimension(*), intent(in) :: dir
      integer(c_long_long), value :: time_integer
    end function
    integer(c_int) function coral_timeseries(h, vals, n) bind(C, name="coral_timeseries")
      import :: c_int, c_ptr, c_double
      type(c_ptr), value :: h
      real(c_double), dimension(*) :: vals
      integer(c_int), value :: n
    end function
    integer(c_int) function coral_set_time(h, time, dt, i_timestep) bind(C, name="coral_set_time")
      import :: c_int, c_ptr, c_double, c_long_long
      type(c_ptr), value :: h
      real(c_double), value :: time, dt
      integer(c_long_long), value :: i_timestep
    end function
    integer(c_int) function coral_get_time(h, out4) bind(C, name="coral_get_time")
      import :: c_int, c_ptr, c_double
      type(c_ptr), value :: h
      real(c_double), dimension(4) :: out4
    end function
    integer(c_int) function coral_set_hermitian_kx0(h, on) bind(C, name="coral_set_hermitian_kx0")
      import :: c_int, c_ptr
      type(c_ptr), value :: h
      integer(c_int), value :: on
    end function
    integer(c_int) function coral_set_z_transform(h, form) bind(C, name="coral_set_z_transform")
      import :: c_int, c_ptr
      type(c_ptr), value :: h
      integer(c_int), value :: form
    end function
    integer(c_int) function coral_set_source(h, idx, profile) bind(C, name="coral_set_source")
      import :: c_int, c_ptr, c_double
      type(c_ptr), value :: h
      integer(c_int), value :: idx
      real(c_double), dimension(*), intent(in) :: profile
    end function
    integer(c_int) function coral_set_penalisation_mask(h, mask) bind(C, name="coral_set_penalisation_mask")
      import :: c_int, c_ptr, c_double
      type(c_ptr), value :: h
      real(c_double), dimension(*), intent(in) :: mask
    end function
    integer(c_int) function coral_autotune(h, dt, repeats, report, n) bind(C, name="coral_autotune")
      import :: c_int, c_ptr, c_double, c_char
      type(c_ptr), value :: h
      real(c_double), value :: dt
      integer(c_int), value :: repeats, n
      character(kind=c_char), dimension(*) :: report
    end function
    integer(c_int) function coral_set_variant(h, knob, value) bind(C, name="coral_set_variant")
      import :: c_int, c_ptr, c_char
      type(c_ptr), value :: h
      character(kind=c_char), dimension(*) :: knob
      integer(c_int), value :: value
    end function
    ! ---- state, transforms, QuickSave and checkpoints -----------------------------------
    integer(c_int) function coral_get_field(h, isys, field) bind(C, name="coral_get_field")
      import :: c_int, c_ptr, c_double_complex
      type(c_ptr), value :: h
      integer(c_int), value :: isys
      complex(c_double_complex), dimension(*) :: field
    end function
    integer(c_int) function coral_set_field(h, isys, field) bind(C, name="coral_set_field")
      import :: c_int, c_ptr, c_double_complex
      type(c_ptr), value :: h
      integer(c_int), value :: isys
      complex(c_double_complex), dimension(*), intent(in) :: field
    end function
    integer(c_int) function coral_get_mean_field(h, isys, field) bind(C, name="coral_get_mean_field")
      import :: c_int, c_ptr, c_double
      type(c_ptr), value :: h
      integer(c_int), value :: isys
      real(c_double), dimension(*) :: field
    end function
    integer(c_int) function coral_set_mean_field(h, isys, field) bind(C, name="coral_set_mean_field")
      import :: c_int, c_ptr, c_double
      type(c_ptr), value :: h
      integer(c_int), value :: isys
      real(c_double), dimension(*), intent(in) :: field
    end function
    integer(c_int) function coral_spec_to_phys(h, spec, phys) bind(C, name="coral_spec_to_phys")
      import :: c_int, c_ptr, c_double, c_double_complex
      type(c_ptr), value :: h
      complex(c_double_complex), dimension(*), intent(in) :: spec
      real(c_double), dimension(*) :: phys
    end function
    integer(c_int) function coral_phys_to_spec(h, phys, spec) bind(C, name="coral_phys_to_spec")
      import :: c_int, c_ptr, c_double, c_double_complex
      type(c_ptr), value :: h
      real(c_double), dimension(*), intent(in) :: phys
      complex(c_double_complex), dimension(*) :: spec
    end function
    integer(c_int) function coral_get_full_phys(h, ivar, phys) bind(C, name="coral_get_full_phys")
      import :: c_int, c_ptr, c_double
      type(c_ptr), value :: h
      integer(c_int), value :: ivar
      real(c_double), dimension(*) :: phys
    end function
    integer(c_int) function coral_set_var_phys(h, isys, ivar, phys) bind(C, name="coral_set_var_phys")
      import :: c_int, c_ptr, c_double
      type(c_ptr), value :: h
      integer(c_int), value :: isys, ivar
      real(c_double), dimension(*), intent(in) :: phys
    end function
    integer(c_int) function coral_set_mean_var_profile(h, isys, ivar, prof) bind(C, name="coral_set_mean_var_profile")
      import :: c_int, c_ptr, c_double
      type(c_ptr), value :: h
      integer(c_int), value :: isys, ivar
      real(c_double), dimension(*), intent(in) :: prof
    end function
    integer(c_int) function coral_import_quicksave(h, dir, rolling) bind(C, name="coral_import_quicksave")
      import :: c_int, c_ptr, c_char
      type(c_ptr), value :: h
      character(kind=c_char), dimension(*), intent(in) :: dir
      integer(c_int), value :: rolling
    end function
    integer(c_int) function coral_export_checkpoint(h, dir, rolling) bind(C, name="coral_export_checkpoint")
      import :: c_int, c_ptr, c_char
      type(c_ptr), value :: h
      character(kind=c_char), dimension(*), intent(in) :: dir
      integer(c_int), value :: rolling
    end function
    integer(c_int) function coral_spec_to_phys_noalloc(nx, ny, nz, spec_dev, phys_dev, stream) &
        bind(C, name="coral_spec_to_phys_noalloc")
      import :: c_int, c_ptr
      integer(c_int), value :: nx, ny, nz
      type(c_ptr), value :: spec_dev, phys_dev, stream
    end function
    ! ---- ensembles -----------------------------------------------------------------------
    integer(c_int) function coral_ensemble_create(n, eqs_texts, pars_texts, scheme, device, e) &
        bind(C, name="coral_ensemble_create")
      import :: c_int, c_ptr, c_char
      integer(c_int), value :: n, device
      type(c_ptr), dimension(*), intent(in) :: eqs_texts, pars_texts   ! c_loc of NUL-terminated strings
      character(kind=c_char), dimension(*), intent(in) :: scheme
      type(c_ptr), intent(out) :: e
    end function
    subroutine coral_ensemble_destroy(e) bind(C, name="coral_ensemble_destroy")
      import :: c_ptr
      type(c_ptr), value :: e
    end subroutine
    type(c_ptr) function coral_ensemble_last_error(e) bind(C, name="coral_ensemble_last_error")
      import :: c_ptr
      type(c_ptr), value :: e
    end function
    integer(c_int) function coral_ensemble_member(e, i, h) bind(C, name="coral_ensemble_member")
      import :: c_int, c_ptr
      type(c_ptr), value :: e
      integer(c_int), value :: i
      type(c_ptr), intent(out) :: h
    end function
    integer(c_int) function coral_ensemble_march(e, dt, nsteps) bind(C, name="coral_ensemble_march")
      import :: c_int, c_ptr, c_double
      type(c_ptr), value :: e
      real(c_double), value :: dt
      integer(c_int), value :: nsteps
    end function
    integer(c_int) function coral_ensemble_synchronize(e) bind(C, name="coral_ensemble_synchronize")
      import :: c_int, c_ptr
      type(c_ptr), value :: e
    end function
    integer(c_int) function coral_ensemble_query(e, what, val) bind(C, name="coral_ensemble_query")
      import :: c_int, c_ptr, c_long_long
      type(c_ptr), value :: e
      integer(c_int), value :: what
      integer(c_long_long), intent(out) :: val
    end function
    ! ---- learned closure --------------------------------------------------------------------
    integer(c_int) function coral_closure_create(device, seed, c) bind(C, name="coral_closure_create")
      import :: c_int, c_ptr, c_long_long
      integer(c_int), value :: device
      integer(c_long_long), value :: seed
      type(c_ptr), intent(out) :: c
    end function
    subroutine coral_closure_destroy(c) bind(C, name="coral_closure_destroy")
      import :: c_ptr
      type(c_ptr), value :: c
    end subroutine
    type(c_ptr) function coral_closure_last_error(c) bind(C, name="coral_closure_last_error")
      import :: c_ptr
      type(c_ptr), value :: c
    end function
    integer(c_int) function coral_closure_param_count() bind(C, name="coral_closure_param_count")
      import :: c_int
    end function
    integer(c_int) function coral_closure_set_scales(c, in4, out9) bind(C, name="coral_closure_set_scales")
      import :: c_int, c_ptr, c_float
      type(c_ptr), value :: c
      real(c_float), dimension(4), intent(in) :: in4
      real(c_float), dimension(9), intent(in) :: out9
    end function
    integer(c_int) function coral_closure_get_params(c, params, n) bind(C, name="coral_closure_get_params")
      import :: c_int, c_ptr, c_float
      type(c_ptr), value :: c
      real(c_float), dimension(*) :: params
      integer(c_int), value :: n
    end function
    integer(c_int) function coral_closure_set_params(c, params, n) bind(C, name="coral_closure_set_params")
      import :: c_int, c_ptr, c_float
      type(c_ptr), value :: c
      real(c_float), dimension(*), intent(in) :: params
      integer(c_int), value :: n
    end function
    integer(c_int) function coral_closure_get_gradient(c, grad, n) bind(C, name="coral_closure_get_gradient")
      import :: c_int, c_ptr, c_float
      type(c_ptr), value :: c
      real(c_float), dimension(*) :: grad
      integer(c_int), value :: n
    end function
    integer(c_int) function coral_closure_zero_gradient(c) bind(C, name="coral_closure_zero_gradient")
      import :: c_int, c_ptr
      type(c_ptr), value :: c
    end function
    integer(c_int) function coral_closure_train(c, inputs, targets, nsnap, nxaa, nyaa, nzaa, points, npts, lr, &
                                                apply, loss) bind(C, name="coral_closure_train")
      import :: c_int, c_ptr, c_long_long, c_float, c_double
      type(c_ptr), value :: c, inputs, targets, points   ! device addresses
      integer(c_int), value :: nsnap, nxaa, nyaa, nzaa, apply
      integer(c_long_long), value :: npts
      real(c_float), value :: lr
      real(c_double), intent(out) :: loss
    end function
    integer(c_int) function coral_closure_infer(c, fields, nxaa, nyaa, nzaa, tau, stream) &
        bind(C, name="coral_closure_infer")
      import :: c_int, c_ptr
      type(c_ptr), value :: c, fields, tau, stream      ! device addresses, CUDA stream
      integer(c_int), value :: nxaa, nyaa, nzaa
    end function
    integer(c_int) function coral_closure_attach(h, c) bind(C, name="coral_closure_attach")
      import :: c_int, c_ptr
      type(c_ptr), value :: h, c
    end function
  end interface
end module coral_b200_c
