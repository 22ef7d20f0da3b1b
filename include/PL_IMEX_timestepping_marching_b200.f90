! PL_IMEX_timestepping_marching_b200.f90 -- a replacement for the include
! PL_IMEX_timestepping_marching.f90 of Coral's plane-layer solver
! (src/plane_layer/PL_IMEX_timestepping.f90:661), for a build whose time step
! runs on a B200 through libcoral_b200.so.
!
! Use: in src/plane_layer/PL_IMEX_timestepping.f90 replace
!        include "PL_IMEX_timestepping_marching.f90"
!      by
!        include "PL_IMEX_timestepping_marching_b200.f90"
!      compile include/coral_b200.f90 (module coral_b200_c) before it, and link
!      with -L<repo>/coral_b200 -lcoral_b200 -lcudart.  plane_layer_main.f90 and
!      the other includes are unchanged.
!
! It defines every procedure the type full_problem_data_structure_T binds to the
! original include (PL_IMEX_timestepping.f90:163-218).  march_forward
! (one_step_beyond) creates the device solver on its first call from the
! working directory's coral.equations, coral.parameters.in, coral.timeseries and
! coral.usrOutput and from the program's command-line switches, copies in the
! state that import_quickSave or noisy_initial_conditions left in the fields,
! and from then on runs each step on the GPU with coral_run (the reference's
! step, its Timeseries/, Volumes/, Slices/ and Profiles/ files at their
! periods), then copies the state back so that export_checkpoints and the other
! host procedures see it.  The stage internals (right-hand sides, solves, NL
! terms) have no host counterpart here and stop if called.  The sources and the
! penalisation mask still come from the user's PL_user_sources_definitions.f90
! and PL_user_penalisation_mask.f90, included as in the reference; they are
! handed to the device when it is created.
!
! Costs of this route against the driver-loop replacement (INTEGRATION.md):
! the host still assembles and factorises its operators (factorize_operators is
! in PL_IMEX_timestepping.f90), and the state crosses PCIe once per step.
!
! No Fortran compiler exists where this file was written: it is checked
! textually (tests/test_capi.py), not compiled.

 subroutine coral_b200_check(rc, what)
   use coral_b200_c
   integer(c_int), intent(in) :: rc
   character(len=*), intent(in) :: what
   character(kind=c_char), pointer :: msg(:)
   integer :: n
   if (rc == CORAL_OK) return
   call c_f_pointer(coral_last_error(coral_b200_handle), msg, [1024])
   n = 0
   do while (n < 1024)
      if (msg(n + 1) == c_null_char) exit
      n = n + 1
   end do
   write (*, '(3a,i0,2a)') 'libcoral_b200: ', what, ' returned ', rc, ': ', transfer(msg(1:n), repeat(' ', n))
   error stop 'libcoral_b200'
 end subroutine coral_b200_check

 ! the whole of a text file, NUL-terminated
 function coral_b200_slurp(path) result(text)
   use coral_b200_c
   character(len=*), intent(in) :: path
   character(len=:), allocatable :: text
   integer :: u, nbytes
   open (newunit=u, file=path, access='stream', form='unformatted', status='old', action='read')
   inquire (unit=u, size=nbytes)
   allocate (character(len=nbytes + 1) :: text)
   read (u) text(1:nbytes)
   close (u)
   text(nbytes + 1:nbytes + 1) = c_null_char
 end function coral_b200_slurp

 ! the switches of the command line that change the solver (coral_create_with_args)
 function coral_b200_switches() result(args)
   use coral_b200_c
   character(len=:), allocatable :: args
   character(len=256) :: a, b
   integer :: k, n
   args = ''
   n = command_argument_count()
   k = 1
   do while (k <= n)
      call get_command_argument(k, a)
      select case (trim(a))
      case ('--withHorizontalSmagorinsky')
         args = args//' '//trim(a)
      case ('--smagorinsky-prefactor', '--cflFactor-along-z')
         if (k < n) then
            call get_command_argument(k + 1, b)
            args = args//' '//trim(a)//' '//trim(b)
            k = k + 1
         end if
      end select
      k = k + 1
   end do
   args = args//c_null_char
 end function coral_b200_switches

 ! create the device solver and give it the host's state, sources and mask
 subroutine coral_b200_start(self)
   use coral_b200_c
   class(full_problem_data_structure_T), intent(inOut) :: self
   character(len=:), allocatable :: eqs, pars, args
   integer :: iVar, iSrc
   logical :: there
   eqs = coral_b200_slurp('coral.equations')
   pars = coral_b200_slurp('coral.parameters.in')
   args = coral_b200_switches()
   call coral_b200_check(coral_create_with_args(eqs, pars, c_null_char, 0_c_int, args, coral_b200_handle), &
                         'coral_create_with_args')
   inquire (file='coral.timeseries', exist=there)
   if (there) call coral_b200_check(coral_set_timeseries_from_file(coral_b200_handle, &
                                    'coral.timeseries'//c_null_char), 'coral_set_timeseries_from_file')
   inquire (file='coral.usrOutput', exist=there)
   if (there) call coral_b200_check(coral_set_usr_output_from_file(coral_b200_handle, &
                                    'coral.usrOutput'//c_null_char), 'coral_set_usr_output_from_file')
   do iSrc = 1, self%numberOf_sources
      if (allocated(self%sources(iSrc)%physical)) &
         call coral_b200_check(coral_set_source(coral_b200_handle, int(iSrc, c_int), self%sources(iSrc)%physical), &
                               'coral_set_source')
   end do
   do iVar = 1, self%recipe%numberOf_linear_variables_full
      if (self%recipe%linear_vars_full(iVar)%penalisation) then
         ! init_penalisation below left the mask (not the field) here
         call coral_b200_check(coral_set_penalisation_mask(coral_b200_handle, self%linear_variables(iVar)%phys), &
                               'coral_set_penalisation_mask')
         exit
      end if
   end do
   call coral_b200_push_state(self)
 end subroutine coral_b200_start

 subroutine coral_b200_push_state(self)
   use coral_b200_c
   class(full_problem_data_structure_T), intent(inOut) :: self
   integer :: iSys
   do iSys = 1, self%recipe%numberOf_coupled_kxky_systems
      call coral_b200_check(coral_set_field(coral_b200_handle, int(iSys - 1, c_int), &
                            self%coupled_kxky_set(iSys)%field), 'coral_set_field')
   end do
   do iSys = 1, self%recipe%numberOf_coupled_zero_systems
      call coral_b200_check(coral_set_mean_field(coral_b200_handle, int(iSys - 1, c_int), &
                            self%coupled_zero_set(iSys)%field), 'coral_set_mean_field')
   end do
 end subroutine coral_b200_push_state

 subroutine coral_b200_pull_state(self)
   use coral_b200_c
   class(full_problem_data_structure_T), intent(inOut) :: self
   integer :: iSys
   do iSys = 1, self%recipe%numberOf_coupled_kxky_systems
      call coral_b200_check(coral_get_field(coral_b200_handle, int(iSys - 1, c_int), &
                            self%coupled_kxky_set(iSys)%field), 'coral_get_field')
   end do
   do iSys = 1, self%recipe%numberOf_coupled_zero_systems
      call coral_b200_check(coral_get_mean_field(coral_b200_handle, int(iSys - 1, c_int), &
                            self%coupled_zero_set(iSys)%field), 'coral_get_mean_field')
   end do
 end subroutine coral_b200_pull_state

 ! march_forward: one step on the GPU (one_step_beyond, marching.f90:3-51), with
 ! the outputs of the step and the CFL time step of its fields
 subroutine one_step_beyond(self, my_dt)
   use coral_b200_c
   class(full_problem_data_structure_T), intent(inOut), target :: self
   real(dp), intent(in) :: my_dt
   real(c_double) :: d3(3)
   if (.not. c_associated(coral_b200_handle)) call coral_b200_start(self)
   ! the host loop owns the clock: the device takes its time, step and dt
   call coral_b200_check(coral_set_time(coral_b200_handle, real(timings%absolute_time, c_double), &
                         real(my_dt, c_double), int(timings%i_timestep, c_long_long)), 'coral_set_time')
   call coral_b200_check(coral_run(coral_b200_handle, 1_c_int, &
                         self%io_bookkeeping%output_directory(1:self%io_bookkeeping%output_dir_length)//c_null_char), &
                         'coral_run')
   call coral_b200_check(coral_diagnostics(coral_b200_handle, d3), 'coral_diagnostics')
   self%cargo%cfl_based_DT = d3(1)
   self%cargo%KE_display = d3(2)
   call coral_b200_pull_state(self)
 end subroutine one_step_beyond

 subroutine compute_cfl_based_timestep(self)
   use coral_b200_c
   class(full_problem_data_structure_T), intent(inOut) :: self
   real(c_double) :: d3(3)
   if (.not. c_associated(coral_b200_handle)) return
   call coral_b200_check(coral_diagnostics(coral_b200_handle, d3), 'coral_diagnostics')
   self%cargo%cfl_based_DT = d3(1)
 end subroutine compute_cfl_based_timestep

 ! the full variables of the current state in physical space, from the device
 subroutine compute_full_variables_in_physical_space(self)
   use coral_b200_c
   class(full_problem_data_structure_T), intent(inOut) :: self
   integer :: iVar
   if (.not. c_associated(coral_b200_handle)) call coral_b200_start(self)
   call coral_b200_push_state(self)
   do iVar = 1, self%recipe%numberOf_linear_variables_full
      if (self%recipe%linear_vars_full(iVar)%penalisation) cycle
      call coral_b200_check(coral_get_full_phys(coral_b200_handle, int(iVar - 1, c_int), &
                            self%linear_variables(iVar)%phys), 'coral_get_full_phys')
   end do
 end subroutine compute_full_variables_in_physical_space

 ! the stage internals run inside coral_run on the device
 subroutine coral_b200_internal(name)
   character(len=*), intent(in) :: name
   write (*, '(3a)') 'PL_IMEX_timestepping_marching_b200: ', name, ' runs on the GPU inside march_forward'
   error stop 'libcoral_b200'
 end subroutine coral_b200_internal

 subroutine LPIMEX_backsolve_to_aux(self)
   class(full_problem_data_structure_T), intent(inOut), target :: self
   call coral_b200_internal('backsolve_to_aux')
 end subroutine LPIMEX_backsolve_to_aux

 subroutine LPIMEX_add_K_hat_to_rhs(self, dsca, i)
   class(full_problem_data_structure_T), intent(inOut) :: self
   integer, intent(in) :: i
   real(kind=dp), intent(in) :: dsca
   call coral_b200_internal('add_K_hat_to_rhs')
 end subroutine LPIMEX_add_K_hat_to_rhs

 subroutine LPIMEX_add_K_std_to_rhs(self, dsca, i)
   class(full_problem_data_structure_T), intent(inOut) :: self
   integer, intent(in) :: i
   real(kind=dp), intent(in) :: dsca
   call coral_b200_internal('add_K_std_to_rhs')
 end subroutine LPIMEX_add_K_std_to_rhs

 subroutine LPIMEX_stif_aux_to_K_std(self, i)
   class(full_problem_data_structure_T), intent(inOut) :: self
   integer, intent(in) :: i
   call coral_b200_internal('stif_aux_to_K_std')
 end subroutine LPIMEX_stif_aux_to_K_std

 subroutine LPIMEX_mass_field_to_rhs(self)
   class(full_problem_data_structure_T), intent(inOut) :: self
   call coral_b200_internal('mass_field_to_rhs')
 end subroutine LPIMEX_mass_field_to_rhs

 subroutine LPIMEX_compute_NL_terms_to_K_hat(self, i)
   class(full_problem_data_structure_T), intent(inOut) :: self
   integer, intent(in) :: i
   call coral_b200_internal('compute_NL_terms_to_K_hat')
 end subroutine LPIMEX_compute_NL_terms_to_K_hat

 ! field <-> aux copies: export_checkpoints backs the fields up in aux
 ! (PL_IMEX_timestepping_output.f90:391) and restores them
 subroutine LPIMEX_copy_aux_to_fields(self)
   class(full_problem_data_structure_T), intent(inOut) :: self
   integer :: iSys
   do iSys = 1, self%recipe%numberOf_coupled_kxky_systems
      self%coupled_kxky_set(iSys)%field = self%coupled_kxky_set(iSys)%aux
   end do
   do iSys = 1, self%recipe%numberOf_coupled_zero_systems
      self%coupled_zero_set(iSys)%field = self%coupled_zero_set(iSys)%aux
   end do
 end subroutine LPIMEX_copy_aux_to_fields

 subroutine LPIMEX_copy_fields_to_aux(self)
   class(full_problem_data_structure_T), intent(inOut) :: self
   integer :: iSys
   do iSys = 1, self%recipe%numberOf_coupled_kxky_systems
      self%coupled_kxky_set(iSys)%aux = self%coupled_kxky_set(iSys)%field
   end do
   do iSys = 1, self%recipe%numberOf_coupled_zero_systems
      self%coupled_zero_set(iSys)%aux = self%coupled_zero_set(iSys)%field
   end do
 end subroutine LPIMEX_copy_fields_to_aux

 ! every (x, y) of a physical field replaced by its horizontal mean (one rank)
 subroutine horizontal_average_of_physical_quantity_inPlace(self, iVar)
   class(full_problem_data_structure_T), intent(inOut) :: self
   integer, intent(in) :: iVar
   real(dp), allocatable :: m(:)
   integer :: ix, iy
   m = sum(sum(self%linear_variables(iVar)%phys, 3), 2) / self%geometry%NXAA / self%geometry%NYAA
   do iy = 1, size(self%linear_variables(iVar)%phys, 3)
      do ix = 1, size(self%linear_variables(iVar)%phys, 2)
         self%linear_variables(iVar)%phys(:, ix, iy) = m
      end do
   end do
 end subroutine horizontal_average_of_physical_quantity_inPlace

 ! the output counters live on the device (coral_set_time sets them from the step)
 subroutine initialise_bookkeeping_counters(self, time_index)
   class(full_problem_data_structure_T), intent(inOut) :: self
   integer, intent(in) :: time_index
   self%io_bookkeeping%time_integer = time_index
 end subroutine initialise_bookkeeping_counters

 ! volumes, slices and profiles are written by coral_run at their periods
 subroutine output_slices_volumes_and_profiles(self)
   class(full_problem_data_structure_T), intent(inOut) :: self
 end subroutine output_slices_volumes_and_profiles

 ! ---- the hooks of the user's PL_user_sources_definitions.f90 ----

 real(kind=dp) function sourceParams(self, paramString)
   class(full_problem_data_structure_T), intent(in) :: self
   character(len=6), intent(in) :: paramString
   integer :: k
   sourceParams = 0._dp
   do k = 1, self%recipe%sources%n_sourceParams
      if (paramString == self%recipe%sources%sourceParams(k)%str) then
         sourceParams = self%recipe%sources%sourceParams(k)%dsca
         return
      end if
   end do
   if (self%recipe%sources%n_sourceParams > 0) then
      write (*, '(3a)') 'sourceParam ', paramString, ' is not in coral.equations'
      error stop 'PL_user_sources_definitions.f90'
   end if
 end function sourceParams

 subroutine allocate_sources(self)
   class(full_problem_data_structure_T), intent(inOut) :: self
   if (allocated(self%sources)) deallocate (self%sources)
   allocate (self%sources(self%numberOf_sources))
 end subroutine allocate_sources

 subroutine add_source_dscalar(self, sourceIndex, definition)
   class(full_problem_data_structure_T), intent(inOut) :: self
   integer, intent(in) :: sourceIndex
   real(dp), intent(in) :: definition
   if (sourceIndex > self%numberOf_sources) error stop 'source index above numberOf_sources'
   if (allocated(self%sources(sourceIndex)%physical)) deallocate (self%sources(sourceIndex)%physical)
   allocate (self%sources(sourceIndex)%physical(self%geometry%NZAA))
   self%sources(sourceIndex)%physical = definition
 end subroutine add_source_dscalar

 subroutine add_source_array(self, sourceIndex, definition)
   class(full_problem_data_structure_T), intent(inOut) :: self
   integer, intent(in) :: sourceIndex
   real(dp), allocatable, intent(in) :: definition(:)
   if (sourceIndex > self%numberOf_sources) error stop 'source index above numberOf_sources'
   self%sources(sourceIndex)%physical = definition
 end subroutine add_source_array

 ! the sources' spectra are made on the device (coral_set_source)
 subroutine transform_sources(self)
   use coral_b200_c
   class(full_problem_data_structure_T), intent(inOut) :: self
   integer :: k
   if (.not. c_associated(coral_b200_handle)) return
   do k = 1, self%numberOf_sources
      if (allocated(self%sources(k)%physical)) &
         call coral_b200_check(coral_set_source(coral_b200_handle, int(k, c_int), self%sources(k)%physical), &
                               'coral_set_source')
   end do
 end subroutine transform_sources

 subroutine init_all_sources(self)
   class(full_problem_data_structure_T), intent(inOut) :: self
   real(kind=dp), allocatable :: z(:)
   real(kind=dp), allocatable :: sourceDef(:)
   call gauss_chebyshev_grid_1d(z, self%geometry%NZAA, self%geometry%center, self%geometry%gap)
   allocate (sourceDef(self%geometry%NZAA))
   include "PL_user_sources_definitions.f90"
   call self%transform_sources()
 end subroutine init_all_sources

 ! the user's masks on the grid, their maximum kept in each penalised variable's
 ! phys (the device forms strength (1 + tanh(width mask)) / 2 itself)
 subroutine init_penalisation(self)
   class(full_problem_data_structure_T), intent(inOut) :: self
   real(dp), allocatable, dimension(:) :: penalisation_mask
   integer :: N_masks, i_mask, iVar, ix, iy, iz
   real(dp) :: pi, x, y, z, lx, ly, zgap, zcenter
   call gauss_chebyshev_grid_1d(self%geometry%zGrid, self%geometry%NZAA, self%geometry%center, self%geometry%gap)
   lx = self%geometry%Lx
   ly = self%geometry%Ly
   zgap = self%geometry%gap
   zcenter = self%geometry%center
   do iVar = 1, self%recipe%numberOf_linear_variables_full
      if (.not. self%recipe%linear_vars_full(iVar)%penalisation) cycle
      do iy = 1, size(self%geometry%yGrid, 1)
         do ix = 1, size(self%geometry%xGrid, 1)
            do iz = 1, self%geometry%NZAA
               x = self%geometry%xGrid(ix)
               y = self%geometry%yGrid(iy)
               z = self%geometry%zGrid(iz)
               i_mask = 0
               include "PL_user_penalisation_mask.f90"
               self%linear_variables(iVar)%phys(iz, ix, iy) = maxval(penalisation_mask)
            end do
         end do
      end do
   end do
 end subroutine init_penalisation
