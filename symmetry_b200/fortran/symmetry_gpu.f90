! symmetry_gpu.f90 -- ISO_C_BINDING interface to libsymmetry_b200.so.
!
! A Fortran driver shaped like the reference's main program replaces the
! bodies of its per-timestep subroutines with calls into the GPU library.
! Device state lives behind an opaque handle; host arrays keep the
! reference's layout (populations (0:18,z,y,x), scalars (z,y,x)).
! This file has not been compiled: no Fortran compiler exists on the build
! image.  Its bind(C) interfaces mirror include/symmetry.h one to one.
module symmetry_gpu
  use, intrinsic :: iso_c_binding
  implicit none

  integer(c_int), parameter :: SYM_OK = 0
  integer(c_int), parameter :: SYM_MODE_REFERENCE = 0, SYM_MODE_CONFIG = 1
  integer(c_int), parameter :: SYM_STORE_FP64 = 0, SYM_STORE_FP32 = 1, SYM_STORE_FP16 = 2
  integer(c_int), parameter :: SYM_F_RI = 0, SYM_F_BI = 1, SYM_F_FI = 2, SYM_F_FFI = 3, &
       SYM_F_RHO = 4, SYM_F_UX = 5, SYM_F_UY = 6, SYM_F_UZ = 7, SYM_F_RHO_N = 8, SYM_F_RHO_R = 9, &
       SYM_F_RHO_B = 10, SYM_F_NX = 11, SYM_F_NY = 12, SYM_F_NZ = 13, SYM_F_GRADX = 14, &
       SYM_F_GRADY = 15, SYM_F_GRADZ = 16, SYM_F_FLAG = 17, SYM_F_WALLS = 18, SYM_F_WALLS_OLD = 19, &
       SYM_F_WALLS_ALL = 20, SYM_F_PIN = 21, SYM_F_POUT = 22
  integer, parameter :: SYM_MAX_PAR = 32

  type, bind(C) :: sym_params
     integer(c_int32_t) :: nx, ny, nz, mode, wall_x, storage, par, la_m, la_n, bounce
     real(c_double) :: rho0, nu_r, nu_b, s_e, s_eps, s_q, s_pi, s_m, sigma, beta, cita
     real(c_double) :: body(3)
     real(c_double) :: rad, rho_p, mass, inertia, fg, alpha, evap_lim
  end type sym_params

  type, bind(C) :: sym_particles
     real(c_double) :: center(3*SYM_MAX_PAR), center_old(3*SYM_MAX_PAR), center0(3*SYM_MAX_PAR)
     real(c_double) :: up(3*SYM_MAX_PAR), rp(3*SYM_MAX_PAR), fp(3*SYM_MAX_PAR), tp(3*SYM_MAX_PAR)
     real(c_double) :: fre(3*SYM_MAX_PAR), tension(3*SYM_MAX_PAR), tension_t(3*SYM_MAX_PAR)
     real(c_double) :: shb(SYM_MAX_PAR)
  end type sym_particles

  interface
     integer(c_int) function sym_params_reference(p, nx, ny, nz) bind(C, name="sym_params_reference")
       import :: c_int, sym_params
       type(sym_params), intent(out) :: p
       integer(c_int), value :: nx, ny, nz
     end function
     integer(c_int) function sym_create(p, device, h) bind(C, name="sym_create")
       import :: c_int, c_ptr, sym_params
       type(sym_params), intent(in) :: p
       integer(c_int), value :: device
       type(c_ptr), intent(out) :: h
     end function
     integer(c_int) function sym_destroy(h) bind(C, name="sym_destroy")
       import :: c_int, c_ptr
       type(c_ptr), value :: h
     end function
     integer(c_int) function sym_set_field(h, field, host) bind(C, name="sym_set_field")
       import :: c_int, c_ptr
       type(c_ptr), value :: h
       integer(c_int), value :: field
       type(c_ptr), value :: host
     end function
     integer(c_int) function sym_get_field(h, field, host) bind(C, name="sym_get_field")
       import :: c_int, c_ptr
       type(c_ptr), value :: h
       integer(c_int), value :: field
       type(c_ptr), value :: host
     end function
     integer(c_int) function sym_set_particles(h, s) bind(C, name="sym_set_particles")
       import :: c_int, c_ptr, sym_particles
       type(c_ptr), value :: h
       type(sym_particles), intent(in) :: s
     end function
     integer(c_int) function sym_get_particles(h, s) bind(C, name="sym_get_particles")
       import :: c_int, c_ptr, sym_particles
       type(c_ptr), value :: h
       type(sym_particles), intent(out) :: s
     end function
     integer(c_int) function sym_streaming(h, which) bind(C, name="sym_streaming")
       import :: c_int, c_ptr
       type(c_ptr), value :: h
       integer(c_int), value :: which
     end function
     integer(c_int) function sym_step(h, nsteps) bind(C, name="sym_step")
       import :: c_int, c_ptr
       type(c_ptr), value :: h
       integer(c_int), value :: nsteps
     end function
     integer(c_int) function sym_output3(h, hmin, y0) bind(C, name="sym_output3")
       import :: c_int, c_ptr, c_double, c_int32_t
       type(c_ptr), value :: h
       real(c_double), intent(out) :: hmin
       integer(c_int32_t), intent(out) :: y0
     end function
     ! output steps (Source1.f90:218-234); paths are NUL-terminated character arrays
     integer(c_int) function sym_get_macros(h, rho, ux, uy, uz, rho_n) bind(C, name="sym_get_macros")
       import :: c_int, c_ptr
       type(c_ptr), value :: h, rho, ux, uy, uz, rho_n
     end function
     integer(c_int) function sym_energy(h, out) bind(C, name="sym_energy")
       import :: c_int, c_ptr, c_double
       type(c_ptr), value :: h
       real(c_double), intent(out) :: out(6)
     end function
     integer(c_int) function sym_output_results(h, path) bind(C, name="sym_output_results")
       import :: c_int, c_ptr, c_char
       type(c_ptr), value :: h
       character(kind=c_char), intent(in) :: path(*)
     end function
     integer(c_int) function sym_output_result2(h, prefix, t, tr) bind(C, name="sym_output_result2")
       import :: c_int, c_ptr, c_char, c_double
       type(c_ptr), value :: h
       character(kind=c_char), intent(in) :: prefix(*)
       integer(c_int), value :: t
       real(c_double), value :: tr
     end function
     integer(c_int) function sym_output3_write(h, path, t, tr, rad_c, lamda_d) bind(C, name="sym_output3_write")
       import :: c_int, c_ptr, c_char, c_double
       type(c_ptr), value :: h
       character(kind=c_char), intent(in) :: path(*)
       integer(c_int), value :: t
       real(c_double), value :: tr, rad_c, lamda_d
     end function
     integer(c_int) function sym_output4(h, path, t, tr, rad_c, wcap_acc) bind(C, name="sym_output4")
       import :: c_int, c_ptr, c_char, c_double
       type(c_ptr), value :: h
       character(kind=c_char), intent(in) :: path(*)
       integer(c_int), value :: t
       real(c_double), value :: tr, rad_c
       real(c_double), intent(inout) :: wcap_acc
     end function
     ! error flags the fused kernels recorded (SYM_DEV_NONFINITE = 1, SYM_DEV_TIMEOUT = 2)
     integer(c_int) function sym_device_status(h, flags) bind(C, name="sym_device_status")
       import :: c_int, c_ptr, c_int32_t
       type(c_ptr), value :: h
       integer(c_int32_t), intent(out) :: flags
     end function
     ! checkpoint / restart (no counterpart in the reference)
     integer(c_int) function sym_checkpoint_save(h, path) bind(C, name="sym_checkpoint_save")
       import :: c_int, c_ptr, c_char
       type(c_ptr), value :: h
       character(kind=c_char), intent(in) :: path(*)
     end function
     integer(c_int) function sym_checkpoint_load(h, path) bind(C, name="sym_checkpoint_load")
       import :: c_int, c_ptr, c_char
       type(c_ptr), value :: h
       character(kind=c_char), intent(in) :: path(*)
     end function
  end interface

  ! one binding per reference subroutine (Source1.f90 names)
  interface
     integer(c_int) function c_initia_center(h) bind(C, name="sym_initia_center")
       import :: c_int, c_ptr; type(c_ptr), value :: h; end function
     integer(c_int) function c_initialization(h) bind(C, name="sym_initialization")
       import :: c_int, c_ptr; type(c_ptr), value :: h; end function
     integer(c_int) function c_set_walls(h) bind(C, name="sym_set_walls")
       import :: c_int, c_ptr; type(c_ptr), value :: h; end function
     integer(c_int) function c_calmacros(h) bind(C, name="sym_calmacros")
       import :: c_int, c_ptr; type(c_ptr), value :: h; end function
     integer(c_int) function c_derivatives(h) bind(C, name="sym_derivatives")
       import :: c_int, c_ptr; type(c_ptr), value :: h; end function
     integer(c_int) function c_collision(h) bind(C, name="sym_collision")
       import :: c_int, c_ptr; type(c_ptr), value :: h; end function
     integer(c_int) function c_recolor(h) bind(C, name="sym_recolor")
       import :: c_int, c_ptr; type(c_ptr), value :: h; end function
     integer(c_int) function c_boundary(h) bind(C, name="sym_boundary")
       import :: c_int, c_ptr; type(c_ptr), value :: h; end function
     integer(c_int) function c_curve(h) bind(C, name="sym_curve")
       import :: c_int, c_ptr; type(c_ptr), value :: h; end function
     integer(c_int) function c_lagrange_points(h) bind(C, name="sym_lagrange_points")
       import :: c_int, c_ptr; type(c_ptr), value :: h; end function
     integer(c_int) function c_capillary_force2(h) bind(C, name="sym_capillary_force2")
       import :: c_int, c_ptr; type(c_ptr), value :: h; end function
     integer(c_int) function c_momentum(h) bind(C, name="sym_momentum")
       import :: c_int, c_ptr; type(c_ptr), value :: h; end function
     integer(c_int) function c_repulsive(h) bind(C, name="sym_repulsive")
       import :: c_int, c_ptr; type(c_ptr), value :: h; end function
     integer(c_int) function c_movement(h) bind(C, name="sym_movement")
       import :: c_int, c_ptr; type(c_ptr), value :: h; end function
     integer(c_int) function c_refilling(h) bind(C, name="sym_refilling")
       import :: c_int, c_ptr; type(c_ptr), value :: h; end function
  end interface

  type(c_ptr), save :: sym_h = c_null_ptr

contains

  subroutine sym_check(rc, what)
    integer(c_int), intent(in) :: rc
    character(*), intent(in) :: what
    if (rc /= SYM_OK) then
       write(*,*) 'symmetry_gpu: ', what, ' failed with status ', rc
       stop 1
    end if
  end subroutine

  ! same-named replacements of the reference's per-step subroutines: the
  ! arguments stay on the device, so the wrappers take none.
  subroutine gpu_calmacros();        call sym_check(c_calmacros(sym_h), 'calmacros');               end subroutine
  subroutine gpu_derivatives();      call sym_check(c_derivatives(sym_h), 'derivatives');           end subroutine
  subroutine gpu_collision();        call sym_check(c_collision(sym_h), 'collision');               end subroutine
  subroutine gpu_recolor();          call sym_check(c_recolor(sym_h), 'Recolor');                   end subroutine
  subroutine gpu_boundary();         call sym_check(c_boundary(sym_h), 'boundary');                 end subroutine
  subroutine gpu_streaming_r();      call sym_check(sym_streaming(sym_h, 0_c_int), 'streaming(ri)'); end subroutine
  subroutine gpu_streaming_b();      call sym_check(sym_streaming(sym_h, 1_c_int), 'streaming(bi)'); end subroutine
  subroutine gpu_curve();            call sym_check(c_curve(sym_h), 'curve');                       end subroutine
  subroutine gpu_lagrange_points();  call sym_check(c_lagrange_points(sym_h), 'Lagrange_points');   end subroutine
  subroutine gpu_capillary_force2(); call sym_check(c_capillary_force2(sym_h), 'capillary_force2'); end subroutine
  subroutine gpu_momentum();         call sym_check(c_momentum(sym_h), 'momentum');                 end subroutine
  subroutine gpu_repulsive();        call sym_check(c_repulsive(sym_h), 'repulsive');               end subroutine
  subroutine gpu_movement();         call sym_check(c_movement(sym_h), 'movement');                 end subroutine
  subroutine gpu_set_walls();        call sym_check(c_set_walls(sym_h), 'set_walls');               end subroutine
  subroutine gpu_refilling();        call sym_check(c_refilling(sym_h), 'refilling');               end subroutine

end module symmetry_gpu
