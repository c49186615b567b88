! ndyn_gpu_mod.f90 -- ISO_C_BINDING interface to the B200 Ndyn timestep
! library (include/ndyn_gpu.h, libndyn_gpu.so).
!
! The reference's timestep routines are argument-less subroutines on module
! globals (src/mods.f90); each interface below takes that module data
! explicitly, in the reference's own layouts: pos/vel/acc/force(3,np)
! real(8) column-major, typ(np), PairMat(Ntypes,Ntypes),
! PPairTable/FPairTable(PTsize+1,NPairs), box(3), virial(6).  Every function
! returns 0 or a negative status where the reference would STOP
! (ndg_error_string gives its message).
!
! Scalars pass by value, arrays and results by reference, the context as a
! type(c_ptr).  The derived types are bind(C) copies of ndg_control and
! ndg_thermo: same fields, same order (tests/test_fortran_binding.py checks
! both against the C header).
module ndyn_gpu
  use iso_c_binding
  implicit none

  integer(c_int), parameter :: NDG_OK = 0, NDG_ERR_ARG = -1, NDG_ERR_NEIMAX = -2, &
       NDG_ERR_OUT_OF_BOX = -3, NDG_ERR_POTENTIAL = -4, NDG_ERR_CELLS = -5, &
       NDG_ERR_NOMEM = -6, NDG_ERR_CUDA = -7
  integer(c_int), parameter :: NDG_PREC_FP64 = 0, NDG_PREC_MIXED = 1
  integer(c_int), parameter :: NDG_QUIRK_REF = 0, NDG_QUIRK_FIXED = 1

  ! module 'control' and 'listData' (src/mods.f90:79-95) of one run
  type, bind(C) :: ndg_control
    real(c_double) :: dt, skin
    integer(c_int) :: neimax, renei, renei_freq, out_steps, step
    integer(c_int) :: isokinetic, ke_freq
    real(c_double) :: ke_target, ke_parm
    integer(c_int) :: isobaric, p_freq
    real(c_double) :: p_target(3), p_parm
    integer(c_int) :: isoenergetic, e_freq
    real(c_double) :: e_parm
    integer(c_int) :: box_load
    real(c_double) :: box_vel(3)
    integer(c_int) :: quirk
  end type ndg_control

  ! one write_thermo record (src/read_input.f90:433-446) with the raw
  ! virial and box
  type, bind(C) :: ndg_thermo
    integer(c_int) :: sys, step
    real(c_double) :: potential, kinetic, energy_error, pressure, volume
    real(c_double) :: virial(6), box(3)
  end type ndg_thermo

  interface
    integer(c_int) function ndg_abi_version() bind(C, name="ndg_abi_version")
      import
    end function
    type(c_ptr) function ndg_error_string(status) bind(C, name="ndg_error_string")
      import
      integer(c_int), value :: status
    end function
    integer(c_int) function ndg_create(ctx, device, precision) bind(C, name="ndg_create")
      import
      type(c_ptr) :: ctx
      integer(c_int), value :: device, precision
    end function
    integer(c_int) function ndg_destroy(ctx) bind(C, name="ndg_destroy")
      import
      type(c_ptr), value :: ctx
    end function
    ! interpot (src/mods.f90:51-77) and the atoms of one system
    integer(c_int) function ndg_add_system(ctx, np, ntypes, npairs, ptsize, ptrmin, mass, &
        pairmat, rcpair, ppair, fpair, typ, pos, vel, acc, box, sys) &
        bind(C, name="ndg_add_system")
      import
      type(c_ptr), value :: ctx
      integer(c_int), value :: np, ntypes, npairs, ptsize
      real(c_double), value :: ptrmin
      real(c_double) :: mass(*), rcpair(*), ppair(*), fpair(*), pos(*), vel(*), acc(*), box(3)
      integer(c_int) :: pairmat(*), typ(*), sys
    end function
    integer(c_int) function ndg_set_control(ctx, sys, c) bind(C, name="ndg_set_control")
      import
      type(c_ptr), value :: ctx
      integer(c_int), value :: sys
      type(ndg_control) :: c
    end function
    integer(c_int) function ndg_get_control(ctx, sys, c) bind(C, name="ndg_get_control")
      import
      type(c_ptr), value :: ctx
      integer(c_int), value :: sys
      type(ndg_control) :: c
    end function
    ! Hold/Disp (src/read_input.f90:177-190): hold(np), bcDir/bcParm per group
    integer(c_int) function ndg_set_holds(ctx, sys, hold, ngroups, dir, du) &
        bind(C, name="ndg_set_holds")
      import
      type(c_ptr), value :: ctx
      integer(c_int), value :: sys, ngroups
      integer(c_int) :: hold(*), dir(*)
      real(c_double) :: du(*)
    end function
    ! spring lines and InitPos (src/read_input.f90:136,165; src/nd.f90:1731-1762)
    integer(c_int) function ndg_set_springs(ctx, sys, spring, params) &
        bind(C, name="ndg_set_springs")
      import
      type(c_ptr), value :: ctx
      integer(c_int), value :: sys
      integer(c_int) :: spring(*)
      real(c_double) :: params(*)
    end function
    integer(c_int) function ndg_set_initial_positions(ctx, sys, ipos, ibox) &
        bind(C, name="ndg_set_initial_positions")
      import
      type(c_ptr), value :: ctx
      integer(c_int), value :: sys
      real(c_double) :: ipos(*), ibox(3)
    end function
    integer(c_int) function ndg_load_state(ctx, sys, pos, vel, acc, box) &
        bind(C, name="ndg_load_state")
      import
      type(c_ptr), value :: ctx
      integer(c_int), value :: sys
      real(c_double) :: pos(*), vel(*), acc(*), box(*)
    end function
    integer(c_int) function ndg_get_state(ctx, sys, pos, vel, acc, box) &
        bind(C, name="ndg_get_state")
      import
      type(c_ptr), value :: ctx
      integer(c_int), value :: sys
      real(c_double) :: pos(*), vel(*), acc(*), box(*)
    end function
    ! the dynamics loop (src/nd.f90:137-180); cb receives type(ndg_thermo)
    integer(c_int) function ndg_run(ctx, nsteps, cb, user) bind(C, name="ndg_run")
      import
      type(c_ptr), value :: ctx, user
      integer(c_int), value :: nsteps
      type(c_funptr), value :: cb
    end function
    integer(c_int) function ndg_run_continue(ctx, nsteps, cb, user) &
        bind(C, name="ndg_run_continue")
      import
      type(c_ptr), value :: ctx, user
      integer(c_int), value :: nsteps
      type(c_funptr), value :: cb
    end function
    integer(c_int) function ndg_get_list_updates(ctx, sys, n) &
        bind(C, name="ndg_get_list_updates")
      import
      type(c_ptr), value :: ctx
      integer(c_int), value :: sys
      integer(c_int) :: n
    end function
    ! one call per reference routine, with the reference's flags
    integer(c_int) function ndg_setup_lists(ctx) bind(C, name="ndg_setup_lists")
      import
      type(c_ptr), value :: ctx
    end function
    integer(c_int) function ndg_build_cell_list(ctx) bind(C, name="ndg_build_cell_list")
      import
      type(c_ptr), value :: ctx
    end function
    integer(c_int) function ndg_check_list_update(ctx, n) bind(C, name="ndg_check_list_update")
      import
      type(c_ptr), value :: ctx
      integer(c_int) :: n
    end function
    integer(c_int) function ndg_integrate1(ctx) bind(C, name="ndg_integrate1")
      import
      type(c_ptr), value :: ctx
    end function
    integer(c_int) function ndg_compute(ctx, cv, cu) bind(C, name="ndg_compute")
      import
      type(c_ptr), value :: ctx
      integer(c_int), value :: cv, cu
    end function
    integer(c_int) function ndg_integrate2(ctx, ck) bind(C, name="ndg_integrate2")
      import
      type(c_ptr), value :: ctx
      integer(c_int), value :: ck
    end function
    integer(c_int) function ndg_mk_iso_ke(ctx, sys) bind(C, name="ndg_mk_iso_ke")
      import
      type(c_ptr), value :: ctx
      integer(c_int), value :: sys
    end function
    integer(c_int) function ndg_mk_iso_e(ctx, sys) bind(C, name="ndg_mk_iso_e")
      import
      type(c_ptr), value :: ctx
      integer(c_int), value :: sys
    end function
    integer(c_int) function ndg_mk_iso_p(ctx, sys) bind(C, name="ndg_mk_iso_p")
      import
      type(c_ptr), value :: ctx
      integer(c_int), value :: sys
    end function
    integer(c_int) function ndg_get_forces(ctx, sys, f, pe, vir, ke) &
        bind(C, name="ndg_get_forces")
      import
      type(c_ptr), value :: ctx
      integer(c_int), value :: sys
      real(c_double) :: f(*), pe, vir(6), ke
    end function
  end interface

contains

  ! the library's text for a status, as a Fortran string
  function ndg_message(status) result(msg)
    integer(c_int), intent(in) :: status
    character(len=80) :: msg
    character(kind=c_char), pointer :: p(:)
    integer :: k
    msg = ' '
    call c_f_pointer(ndg_error_string(status), p, [80])
    do k = 1, 80
      if (p(k) == c_null_char) exit
      msg(k:k) = p(k)
    end do
  end function ndg_message

end module ndyn_gpu
