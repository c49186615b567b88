! dynamics_gpu.f90 -- the reference's `dynamics` (src/nd.f90:60-199) with its
! time-step loop on the B200 library.
!
! Drop-in: build the reference's sources (src/*.f90) with this file in place
! of the `dynamics` subroutine of src/nd.f90 (lines 60-199), compile
! ndyn_gpu_mod.f90 first, and link ndyn_omp_b200/lib/libndyn_gpu.so:
!
!   gfortran -O2 -fopenmp -c ndyn_gpu_mod.f90
!   gfortran -O2 -fopenmp <reference modules and sources, dynamics removed> \
!            dynamics_gpu.f90 -L<repo>/ndyn_omp_b200/lib -lndyn_gpu -lstdc++
!
! The prologue (skin default, MCELL, NeiMax, the messages) and the output
! (write_thermo lines, write_model every ConfOuts steps) stay the
! reference's; the loop body of src/nd.f90:137-180 runs on the GPU, in pieces
! that end where write_model is due.  The module state (pos, vel, acc, box,
! force, step, potential, kinetic, virial, NlistUpdates) is copied back, so
! the routines that run after dynamics see what the reference leaves.
! A nonzero status stops the program with the reference's message, where
! the reference would STOP.
module ndyn_gpu_dynamics
  use iso_c_binding
  use ndyn_gpu
  implicit none
contains

  ! write_thermo (src/read_input.f90:433-446) from one library record
  subroutine ndg_thermo_line(t, user) bind(C)
    type(ndg_thermo), intent(in) :: t
    type(c_ptr), value :: user
    write(6, '(x,i8,x,g14.6,x,g14.6,x,g14.6,x,g14.6,x,g14.6)') &
      t%step, t%potential, t%kinetic, t%energy_error, t%pressure, t%volume
    call flush(6)
  end subroutine ndg_thermo_line

  subroutine ndg_check(rc, what)
    integer(c_int), intent(in) :: rc
    character(*), intent(in) :: what
    if (rc /= NDG_OK) then
      write(0,'(A)') what//': '//trim(ndg_message(rc))
      STOP 'ndyn_gpu'
    endif
  end subroutine ndg_check

end module ndyn_gpu_dynamics

subroutine dynamics
  use omp_lib
  use iso_c_binding
  use ndyn_gpu
  use ndyn_gpu_dynamics
  use mostCommon
  use control
  use interpot
  use listData
  use groupStuff
  implicit none
  type(c_ptr) :: ctx
  type(ndg_control) :: ctl
  integer(c_int) :: rc, sys, nrun, done
  integer(c_int), allocatable :: spring(:), dirs(:,:)
  real(8) :: pe, vir(6), ke
  integer :: g

  ! the reference's prologue, src/nd.f90:73-108
  if (.not.allocated(pos)) then
    call read_model
  endif
  if (skin < 0.d0) then
    skin = rcut*0.2d0
  endif
  MCELL(1) = int(box(1)/(rcut+skin))
  MCELL(2) = int(box(2)/(rcut+skin))
  MCELL(3) = int(box(3)/(rcut+skin))
  NCELL = MCELL(1)*MCELL(2)*MCELL(3)
  write(6,'(A,3i4)') "# Number of link cell: ",MCELL
  if (NeiMax.eq.0) then
    NeiMax = int(4./3.*PI*((rcut+skin)*1.1)**3*np/(box(1)*box(2)*box(3)))
  endif
  write(6,'(A,i4)') "# Estimating max number of neighbours: ",NeiMax
  if (.not.allocated(mass)) then
     allocate( mass(Ntypes), typeName(Ntypes) )
     mass(1) = 1.d0; typeName(1) = "test"
  endif
  if (ConfOuts.eq.0) ConfOuts = step_num
  if (trim(ModelOutType).eq.'NA') ModelOutType='xyz'
  if (springpots.and..not.allocated( ipos )) call initPositionSet
  skinsq = skin*skin

  ! the system on the device
  rc = ndg_create(ctx, 0, NDG_PREC_FP64)
  call ndg_check(rc, 'ndg_create')
  rc = ndg_add_system(ctx, np, Ntypes, NPairs, PTsize, PTrMin, mass, PairMat, &
                      PairParams(1,1:NPairs), PPairTable, FPairTable, typ, pos, vel, acc, box, sys)
  call ndg_check(rc, 'ndg_add_system')
  ctl = ndg_control(dt, skin, NeiMax, merge(1,0,ReNei), ReNeiFreq, OutSteps, step, &
                    merge(1,0,isokinetic), KEfreq, KEtarget, KEparm, merge(1,0,isobaric), &
                    Pfreq, Ptarget, Pparm, merge(1,0,isoenergetic), Efreq, Eparm, &
                    merge(1,0,boxLoad), boxVel, NDG_QUIRK_REF)
  rc = ndg_set_control(ctx, sys, ctl)
  call ndg_check(rc, 'ndg_set_control')
  if (springpots) then
    allocate( spring(NPairs) )
    spring = merge(1, 0, PairName(1:NPairs) == "spring")
    rc = ndg_set_springs(ctx, sys, spring, PairParams)
    call ndg_check(rc, 'ndg_set_springs')
    rc = ndg_set_initial_positions(ctx, sys, ipos, initBox)
    call ndg_check(rc, 'ndg_set_initial_positions')
  endif
  if (Nhold > 0) then
    ! displacement conditions: the axes bcDir marks on groups of type 'd'
    allocate( dirs(3,Nhold) )
    do g = 1, Nhold
      dirs(:,g) = merge(1, 0, bcDir(:,g) .and. bcTyp(g) == 'd')
    enddo
    rc = ndg_set_holds(ctx, sys, hold, Nhold, dirs, bcParm(1:3,1:Nhold))
    call ndg_check(rc, 'ndg_set_holds')
  endif

  write(6,'(a)') ''
  write(6,'(a)') '#  Computing initial forces and energies.'
  write(6,'(a,i8)') '#  Number of time steps: ', step_num
  write(6,'(a,g14.6)') '#  Time step increment: ', dt
  write(6,'(a,g14.6)') '#  Cutoff radius: ', rcut
  write(6,'(a,g14.6)') '#  Cutoff skin: ', skin
  write(6,'(a)') '# Model Output format: '//trim(ModelOutType)
  write(6,'(a)') ''
  write(6,'(a)') '#  Step   Potential     Kinetic        EnergyError    pressure       volume'
  call flush(6)
  box0(1:3) = box(1:3)

  wtime = omp_get_wtime ( )
  open(11,file='out.'//trim(ModelOutType),position="append")
  call write_model(11)

  ! the loop of src/nd.f90:137-180 in pieces that end where write_model is
  ! due (mod(step,ConfOuts) == 0); ndg_run builds the lists first, as the
  ! prologue's buildCellList does, and ndg_run_continue carries the run on
  done = 0
  do while (done < step_num)
    nrun = min(step_num - done, ConfOuts - mod(step + done, ConfOuts))
    if (done == 0) then
      rc = ndg_run(ctx, nrun, c_funloc(ndg_thermo_line), c_null_ptr)
    else
      rc = ndg_run_continue(ctx, nrun, c_funloc(ndg_thermo_line), c_null_ptr)
    endif
    call ndg_check(rc, 'ndg_run')
    done = done + nrun
    if (mod(step + done, ConfOuts) == 0) then
      rc = ndg_get_state(ctx, sys, pos, vel, acc, box)
      call ndg_check(rc, 'ndg_get_state')
      step = step + done
      call write_model(11)
      step = step - done
    endif
  end do

  ! the module state the reference leaves behind
  rc = ndg_get_state(ctx, sys, pos, vel, acc, box)
  call ndg_check(rc, 'ndg_get_state')
  rc = ndg_get_control(ctx, sys, ctl)
  call ndg_check(rc, 'ndg_get_control')
  step = ctl%step
  rc = ndg_get_forces(ctx, sys, force, pe, vir, ke)
  call ndg_check(rc, 'ndg_get_forces')
  potential = pe; kinetic = ke; virial = vir
  rc = ndg_get_list_updates(ctx, sys, NlistUpdates)
  call ndg_check(rc, 'ndg_get_list_updates')
  rc = ndg_destroy(ctx)

  call flush(0);   call flush(6);   call flush(11)
  close(11)

  wtime = omp_get_wtime ( ) - wtime
  write(6, '(a,i8)' ) '# Number of neighbour list updates:',NlistUpdates
  write(6, '(a)' ) ''
  write(6, '(a)' ) '#  Elapsed time for main dynamics:'
  write(6, '(a,g14.6,a)' ) '#  ',wtime, ' seconds'
  call timestamp ( )

  Return
end subroutine dynamics
