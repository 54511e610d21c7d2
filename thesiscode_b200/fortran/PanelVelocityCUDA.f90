module PanelVelocityCUDAModule
!  Drop-in replacement for PanelVelocityParallelModule (PanelVelocityParallel.f90:1-20 in the
!  reference) on top of the C ABI of libthesiscode_b200 (include/thesiscode_b200.h).
!  A BVE driver switches by replacing `use PanelVelocityParallelModule` with
!  `use PanelVelocityCUDAModule`; the public names, argument lists and module state are the same:
!
!      BVERK4(aParticles, aPanels, dt, procRank, numProcs)     :435-658
!      StratosphereRK4(aParticles, aPanels, t, dt, procRank, numProcs)  :661-919
!      InitializeMPIRK4, FinalizeMPIRK4, LoadBalance           :126-230
!      ResetRK4, SetSmooth, GetSmooth, ResetArea               :96-120, :321
!      totalKE, kineticEnergy                                  :25-26
!
!  Rank r uses GPU r mod (number of visible GPUs). With numProcs > 1, BVERK4 shards like the
!  reference (:465-489): every rank holds the whole state on its GPU, computes the LoadBalance
!  rows (:182-204) of each class for each RK4 stage (tc_rk4_stage_range), and after each stage
!  the ranks exchange the next stage's packed source rows of the active panels with one
!  MPI_ALLGATHERV (the reference broadcasts every class's velocity rows instead); the final rows
!  of every class are gathered once per step. StratosphereRK4 runs the whole step on every
!  rank (identical results). GatherPanels / ScatterPanels run on the host as in the reference.
!
!  Build: needs the reference's ParticlesEdgesPanelsModule and TracerAndVorticityDistributionModule,
!  MPI, and a link against libthesiscode_b200.so, e.g.
!      mpif90 -O2 -c PanelVelocityCUDA.f90 && mpif90 ... -L<lib dir> -lthesiscode_b200
use iso_c_binding
use NumberKindsModule
use ParticlesEdgesPanelsModule
use TracerAndVorticityDistributionModule, only : Omega

implicit none

include 'mpif.h'

private
public totalKE, kineticEnergy
public BVERK4, StratosphereRK4, ResetRK4, ResetArea, SetSmooth, GetSmooth
public InitializeMPIRK4, FinalizeMPIRK4, LoadBalance
public SetPrecisionCUDA

integer(c_int), parameter :: TC_FP64 = 0, TC_FP32C = 1
integer(c_int), parameter :: TC_BUF_SOURCES = 0, TC_BUF_XA = 1, TC_BUF_ZETA = 2, TC_BUF_XV = 3, &
                             TC_BUF_XQ = 4, TC_BUF_KE = 5

interface
  integer(c_int) function tc_create(device, precision, ctx) bind(C, name="tc_create")
    import :: c_int, c_ptr
    integer(c_int), value :: device, precision
    type(c_ptr) :: ctx
  end function
  integer(c_int) function tc_destroy(ctx) bind(C, name="tc_destroy")
    import :: c_int, c_ptr
    type(c_ptr), value :: ctx
  end function
  integer(c_int) function tc_set_omega(ctx, omega) bind(C, name="tc_set_omega")
    import :: c_int, c_ptr, c_double
    type(c_ptr), value :: ctx
    real(c_double), value :: omega
  end function
  integer(c_int) function tc_set_deltas(ctx, da, dv, dq) bind(C, name="tc_set_deltas")
    import :: c_int, c_ptr, c_double
    type(c_ptr), value :: ctx
    real(c_double), value :: da, dv, dq
  end function
  integer(c_int) function tc_reset_rk4(ctx) bind(C, name="tc_reset_rk4")
    import :: c_int, c_ptr
    type(c_ptr), value :: ctx
  end function
  integer(c_int) function tc_rk4_step(ctx, xA, zetaA, areaA, nA, xV, nV, xQ, nQ, dt, nsteps, &
                                      tke, ke) bind(C, name="tc_rk4_step")
    import :: c_int, c_ptr, c_double
    type(c_ptr), value :: ctx
    real(c_double) :: xA(3,*), zetaA(*), areaA(*), xV(3,*), xQ(3,*), tke(*), ke(*)
    integer(c_int), value :: nA, nV, nQ, nsteps
    real(c_double), value :: dt
  end function
  integer(c_int) function tc_strat_rk4_step(ctx, xA, absVortA, relVortA, areaA, nA, xV, &
                                            absVortV, relVortV, nV, xQ, nQ, t, dt, nsteps, &
                                            tke, ke) bind(C, name="tc_strat_rk4_step")
    import :: c_int, c_ptr, c_double
    type(c_ptr), value :: ctx
    real(c_double) :: xA(3,*), absVortA(*), relVortA(*), areaA(*), xV(3,*), absVortV(*), &
                      relVortV(*), xQ(3,*), tke(*), ke(*)
    integer(c_int), value :: nA, nV, nQ, nsteps
    real(c_double), value :: t, dt
  end function
  type(c_ptr) function tc_last_error() bind(C, name="tc_last_error")
    import :: c_ptr
  end function
  integer(c_int) function tc_device_count(count) bind(C, name="tc_device_count")
    import :: c_int
    integer(c_int) :: count
  end function
  integer(c_int) function tc_synchronize(ctx) bind(C, name="tc_synchronize")
    import :: c_int, c_ptr
    type(c_ptr), value :: ctx
  end function
  integer(c_int) function tc_rk4_load(ctx, xA, zetaA, areaA, nA, xV, nV, xQ, nQ, onDevice) &
                                      bind(C, name="tc_rk4_load")
    import :: c_int, c_ptr, c_double
    type(c_ptr), value :: ctx
    real(c_double) :: xA(3,*), zetaA(*), areaA(*), xV(3,*), xQ(3,*)
    integer(c_int), value :: nA, nV, nQ, onDevice
  end function
  integer(c_int) function tc_rk4_store(ctx, xA, zetaA, xV, xQ, ke, onDevice) &
                                       bind(C, name="tc_rk4_store")
    import :: c_int, c_ptr, c_double
    type(c_ptr), value :: ctx
    real(c_double) :: xA(3,*), zetaA(*), xV(3,*), xQ(3,*), ke(*)
    integer(c_int), value :: onDevice
  end function
  integer(c_int) function tc_rk4_pack_sources(ctx) bind(C, name="tc_rk4_pack_sources")
    import :: c_int, c_ptr
    type(c_ptr), value :: ctx
  end function
  integer(c_int) function tc_rk4_stage_range(ctx, stage, dt, a0, a1, v0, v1, q0, q1, keDevice) &
                                             bind(C, name="tc_rk4_stage_range")
    import :: c_int, c_ptr, c_double
    type(c_ptr), value :: ctx, keDevice
    integer(c_int), value :: stage, a0, a1, v0, v1, q0, q1
    real(c_double), value :: dt
  end function
  integer(c_int) function tc_rk4_copy_rows(ctx, which, row0, nrows, ptr, toBuffer) &
                                           bind(C, name="tc_rk4_copy_rows")
    import :: c_int, c_ptr
    type(c_ptr), value :: ctx, ptr
    integer(c_int), value :: which, row0, nrows, toBuffer
  end function
end interface

real(kreal), allocatable, save :: kineticEnergy(:)
real(kreal), save :: totalKE = 0.0_kreal
real(kreal), save :: smooth = 0.05_kreal
logical(klog), save :: resetAreas = .False.
logical(klog), save :: rk4IsReady = .False.
logical(klog), save :: mpiIsReady = .False.
integer(c_int), save :: precisionMode = TC_FP64
type(c_ptr), save :: ctx = c_null_ptr
type(Panels), pointer, save :: activePanels => null(), passivePanels => null()
integer(kint), allocatable, save :: activeMap(:), passiveMap(:)
integer(kint), allocatable, save :: particlesIndexStart(:), particlesIndexEnd(:), &
                                    activePanelsIndexStart(:), activePanelsIndexEnd(:), &
                                    passivePanelsIndexStart(:), passivePanelsIndexEnd(:)

contains

subroutine SetSmooth(newSmooth)
  real(kreal), intent(in) :: newSmooth
  smooth = newSmooth
end subroutine

function GetSmooth()
  real(kreal) :: GetSmooth
  GetSmooth = smooth
end function

subroutine ResetArea(onOff)
  logical(klog), intent(in), optional :: onOff
  if (present(onOff)) then
    resetAreas = onOff
  else
    resetAreas = .True.
  endif
end subroutine

subroutine SetPrecisionCUDA(fp32Compensated)
  ! Selects the FP32-compensated pair arithmetic (.true.) or FP64 (.false., the default).
  logical(klog), intent(in) :: fp32Compensated
  if (fp32Compensated) then
    precisionMode = TC_FP32C
  else
    precisionMode = TC_FP64
  endif
  if (c_associated(ctx)) call FreeContext()
end subroutine

subroutine CheckStatus(rc, where)
  integer(c_int), intent(in) :: rc
  character(len=*), intent(in) :: where
  if (rc /= 0) then
    print *, where, " ERROR : libthesiscode_b200 status ", rc
    stop
  endif
end subroutine

subroutine FreeContext()
  integer(c_int) :: rc
  if (c_associated(ctx)) then
    rc = tc_destroy(ctx)
    ctx = c_null_ptr
  endif
end subroutine

subroutine InitializeMPIRK4(aParticles, aPanels, procRank, numProcs)
  type(Particles), intent(in) :: aParticles
  type(Panels), intent(in) :: aPanels
  integer(kint), intent(in) :: procRank, numProcs
  integer(c_int) :: rc
  allocate(particlesIndexStart(0:numProcs-1), particlesIndexEnd(0:numProcs-1))
  allocate(activePanelsIndexStart(0:numProcs-1), activePanelsIndexEnd(0:numProcs-1))
  allocate(passivePanelsIndexStart(0:numProcs-1), passivePanelsIndexEnd(0:numProcs-1))
  mpiIsReady = .True.
  call LoadBalance(aParticles, aPanels, numProcs)
  call EnsureContext(procRank)
end subroutine

subroutine EnsureContext(procRank)
  ! One context per rank, on GPU procRank mod (number of visible GPUs).
  integer(kint), intent(in) :: procRank
  integer(c_int) :: rc, nDevices
  if (c_associated(ctx)) return
  rc = tc_device_count(nDevices)
  call CheckStatus(rc, "EnsureContext device count")
  rc = tc_create(int(mod(procRank, max(nDevices, 1)), c_int), precisionMode, ctx)
  call CheckStatus(rc, "EnsureContext")
end subroutine

subroutine LoadBalance(aParticles, aPanels, numProcs)
  ! Same contiguous partition as the reference (:182-204); the GPU step does not need it but
  ! drivers read the index arrays.
  type(Particles), intent(in) :: aParticles
  type(Panels), intent(in) :: aPanels
  integer(kint), intent(in) :: numProcs
  integer(kint) :: chunkSize, j
  chunkSize = aParticles%N / numProcs
  do j = 0, numProcs - 1
    particlesIndexStart(j) = j*chunkSize + 1
    particlesIndexEnd(j) = (j+1)*chunkSize
  enddo
  particlesIndexEnd(numProcs-1) = aParticles%N
  chunkSize = aPanels%N_Active / numProcs
  do j = 0, numProcs - 1
    activePanelsIndexStart(j) = j*chunkSize + 1
    activePanelsIndexEnd(j) = (j+1)*chunkSize
  enddo
  activePanelsIndexEnd(numProcs-1) = aPanels%N_Active
  chunkSize = (aPanels%N - aPanels%N_Active) / numProcs
  do j = 0, numProcs - 1
    passivePanelsIndexStart(j) = j*chunkSize + 1
    passivePanelsIndexEnd(j) = (j+1)*chunkSize
  enddo
  passivePanelsIndexEnd(numProcs-1) = aPanels%N - aPanels%N_Active
end subroutine

subroutine FinalizeMPIRK4()
  if (rk4IsReady) call ResetRK4()
  if (allocated(particlesIndexStart)) then
    deallocate(particlesIndexStart, particlesIndexEnd, activePanelsIndexStart)
    deallocate(activePanelsIndexEnd, passivePanelsIndexStart, passivePanelsIndexEnd)
  endif
  call FreeContext()
  mpiIsReady = .False.
end subroutine

subroutine ResetRK4()
  integer(c_int) :: rc
  if (allocated(activeMap)) deallocate(activeMap)
  if (allocated(passiveMap)) deallocate(passiveMap)
  if (allocated(kineticEnergy)) deallocate(kineticEnergy)
  if (associated(activePanels)) then
    call Delete(activePanels)
    deallocate(activePanels)
  endif
  if (associated(passivePanels)) then
    call Delete(passivePanels)
    deallocate(passivePanels)
  endif
  if (c_associated(ctx)) rc = tc_reset_rk4(ctx)
  rk4IsReady = .False.
end subroutine

subroutine InitRK4(aParticles, aPanels)
  type(Particles), intent(in) :: aParticles
  type(Panels), intent(in) :: aPanels
  integer(kint) :: nActive, nPassive
  nActive = aPanels%N_Active
  nPassive = aPanels%N - aPanels%N_Active
  allocate(activePanels, passivePanels)
  allocate(activeMap(nActive), passiveMap(nPassive), kineticEnergy(nActive))
  call New(activePanels, nActive, GetPanelKind(aPanels), GetNTracer(aPanels), GetProblemKind(aPanels))
  call New(passivePanels, nPassive, GetPanelKind(aPanels), GetNTracer(aPanels), GetProblemKind(aPanels))
  activePanels%N = nActive
  activePanels%N_Active = nActive
  passivePanels%N = nPassive
  rk4IsReady = .True.
end subroutine

subroutine BVERK4(aParticles, aPanels, dt, procRank, numProcs)
  type(Particles), intent(inout) :: aParticles
  type(Panels), intent(inout) :: aPanels
  real(kreal), intent(in) :: dt
  integer(kint), intent(in) :: procRank, numProcs
  integer(c_int) :: rc
  real(c_double) :: tke(1)
  if (procRank < 0 .OR. numProcs < 1 .OR. procRank >= numProcs) then
    print *, "BVERK4 ERROR : bad MPI arguments ", procRank, numProcs
    return
  endif
  call EnsureContext(procRank)
  if (.NOT. rk4IsReady) then
    call InitRK4(aParticles, aPanels)
    if (numProcs > 1) then
      if (.NOT. mpiIsReady) call InitializeMPIRK4(aParticles, aPanels, procRank, numProcs)
      call LoadBalance(aParticles, aPanels, numProcs)
    endif
  endif
  call GatherPanels(aPanels, activePanels, activeMap, passivePanels, passiveMap)
  rc = tc_set_omega(ctx, real(Omega, c_double))
  call CheckStatus(rc, "BVERK4 omega")
  rc = tc_set_deltas(ctx, 0.0_c_double, 0.0_c_double, real(smooth, c_double))
  call CheckStatus(rc, "BVERK4 smooth")
  if (numProcs == 1) then
    rc = tc_rk4_step(ctx, activePanels%x, activePanels%relVort, activePanels%area, &
                     int(activePanels%N, c_int), aParticles%x, int(aParticles%N, c_int), &
                     passivePanels%x, int(passivePanels%N, c_int), real(dt, c_double), 1_c_int, &
                     tke, kineticEnergy)
    call CheckStatus(rc, "BVERK4 step")
    totalKE = tke(1)
  else
    call ShardedStep(aParticles, dt, procRank, numProcs)
  endif
  if (GetNTracer(aPanels) >= 2) activePanels%tracer(:,2) = kineticEnergy
  ! :651 particles' relative vorticity follows the new latitude
  aParticles%relVort(1:aParticles%N) = aParticles%absVort(1:aParticles%N) &
                                       - 2.0_kreal*Omega*aParticles%x(3,1:aParticles%N)
  call ScatterPanels(aPanels, activePanels, activeMap, passivePanels, passiveMap)
end subroutine

subroutine ShardedStep(aParticles, dt, procRank, numProcs)
  ! One RK4 step over numProcs ranks: this rank's LoadBalance rows of each stage on its GPU, the
  ! next stage's source rows exchanged after every stage, every class gathered at the end.
  type(Particles), intent(inout) :: aParticles
  real(kreal), intent(in) :: dt
  integer(kint), intent(in) :: procRank, numProcs
  integer(c_int) :: rc, stage, nA, nV, nQ
  nA = int(activePanels%N, c_int)
  nV = int(aParticles%N, c_int)
  nQ = int(passivePanels%N, c_int)
  rc = tc_rk4_load(ctx, activePanels%x, activePanels%relVort, activePanels%area, nA, &
                   aParticles%x, nV, passivePanels%x, nQ, 0_c_int)
  call CheckStatus(rc, "BVERK4 load")
  rc = tc_rk4_pack_sources(ctx)
  call CheckStatus(rc, "BVERK4 sources")
  do stage = 0, 3
    ! 1-based inclusive LoadBalance indices -> 0-based half-open rows
    rc = tc_rk4_stage_range(ctx, stage, real(dt, c_double), &
                            int(activePanelsIndexStart(procRank) - 1, c_int), &
                            int(activePanelsIndexEnd(procRank), c_int), &
                            int(particlesIndexStart(procRank) - 1, c_int), &
                            int(particlesIndexEnd(procRank), c_int), &
                            int(passivePanelsIndexStart(procRank) - 1, c_int), &
                            int(passivePanelsIndexEnd(procRank), c_int), c_null_ptr)
    call CheckStatus(rc, "BVERK4 stage")
    call AllgatherRows(TC_BUF_SOURCES, 4, activePanelsIndexStart, activePanelsIndexEnd, &
                       procRank, numProcs)
  enddo
  ! final state of every class and the stage-1 kinetic energy, all rows on every rank
  call AllgatherRows(TC_BUF_XA, 3, activePanelsIndexStart, activePanelsIndexEnd, procRank, numProcs)
  call AllgatherRows(TC_BUF_ZETA, 1, activePanelsIndexStart, activePanelsIndexEnd, procRank, numProcs)
  call AllgatherRows(TC_BUF_KE, 1, activePanelsIndexStart, activePanelsIndexEnd, procRank, numProcs)
  call AllgatherRows(TC_BUF_XV, 3, particlesIndexStart, particlesIndexEnd, procRank, numProcs)
  if (nQ > 0) call AllgatherRows(TC_BUF_XQ, 3, passivePanelsIndexStart, passivePanelsIndexEnd, &
                                 procRank, numProcs)
  rc = tc_rk4_store(ctx, activePanels%x, activePanels%relVort, aParticles%x, passivePanels%x, &
                    kineticEnergy, 0_c_int)
  call CheckStatus(rc, "BVERK4 store")
  totalKE = 0.5_kreal*sum(kineticEnergy*activePanels%area(1:activePanels%N))   ! :500
end subroutine

subroutine AllgatherRows(which, width, indexStart, indexEnd, procRank, numProcs)
  ! Rows [indexStart(j), indexEnd(j)] (1-based) of RK4 buffer `which` (width doubles per row)
  ! computed by rank j are copied to every rank: device -> host, MPI_ALLGATHERV, host -> device.
  integer(c_int), intent(in) :: which
  integer(kint), intent(in) :: width, procRank, numProcs
  integer(kint), intent(in) :: indexStart(0:), indexEnd(0:)
  real(c_double), allocatable, target :: mine(:), everyone(:)
  integer(kint) :: counts(0:numProcs-1), displs(0:numProcs-1), j, total, mpiErrorCode
  integer(c_int) :: rc
  do j = 0, numProcs - 1
    counts(j) = width*(indexEnd(j) - indexStart(j) + 1)
    displs(j) = width*(indexStart(j) - 1)
  enddo
  total = displs(numProcs-1) + counts(numProcs-1)
  allocate(mine(max(counts(procRank), 1)), everyone(max(total, 1)))
  if (counts(procRank) > 0) then
    rc = tc_rk4_copy_rows(ctx, which, int(indexStart(procRank) - 1, c_int), &
                          int(indexEnd(procRank) - indexStart(procRank) + 1, c_int), c_loc(mine), &
                          0_c_int)
    call CheckStatus(rc, "AllgatherRows export")
  endif
  rc = tc_synchronize(ctx)
  call CheckStatus(rc, "AllgatherRows synchronize")
  call MPI_ALLGATHERV(mine, counts(procRank), MPI_DOUBLE_PRECISION, everyone, counts, displs, &
                      MPI_DOUBLE_PRECISION, MPI_COMM_WORLD, mpiErrorCode)
  if (mpiErrorCode /= MPI_SUCCESS) then
    print *, "AllgatherRows ERROR : MPI_ALLGATHERV returned ", mpiErrorCode
    stop
  endif
  do j = 0, numProcs - 1
    if (j /= procRank .AND. counts(j) > 0) then
      rc = tc_rk4_copy_rows(ctx, which, int(indexStart(j) - 1, c_int), &
                            int(indexEnd(j) - indexStart(j) + 1, c_int), c_loc(everyone(displs(j)+1)), &
                            1_c_int)
      call CheckStatus(rc, "AllgatherRows import")
    endif
  enddo
  rc = tc_synchronize(ctx)
  call CheckStatus(rc, "AllgatherRows synchronize")
  deallocate(mine, everyone)
end subroutine

subroutine StratosphereRK4(aParticles, aPanels, t, dt, procRank, numProcs)
  ! Forced model (:661-919): positions advance; the relative vorticity of panels and particles
  ! is rebuilt from absVort, the rotation and the Juckes forcing at t + dt (:908-915).
  type(Particles), intent(inout) :: aParticles
  type(Panels), intent(inout) :: aPanels
  real(kreal), intent(in) :: t, dt
  integer(kint), intent(in) :: procRank, numProcs
  integer(c_int) :: rc
  real(c_double) :: tke(1)
  if (procRank < 0 .OR. numProcs < 1 .OR. procRank >= numProcs) then
    print *, "StratosphereRK4 ERROR : bad MPI arguments ", procRank, numProcs
    return
  endif
  call EnsureContext(procRank)
  if (.NOT. rk4IsReady) call InitRK4(aParticles, aPanels)
  call GatherPanels(aPanels, activePanels, activeMap, passivePanels, passiveMap)
  rc = tc_set_omega(ctx, real(Omega, c_double))
  call CheckStatus(rc, "StratosphereRK4 omega")
  rc = tc_set_deltas(ctx, 0.0_c_double, 0.0_c_double, real(smooth, c_double))
  call CheckStatus(rc, "StratosphereRK4 smooth")
  rc = tc_strat_rk4_step(ctx, activePanels%x, activePanels%absVort, activePanels%relVort, &
                         activePanels%area, int(activePanels%N, c_int), aParticles%x, &
                         aParticles%absVort, aParticles%relVort, int(aParticles%N, c_int), &
                         passivePanels%x, int(passivePanels%N, c_int), real(t, c_double), &
                         real(dt, c_double), 1_c_int, tke, kineticEnergy)
  call CheckStatus(rc, "StratosphereRK4 step")
  totalKE = tke(1)
  if (GetNTracer(aPanels) >= 2) activePanels%tracer(:,2) = kineticEnergy
  call ScatterPanels(aPanels, activePanels, activeMap, passivePanels, passiveMap)
end subroutine

end module
