!--------------------------------------------------------------------------------------------------
!> @brief Drop-in for DAMASK's grid mechanical solver 'spectral_basic' on one B200: the five
!> procedures the grid driver selects (src/grid/DAMASK_grid.f90:110-119,171-206), with the
!> signatures of grid_mechanical_spectral_basic_* (src/grid/grid_mech_spectral_basic.f90:103,243,
!> 284,361,378), forwarding to the C-ABI of libdamask_b200 (include/damask_b200.h) through
!> ISO_C_BINDING.  The solver fields and the per-voxel phase state live in device memory; the
!> host keeps the increment loop, load cases, cutback and output triggers.
!>
!> Selected in DAMASK_grid.f90 by one more case of `solver: mechanical:`:
!>   case ('spectral_basic_b200')
!>     grid_mechanical_init         => grid_mechanical_spectral_b200_init
!>     grid_mechanical_forward      => grid_mechanical_spectral_b200_forward
!>     grid_mechanical_solution     => grid_mechanical_spectral_b200_solution
!>     grid_mechanical_updateCoords => grid_mechanical_spectral_b200_updateCoords
!>     grid_mechanical_restartWrite => grid_mechanical_spectral_b200_restartWrite
!> and, since the mechanical phase state is on the device, materialpoint_forward is followed by
!> grid_mechanical_spectral_b200_materialpointForward (phase_mechanical.f90:987-1002 on the GPU).
!>
!> Scope of this module: one phase (Hooke + phenopowerlaw slip, cF or cI), one constituent per
!> material point, one MPI rank (the whole grid on one GPU).  It uses DAMASK's own modules and is
!> compiled inside the reference's source tree (src/grid), linked with -ldamask_b200.
!--------------------------------------------------------------------------------------------------
module grid_mechanical_spectral_b200
  use, intrinsic :: ISO_C_BINDING
  use HDF5
  use prec
  use parallelization
  use CLI
  use IO
  use types
  use config
  use math
  use rotations
  use HDF5_utilities
  use discretization
  use discretization_grid
  use material
  use spectral_utilities, only: tSolutionState
  use grid_utilities, only: tBCmech

  implicit none(type,external)
  private

  ! C-ABI types, field for field as in include/damask_b200.h
  type, bind(C) :: dmk_phase
    integer(C_INT)  :: lattice, n_families, N_sl(4)
    real(C_DOUBLE)  :: C11, C12, C44
    real(C_DOUBLE)  :: dot_gamma_0(4), n(4), a(4), h_0(4), xi_0(4), xi_inf(4), c_1(4), c_2(4), f_sat(4)
    integer(C_INT)  :: n_h
    real(C_DOUBLE)  :: h_sl_sl(64)
    integer(C_INT)  :: n_nonschmid
    real(C_DOUBLE)  :: a_nonschmid(6)
    real(C_DOUBLE)  :: atol_xi, atol_gamma
  end type dmk_phase

  type, bind(C) :: dmk_numerics
    integer(C_INT)  :: N_iter_min, N_iter_max
    real(C_DOUBLE)  :: eps_abs_div, eps_rel_div, eps_abs_P, eps_rel_P
    integer(C_INT)  :: update_gamma, divergence_correction, derivative
    real(C_DOUBLE)  :: r_cutback_min, r_cutback, r_increase, eps_rel_state
    integer(C_INT)  :: N_iter_state_max, N_iter_Lp_max
    real(C_DOUBLE)  :: r_linesearch_Lp, eps_rel_Lp, eps_abs_Lp
    integer(C_INT)  :: f_update_jacobi_Lp, N_iter_Li_max
    real(C_DOUBLE)  :: r_linesearch_Li, eps_rel_Li, eps_abs_Li
    integer(C_INT)  :: f_update_jacobi_Li, snes_type, anderson_m, solver
    real(C_DOUBLE)  :: alpha, beta, eps_abs_curl, eps_rel_curl
    integer(C_INT)  :: snes_max_it
  end type dmk_numerics

  type, bind(C) :: dmk_bc
    real(C_DOUBLE)  :: values(9)
    integer(C_INT)  :: mask(9)                                                                      !< 1 where the component is 'x'
    integer(C_INT)  :: type                                                                         !< 0 none, 1 L, 2 dot_F, 3 F, 4 P, 5 dot_P
  end type dmk_bc

  type, bind(C) :: dmk_solution_state
    integer(C_INT)  :: iterationsNeeded, converged, stagConverged, residualEvals
    real(C_DOUBLE)  :: err_div, err_BC, P_av(9)
  end type dmk_solution_state

  type, bind(C) :: dmk_restart
    type(C_PTR)     :: F, F_lastinc, F_phase, F_p, L_p, omega_plastic
    real(C_DOUBLE)  :: P_aim(9), F_aim(9), F_aim_lastinc(9), F_aimDot(9)
    real(C_DOUBLE)  :: C_volAvg(81), C_volAvgLastInc(81), C_minMaxAvg(81)
    type(C_PTR)     :: F_tau, F_tau_lastinc
  end type dmk_restart

  interface
    integer(C_INT) function dmk_mech_init(ctx, cells, geomSize, materialAt, n_materials, quaternions, phase, num, &
                                          precision, device) bind(C, name='dmk_mech_init')
      import :: C_INT, C_DOUBLE, C_PTR, dmk_phase, dmk_numerics
      type(C_PTR),        intent(out)        :: ctx
      integer(C_INT),     intent(in)         :: cells(3), materialAt(*)
      real(C_DOUBLE),     intent(in)         :: geomSize(3), quaternions(4,*)
      integer(C_INT),     value              :: n_materials, precision, device
      type(dmk_phase),    intent(in)         :: phase
      type(dmk_numerics), intent(in)         :: num
    end function dmk_mech_init
    integer(C_INT) function dmk_mech_forward(ctx, cutBack, guess, dt, dt_old, t_remaining, deformation, stress, &
                                             q_rot) bind(C, name='dmk_mech_forward')
      import :: C_INT, C_DOUBLE, C_PTR, dmk_bc
      type(C_PTR),    value      :: ctx
      integer(C_INT), value      :: cutBack, guess
      real(C_DOUBLE), value      :: dt, dt_old, t_remaining
      type(dmk_bc),   intent(in) :: deformation, stress
      real(C_DOUBLE), intent(in) :: q_rot(4)
    end function dmk_mech_forward
    integer(C_INT) function dmk_mech_solution(ctx, out) bind(C, name='dmk_mech_solution')
      import :: C_INT, C_PTR, dmk_solution_state
      type(C_PTR),              value       :: ctx
      type(dmk_solution_state), intent(out) :: out
    end function dmk_mech_solution
    integer(C_INT) function dmk_materialpoint_forward(ctx) bind(C, name='dmk_materialpoint_forward')
      import :: C_INT, C_PTR
      type(C_PTR), value :: ctx
    end function dmk_materialpoint_forward
    integer(C_INT) function dmk_mech_update_coords(ctx) bind(C, name='dmk_mech_update_coords')
      import :: C_INT, C_PTR
      type(C_PTR), value :: ctx
    end function dmk_mech_update_coords
    integer(C_INT) function dmk_get_coords(ctx, ip, nodes) bind(C, name='dmk_get_coords')
      import :: C_INT, C_DOUBLE, C_PTR
      type(C_PTR),    value :: ctx
      real(C_DOUBLE)        :: ip(3,*), nodes(3,*)
    end function dmk_get_coords
    integer(C_INT) function dmk_restart_write(ctx, r) bind(C, name='dmk_restart_write')
      import :: C_INT, C_PTR, dmk_restart
      type(C_PTR),       value         :: ctx
      type(dmk_restart), intent(inout) :: r
    end function dmk_restart_write
    integer(C_INT) function dmk_restart_read(ctx, r) bind(C, name='dmk_restart_read')
      import :: C_INT, C_PTR, dmk_restart
      type(C_PTR),       value      :: ctx
      type(dmk_restart), intent(in) :: r
    end function dmk_restart_read
    type(C_PTR) function dmk_last_error() bind(C, name='dmk_last_error')
      import :: C_PTR
    end function dmk_last_error
  end interface

  type(C_PTR)     :: ctx = C_NULL_PTR
  type(dmk_phase) :: phase_b200
  integer         :: Ns = 0                                                                         !< active slip systems
  character(len=pSTRLEN) :: incInfo

  public :: &
    grid_mechanical_spectral_b200_init, &
    grid_mechanical_spectral_b200_forward, &
    grid_mechanical_spectral_b200_solution, &
    grid_mechanical_spectral_b200_updateCoords, &
    grid_mechanical_spectral_b200_restartWrite, &
    grid_mechanical_spectral_b200_materialpointForward

contains

!--------------------------------------------------------------------------------------------------
!> @brief The phase, numerics and microstructure into a device context; F := I and the initial
!> constitutive sweep (grid_mech_spectral_basic.f90:103-237), or the state of the restart increment.
!--------------------------------------------------------------------------------------------------
subroutine grid_mechanical_spectral_b200_init(num_grid_mech)

  type(tDict), pointer, intent(in) :: num_grid_mech

  type(dmk_numerics) :: num
  real(C_DOUBLE), dimension(:,:), allocatable :: q
  integer(C_INT), dimension(:), allocatable :: materialAt
  integer :: ma


  print'(/,1x,a)', '<<<+-  grid_mechanical_spectral_b200 init  -+>>>'; flush(IO_STDOUT)

  if (worldsize /= 1) call IO_error(894_pI16, ext_msg='spectral_basic_b200 runs the grid on one GPU (one MPI rank)')

  call read_phase(phase_b200)
  call read_numerics(num_grid_mech, num)

  allocate(q(4,size(material_O_0)))
  do ma = 1, size(material_O_0)
    if (size(material_O_0(ma)%data) /= 1) &
      call IO_error(148_pI16, ext_msg='spectral_basic_b200: one constituent per material point')
    q(1:4,ma) = material_O_0(ma)%data(1)%asQuaternion()
  end do
  materialAt = int(discretization_materialAt - 1, C_INT)                                            ! 0-based for the C-ABI

  call check(dmk_mech_init(ctx, int(cells,C_INT), real(geomSize,C_DOUBLE), materialAt, int(size(q,2),C_INT), q, &
                           phase_b200, num, 0_C_INT, 0_C_INT), 'dmk_mech_init')

  if (CLI_restartInc > 0) call restart_read()

end subroutine grid_mechanical_spectral_b200_init


!--------------------------------------------------------------------------------------------------
!> @brief grid_mechanical_spectral_basic_solution (grid_mech_spectral_basic.f90:243-277)
!--------------------------------------------------------------------------------------------------
function grid_mechanical_spectral_b200_solution(incInfoIn) result(solution)

  character(len=*), intent(in) :: incInfoIn
  type(tSolutionState)         :: solution

  type(dmk_solution_state) :: s
  integer(C_INT) :: rc


  incInfo = incInfoIn
  rc = dmk_mech_solution(ctx, s)
  if (rc < 0) call check(rc, 'dmk_mech_solution')                                                  ! library errors stop; constitutive failures are reported as not converged
  solution%converged        = s%converged /= 0
  solution%stagConverged    = s%stagConverged /= 0
  solution%iterationsNeeded = s%iterationsNeeded
  print'(/,1x,a,i0,a,es11.4,a,es11.4)', '... fixed point: ', s%iterationsNeeded, &
    ' iterations, error divergence ', s%err_div, ', error BC ', s%err_BC

end function grid_mechanical_spectral_b200_solution


!--------------------------------------------------------------------------------------------------
!> @brief grid_mechanical_spectral_basic_forward (grid_mech_spectral_basic.f90:284-355)
!--------------------------------------------------------------------------------------------------
subroutine grid_mechanical_spectral_b200_forward(cutBack,guess,Delta_t,Delta_t_old,t_remaining,&
                                                 deformation_BC,stress_BC,rotation_BC)

  logical,         intent(in) :: &
    cutBack, &
    guess
  real(pREAL),     intent(in) :: &
    Delta_t_old, &
    Delta_t, &
    t_remaining
  type(tBCmech),   intent(in) :: &
    stress_BC, &
    deformation_BC
  type(tRotation), intent(in) :: &
    rotation_BC


  call check(dmk_mech_forward(ctx, merge(1_C_INT,0_C_INT,cutBack), merge(1_C_INT,0_C_INT,guess), &
                              real(Delta_t,C_DOUBLE), real(Delta_t_old,C_DOUBLE), real(t_remaining,C_DOUBLE), &
                              as_bc(deformation_BC), as_bc(stress_BC), real(rotation_BC%asQuaternion(),C_DOUBLE)), &
             'dmk_mech_forward')

end subroutine grid_mechanical_spectral_b200_forward


!--------------------------------------------------------------------------------------------------
!> @brief grid_mechanical_spectral_basic_updateCoords (grid_mech_spectral_basic.f90:361-372): the
!> coordinates are integrated on the device and handed to the discretization.
!--------------------------------------------------------------------------------------------------
subroutine grid_mechanical_spectral_b200_updateCoords()

  real(C_DOUBLE), dimension(:,:), allocatable :: ip, nodes


  allocate(ip(3,product(cells)), nodes(3,product(cells+1)))
  call check(dmk_mech_update_coords(ctx), 'dmk_mech_update_coords')
  call check(dmk_get_coords(ctx, ip, nodes), 'dmk_get_coords')
  call discretization_setIPcoords(real(ip,pREAL))
  call discretization_setNodeCoords(real(nodes,pREAL))

end subroutine grid_mechanical_spectral_b200_updateCoords


!--------------------------------------------------------------------------------------------------
!> @brief The solver's and the mechanical phase's restart data (grid_mech_spectral_basic.f90:
!> 378-416, phase_mechanical.f90:1248-1261) from the device into <job>_restart.hdf5.
!--------------------------------------------------------------------------------------------------
subroutine grid_mechanical_spectral_b200_restartWrite()

  type(dmk_restart) :: r
  real(C_DOUBLE), dimension(:,:), allocatable, target :: F, F_lastinc, F_phase, F_p, L_p, omega
  integer(HID_T) :: fileHandle, groupHandle
  integer :: N


  N = product(cells)
  allocate(F(9,N), F_lastinc(9,N), F_phase(9,N), F_p(9,N), L_p(9,N), omega(2*Ns,N))
  r%F = c_loc(F); r%F_lastinc = c_loc(F_lastinc); r%F_phase = c_loc(F_phase)
  r%F_p = c_loc(F_p); r%L_p = c_loc(L_p); r%omega_plastic = c_loc(omega)
  r%F_tau = C_NULL_PTR; r%F_tau_lastinc = C_NULL_PTR
  call check(dmk_restart_write(ctx, r), 'dmk_restart_write')

  print'(1x,a)', 'saving solver data required for restart'; flush(IO_STDOUT)

  fileHandle  = HDF5_openFile(CLI_jobName//'_restart.hdf5','a')
  groupHandle = HDF5_addGroup(fileHandle,'solver')
  call HDF5_write(reshape(F,[3,3,N]),groupHandle,'F')
  call HDF5_write(reshape(F_lastinc,[3,3,N]),groupHandle,'F_lastinc')
  call HDF5_write(reshape(r%P_aim,[3,3]),groupHandle,'P_aim',.false.)
  call HDF5_write(reshape(r%F_aim,[3,3]),groupHandle,'F_aim',.false.)
  call HDF5_write(reshape(r%F_aim_lastinc,[3,3]),groupHandle,'F_aim_lastinc',.false.)
  call HDF5_write(reshape(r%F_aimDot,[3,3]),groupHandle,'F_aimDot',.false.)
  call HDF5_write(reshape(r%C_volAvg,[3,3,3,3]),groupHandle,'C_volAvg',.false.)
  call HDF5_write(reshape(r%C_volAvgLastInc,[3,3,3,3]),groupHandle,'C_volAvgLastInc',.false.)
  call HDF5_write(reshape(r%C_minMaxAvg,[3,3,3,3]),groupHandle,'C_minMaxAvg',.false.)
  call HDF5_closeGroup(groupHandle)
  groupHandle = HDF5_addGroup(fileHandle,'phase')
  groupHandle = HDF5_addGroup(groupHandle,material_name_phase(1))
  call HDF5_write(omega,groupHandle,'omega_plastic')
  call HDF5_write(reshape(F_phase,[3,3,N]),groupHandle,'F')
  call HDF5_write(reshape(F_p,[3,3,N]),groupHandle,'F_p')
  call HDF5_write(spread(math_I3,3,N),groupHandle,'F_i')
  call HDF5_write(reshape(L_p,[3,3,N]),groupHandle,'L_p')
  call HDF5_write(spread(math_0(),3,N),groupHandle,'L_i')
  call HDF5_closeGroup(groupHandle)
  call HDF5_closeFile(fileHandle)

contains
  pure function math_0() result(z)
    real(pREAL), dimension(3,3) :: z
    z = 0.0_pREAL
  end function math_0

end subroutine grid_mechanical_spectral_b200_restartWrite


!--------------------------------------------------------------------------------------------------
!> @brief mechanical_forward (phase_mechanical.f90:987-1002) of the device-resident phase state.
!--------------------------------------------------------------------------------------------------
subroutine grid_mechanical_spectral_b200_materialpointForward()

  call check(dmk_materialpoint_forward(ctx), 'dmk_materialpoint_forward')

end subroutine grid_mechanical_spectral_b200_materialpointForward


!--------------------------------------------------------------------------------------------------
!> @brief The restart increment's data from <job>_restart.hdf5 (the groups written above).
!--------------------------------------------------------------------------------------------------
subroutine restart_read()

  type(dmk_restart) :: r
  real(pREAL), dimension(:,:,:), allocatable :: t33n
  real(pREAL), dimension(3,3) :: t33
  real(pREAL), dimension(3,3,3,3) :: t3333
  real(C_DOUBLE), dimension(:,:), allocatable, target :: F, F_lastinc, F_phase, F_p, L_p, omega
  integer(HID_T) :: fileHandle, groupHandle
  integer :: N


  N = product(cells)
  allocate(F(9,N), F_lastinc(9,N), F_phase(9,N), F_p(9,N), L_p(9,N), omega(2*Ns,N), t33n(3,3,N))
  print'(1x,a,1x,i0)', 'loading restart data of increment', CLI_restartInc; flush(IO_STDOUT)

  fileHandle  = HDF5_openFile(CLI_jobName//'_restart.hdf5','r')
  groupHandle = HDF5_openGroup(fileHandle,'solver')
  call HDF5_read(t33n,groupHandle,'F');              F = reshape(t33n,[9,N])
  call HDF5_read(t33n,groupHandle,'F_lastinc');      F_lastinc = reshape(t33n,[9,N])
  call HDF5_read(t33,groupHandle,'P_aim',.false.);   r%P_aim = reshape(t33,[9])
  call HDF5_read(t33,groupHandle,'F_aim',.false.);   r%F_aim = reshape(t33,[9])
  call HDF5_read(t33,groupHandle,'F_aim_lastinc',.false.); r%F_aim_lastinc = reshape(t33,[9])
  call HDF5_read(t33,groupHandle,'F_aimDot',.false.); r%F_aimDot = reshape(t33,[9])
  call HDF5_read(t3333,groupHandle,'C_volAvg',.false.);        r%C_volAvg = reshape(t3333,[81])
  call HDF5_read(t3333,groupHandle,'C_volAvgLastInc',.false.); r%C_volAvgLastInc = reshape(t3333,[81])
  call HDF5_read(t3333,groupHandle,'C_minMaxAvg',.false.);     r%C_minMaxAvg = reshape(t3333,[81])
  call HDF5_closeGroup(groupHandle)
  groupHandle = HDF5_openGroup(fileHandle,'phase/'//material_name_phase(1))
  call HDF5_read(omega,groupHandle,'omega_plastic')
  call HDF5_read(t33n,groupHandle,'F');    F_phase = reshape(t33n,[9,N])
  call HDF5_read(t33n,groupHandle,'F_p');  F_p = reshape(t33n,[9,N])
  call HDF5_read(t33n,groupHandle,'L_p');  L_p = reshape(t33n,[9,N])
  call HDF5_closeGroup(groupHandle)
  call HDF5_closeFile(fileHandle)

  r%F = c_loc(F); r%F_lastinc = c_loc(F_lastinc); r%F_phase = c_loc(F_phase)
  r%F_p = c_loc(F_p); r%L_p = c_loc(L_p); r%omega_plastic = c_loc(omega)
  r%F_tau = C_NULL_PTR; r%F_tau_lastinc = C_NULL_PTR
  call check(dmk_restart_read(ctx, r), 'dmk_restart_read')

end subroutine restart_read


!--------------------------------------------------------------------------------------------------
!> @brief Hooke + phenopowerlaw of the single phase, with the keys of phase_mechanical_elastic.f90
!> and phase_mechanical_plastic_phenopowerlaw.f90:146-168,264-285.
!--------------------------------------------------------------------------------------------------
subroutine read_phase(p)

  type(dmk_phase), intent(out) :: p

  type(tDict), pointer :: phases, phase, mech, elastic, plastic
  integer, dimension(:), allocatable :: N_sl
  real(pREAL), dimension(:), allocatable :: h
  real(pREAL), dimension(:,:), allocatable :: a_nS
  character(len=:), allocatable :: lattice
  integer :: nf


  phases => config_material%get_dict('phase')
  if (phases%length /= 1) call IO_error(180_pI16, ext_msg='spectral_basic_b200: one phase')
  phase   => phases%get_dict(1)
  mech    => phase%get_dict('mechanical')
  elastic => mech%get_dict('elastic')
  plastic => mech%get_dict('plastic')
  if (elastic%get_asStr('type') /= 'Hooke') call IO_error(200_pI16, label1='elasticity', ext_msg=elastic%get_asStr('type'))
  if (plastic%get_asStr('type') /= 'phenopowerlaw') &
    call IO_error(200_pI16, label1='plasticity', ext_msg=plastic%get_asStr('type'))
  lattice = phase%get_asStr('lattice')
  select case (lattice)
    case ('cF'); p%lattice = 0
    case ('cI'); p%lattice = 1
    case default; call IO_error(130_pI16, ext_msg='spectral_basic_b200: lattice '//lattice)
  end select

  N_sl = plastic%get_as1dInt('N_sl')
  nf = size(N_sl)
  if (nf > 4) call IO_error(145_pI16, ext_msg='spectral_basic_b200: at most 4 slip families')
  p%n_families = int(nf,C_INT)
  p%N_sl = 0
  p%N_sl(1:nf) = int(N_sl,C_INT)
  Ns = sum(N_sl)
  p%C11 = elastic%get_asReal('C_11')
  p%C12 = elastic%get_asReal('C_12')
  p%C44 = elastic%get_asReal('C_44')
  p%dot_gamma_0 = 0.0_C_DOUBLE; p%n = 0.0_C_DOUBLE; p%a = 0.0_C_DOUBLE; p%h_0 = 0.0_C_DOUBLE
  p%xi_0 = 0.0_C_DOUBLE; p%xi_inf = 0.0_C_DOUBLE; p%c_1 = 0.0_C_DOUBLE; p%c_2 = 1.0_C_DOUBLE; p%f_sat = 0.0_C_DOUBLE
  p%dot_gamma_0(1:nf) = plastic%get_as1dReal('dot_gamma_0_sl',requiredSize=nf)
  p%n(1:nf)           = plastic%get_as1dReal('n_sl',requiredSize=nf)
  p%a(1:nf)           = plastic%get_as1dReal('a_sl',requiredSize=nf)
  p%h_0(1:nf)         = plastic%get_as1dReal('h_0_sl-sl',requiredSize=nf)
  p%xi_0(1:nf)        = plastic%get_as1dReal('xi_0_sl',requiredSize=nf)
  p%xi_inf(1:nf)      = plastic%get_as1dReal('xi_inf_sl',requiredSize=nf)
  h = plastic%get_as1dReal('h_sl-sl')
  if (size(h) > 64) call IO_error(146_pI16, ext_msg='spectral_basic_b200: at most 64 h_sl-sl values')
  p%n_h = int(size(h),C_INT)
  p%h_sl_sl = 0.0_C_DOUBLE
  p%h_sl_sl(1:size(h)) = h
  a_nS = plastic%get_as2dReal('a_non-Schmid',defaultVal=reshape(emptyRealArray,[0,0]))
  p%n_nonschmid = 0
  p%a_nonschmid = 0.0_C_DOUBLE
  if (size(a_nS) > 0) then
    p%n_nonschmid = int(min(size(a_nS,2),6),C_INT)
    p%a_nonschmid(1:p%n_nonschmid) = a_nS(1,1:p%n_nonschmid)
  end if
  p%atol_xi    = plastic%get_asReal('atol_xi',defaultVal=1.0_pREAL)
  p%atol_gamma = plastic%get_asReal('atol_gamma',defaultVal=1.0e-6_pREAL)

end subroutine read_phase


!--------------------------------------------------------------------------------------------------
!> @brief solver.grid.mechanical (grid_mech_spectral_basic.f90:130-136), solver.grid (FFT options,
!> spectral_utilities.f90:176-224) and phase.mechanical (phase_mechanical.f90:281-295).
!--------------------------------------------------------------------------------------------------
subroutine read_numerics(num_grid_mech, n)

  type(tDict), pointer, intent(in) :: num_grid_mech
  type(dmk_numerics), intent(out) :: n

  type(tDict), pointer :: num_grid, num_mech, num_plastic
  character(len=:), allocatable :: petsc_options
  integer :: i


  num_grid    => config_numerics%get_dict('solver',defaultVal=emptyDict)
  num_grid    => num_grid%get_dict('grid',defaultVal=emptyDict)
  num_mech    => config_numerics%get_dict('phase',defaultVal=emptyDict)
  num_mech    => num_mech%get_dict('mechanical',defaultVal=emptyDict)
  num_plastic => num_mech%get_dict('plastic',defaultVal=emptyDict)

  n%N_iter_min   = num_grid_mech%get_asInt('N_iter_min',defaultVal=1)
  n%N_iter_max   = num_grid_mech%get_asInt('N_iter_max',defaultVal=100)
  n%update_gamma = merge(1_C_INT,0_C_INT,num_grid_mech%get_asBool('update_gamma',defaultVal=.false.))
  n%eps_abs_div  = num_grid_mech%get_asReal('eps_abs_div(P)',defaultVal=1.0e-4_pREAL)
  n%eps_rel_div  = num_grid_mech%get_asReal('eps_rel_div(P)',defaultVal=5.0e-4_pREAL)
  n%eps_abs_P    = num_grid_mech%get_asReal('eps_abs_P',defaultVal=1.0e3_pREAL)
  n%eps_rel_P    = num_grid_mech%get_asReal('eps_rel_P',defaultVal=1.0e-3_pREAL)
  petsc_options  = num_grid_mech%get_asStr('PETSc_options',defaultVal='')
  n%snes_type    = merge(0_C_INT,1_C_INT,index(petsc_options,'-snes_type nrichardson') > 0)
  n%snes_max_it  = 50                                                                               ! PETSc's default, or -snes_max_it N
  i = index(petsc_options,'-snes_max_it')
  if (i > 0) read(petsc_options(i+len('-snes_max_it'):),*) n%snes_max_it
  n%anderson_m   = 8
  n%solver       = 0
  n%alpha = 1.0_C_DOUBLE; n%beta = 1.0_C_DOUBLE
  n%eps_abs_curl = 1.0e-10_C_DOUBLE; n%eps_rel_curl = 5.0e-4_C_DOUBLE

  select case (num_grid%get_asStr('divergence_correction',defaultVal='grid+size'))
    case ('none');      n%divergence_correction = 0
    case ('size');      n%divergence_correction = 1
    case ('grid+size'); n%divergence_correction = 2
    case default;       call IO_error(301_pI16,ext_msg='divergence_correction')
  end select
  select case (num_grid%get_asStr('derivative',defaultVal='continuous'))
    case ('continuous');         n%derivative = 0
    case ('central_difference'); n%derivative = 1
    case ('FWBW_difference');    n%derivative = 2
    case default;                call IO_error(301_pI16,ext_msg='derivative')
  end select

  n%r_cutback_min      = num_mech%get_asReal('r_cutback_min',defaultVal=1.0e-3_pREAL)
  n%r_cutback          = num_mech%get_asReal('r_cutback',defaultVal=0.25_pREAL)
  n%r_increase         = num_mech%get_asReal('r_increase',defaultVal=1.5_pREAL)
  n%eps_rel_state      = num_mech%get_asReal('eps_rel_state',defaultVal=1.0e-6_pREAL)
  n%N_iter_state_max   = num_mech%get_asInt('N_iter_state_max',defaultVal=20)
  n%N_iter_Lp_max      = num_plastic%get_asInt('N_iter_Lp_max',defaultVal=40)
  n%r_linesearch_Lp    = num_plastic%get_asReal('r_linesearch_Lp',defaultVal=0.5_pREAL)
  n%eps_rel_Lp         = num_plastic%get_asReal('eps_rel_Lp',defaultVal=1.0e-6_pREAL)
  n%eps_abs_Lp         = num_plastic%get_asReal('eps_abs_Lp',defaultVal=1.0e-8_pREAL)
  n%f_update_jacobi_Lp = num_plastic%get_asInt('f_update_jacobi_Lp',defaultVal=1)
  n%N_iter_Li_max      = 40
  n%r_linesearch_Li    = 0.5_C_DOUBLE
  n%eps_rel_Li         = n%eps_rel_Lp
  n%eps_abs_Li         = n%eps_abs_Lp
  n%f_update_jacobi_Li = n%f_update_jacobi_Lp

end subroutine read_numerics


!--------------------------------------------------------------------------------------------------
!> @brief tBCmech (values, mask .true. where 'x', myType) as dmk_bc.
!--------------------------------------------------------------------------------------------------
function as_bc(bc) result(c)

  type(tBCmech), intent(in) :: bc
  type(dmk_bc) :: c


  c%values = reshape(real(bc%values,C_DOUBLE),[9])
  c%mask   = reshape(merge(1_C_INT,0_C_INT,bc%mask),[9])
  c%type   = 0
  if (allocated(bc%myType)) then
    select case (bc%myType)
      case ('L');     c%type = 1
      case ('dot_F'); c%type = 2
      case ('F');     c%type = 3
      case ('P');     c%type = 4
      case ('dot_P'); c%type = 5
    end select
  end if

end function as_bc


!--------------------------------------------------------------------------------------------------
!> @brief Status of a C-ABI call: an error of the library (CUDA, cuFFT, configuration) stops the
!> run with the library's message.
!--------------------------------------------------------------------------------------------------
subroutine check(rc, what)

  integer(C_INT),   intent(in) :: rc
  character(len=*), intent(in) :: what

  character(kind=C_CHAR), dimension(:), pointer :: cmsg
  character(len=pSTRLEN) :: msg
  integer :: i


  if (rc == 0) return
  call c_f_pointer(dmk_last_error(), cmsg, [pSTRLEN])
  msg = ''
  do i = 1, pSTRLEN
    if (cmsg(i) == C_NULL_CHAR) exit
    msg(i:i) = cmsg(i)
  end do
  print'(/,1x,a)', 'libdamask_b200: '//what//': '//trim(msg)
  error stop 'spectral_basic_b200: library error'

end subroutine check

end module grid_mechanical_spectral_b200
