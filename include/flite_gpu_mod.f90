! flite_gpu_mod.f90 -- Fortran interface to the C ABI of flite_gpu.h.
!
! A FLITE3D solver host adds this module to SolverSource/ and, in
! mgnsg3d_mg_par.F90, calls these functions in place of the GridSolver module
! calls they replace (readComputationData, setUpInitialField2, doTimeIterations,
! restrictGrid, prolongateGrid, mapFineToCoarse, oneCycle, writeResiduals'
! norms and calculateLiftAndDrag).  The derived types are bind(C), so they have
! the layout of flite_controls and flite_level_desc field for field; the
! logical controls are integer(c_int) 0/1.  Arrays pass as the host's own
! column-major arrays with 1-based node numbers, without copies.
module flite_gpu
  use iso_c_binding
  implicit none

  integer(c_int), parameter :: FLITE_OK = 0, FLITE_EINVAL = 1, FLITE_EUNSUPPORTED = 2, &
                               FLITE_ENAN = 3, FLITE_ETIMEOUT = 4, FLITE_ECUDA = 5, &
                               FLITE_ENOMEM = 6, FLITE_EIO = 7
  integer(c_int), parameter :: FLITE_FP64 = 0, FLITE_MIXED = 1
  integer(c_int), parameter :: FLITE_RECON_NONE = 0, FLITE_RECON_VAN_ALBADA = 1
  integer(c_int), parameter :: FLITE_OBJ_CL = 0, FLITE_OBJ_CD = 1
  integer(c_int), parameter :: FLITE_ADJ_FIXED_POINT = 0, FLITE_ADJ_GMRES = 1

  ! InputVariablesData fields of the hot path, in flite_controls order
  type, bind(C) :: flite_controls
    real(c_double) :: MachNumber, alpha, beta, ReynoldsNumber, PrandtlNumber, gamma
    real(c_double) :: inflowTemperature, wallTemperature
    integer(c_int) :: wallsAreIsentropic
    integer(c_int) :: fluxType
    integer(c_int) :: HLLCFluxOrder
    real(c_double) :: HLLCClipping
    integer(c_int) :: Automaticlipping
    integer(c_int) :: GradientMethod
    integer(c_int) :: dissipationScheme, coarseGridDissipationScheme
    real(c_double) :: secondOrderDissipationFactor, fourthOrderDissipationFactor
    real(c_double) :: coarseGridDissipationFactor
    integer(c_int) :: useMatrixDissipation
    real(c_double) :: HartensCorrectionFactor
    integer(c_int) :: useDissipationWeighting
    integer(c_int) :: viscosityScheme
    integer(c_int) :: boundaryTerm
    real(c_double) :: CFLNumber, turbulentCFLNumber, turbK, maxIncrementFactor, minimumDensity
    integer(c_int) :: multigridScheme, numberOfRelaxationSteps, numberOfGridsToUse
    real(c_double) :: multigridBCRelaxation, prolongationRelaxation, turbProlongationRelaxation
    integer(c_int) :: prolongationMappingScheme
    integer(c_int) :: numberOfMGIterations, maximumnumberofcycles, writeToFileInterval
    real(c_double) :: initialResidual
    integer(c_int) :: numberOfCFLIncrements
    integer(c_int) :: turbulenceModel, numberOfTurbulenceGrids, numberOfTurbulenceSteps
    real(c_double) :: tripFactor, triggerRadius, turbulenceTriggerValue
    integer(c_int) :: numberOfTriggerSteps
    real(c_double) :: maxTurbulenceValue, turbulentPrandtlNumber
    real(c_double) :: referenceArea, datum(3), groundplane
    integer(c_int) :: forceCalcType, restartNumber, numberOfProcesses
    integer(c_int) :: flowType, explicit_, SAS, GUSTMODEL, movingwall, patchInitialization, nspan
    integer(c_int) :: timeScheme, numberOfRSSteps, numberOfPSSteps
    real(c_double) :: residualSmoothingFactor, prolongationSmoothingFactor, physicalTimeStep
    real(c_double) :: engineBCRelaxation
    integer(c_int) :: engineFlowType, numberOfEORelaxationSteps
    real(c_double) :: enginesFrontMassFlow(2)
    real(c_double) :: enginesRearParameters(14)  ! enginesRearParameters(7,2), column-major
    real(c_double) :: inflowField(12)          ! inflowField(1:6,1:2), column-major
    integer(c_int) :: precision                ! extension: FLITE_FP64 | FLITE_MIXED
    integer(c_int) :: reconstruction           ! extension: FLITE_RECON_*
    integer(c_int) :: rungeKuttaStages         ! extension: 3 or 5
  end type flite_controls

  ! one level as readGridComputationData reads it from the .sol
  type, bind(C) :: flite_level_desc
    integer(c_int32_t) :: n_nodes, n_sides, n_bsides, n_bnodes, n_normals
    type(c_ptr) :: side_idx, side_w, side_len, bnd_idx, bnd_w, node_reg, node_ind
    type(c_ptr) :: volume, wall_dist, coords, coord_move, parent, rweight
    ! moving meshes (flowType 2): GCL weights and previous volumes
    type(c_ptr) :: side_gcl, bnd_gcl, volume_prev, volume_prev2
    ! engine inlet sides: engineInletSideIndexes(n,3), engineInletSideCoefficients(n,3)
    integer(c_int32_t) :: n_engine_sides
    type(c_ptr) :: engine_idx, engine_w
  end type flite_level_desc

  interface
    ! readInputVariables defaults (def_par:217-378) and derivation (:387-415)
    integer(c_int) function flite_controls_default(c) bind(C, name="flite_controls_default")
      import :: c_int, flite_controls
      type(flite_controls), intent(inout) :: c
    end function
    integer(c_int) function flite_controls_derive(c) bind(C, name="flite_controls_derive")
      import :: c_int, flite_controls
      type(flite_controls), intent(inout) :: c
    end function

    ! readComputationData (mg_par:1198-1268): copy the levels to the device
    integer(c_int) function flite_create(c, nlevels, levels, ctx) bind(C, name="flite_create")
      import :: c_int, c_ptr, flite_controls, flite_level_desc
      type(flite_controls), intent(in) :: c
      integer(c_int), value :: nlevels
      type(flite_level_desc), intent(in) :: levels(*)
      type(c_ptr), intent(out) :: ctx
    end function
    integer(c_int) function flite_destroy(ctx) bind(C, name="flite_destroy")
      import :: c_int, c_ptr
      type(c_ptr), value :: ctx
    end function
    integer(c_int) function flite_last_error(ctx, buf, len) bind(C, name="flite_last_error")
      import :: c_int, c_ptr, c_char, c_size_t
      type(c_ptr), value :: ctx
      character(kind=c_char), intent(out) :: buf(*)
      integer(c_size_t), value :: len
    end function

    ! state: u(N, nvar) conserved variables
    integer(c_int) function flite_set_state(ctx, level, u) bind(C, name="flite_set_state")
      import :: c_int, c_ptr, c_double
      type(c_ptr), value :: ctx
      integer(c_int), value :: level
      real(c_double), intent(in) :: u(*)
    end function
    integer(c_int) function flite_get_state(ctx, level, u) bind(C, name="flite_get_state")
      import :: c_int, c_ptr, c_double
      type(c_ptr), value :: ctx
      integer(c_int), value :: level
      real(c_double), intent(out) :: u(*)
    end function
    integer(c_int) function flite_get_pressure(ctx, level, p) bind(C, name="flite_get_pressure")
      import :: c_int, c_ptr, c_double
      type(c_ptr), value :: ctx
      integer(c_int), value :: level
      real(c_double), intent(out) :: p(*)
    end function
    ! setUpInitialField2 (def_par:3740-3996)
    integer(c_int) function flite_init_freestream(ctx) bind(C, name="flite_init_freestream")
      import :: c_int, c_ptr
      type(c_ptr), value :: ctx
    end function
    integer(c_int) function flite_start(ctx) bind(C, name="flite_start")
      import :: c_int, c_ptr
      type(c_ptr), value :: ctx
    end function
    integer(c_int) function flite_next_physical_step(ctx) bind(C, name="flite_next_physical_step")
      import :: c_int, c_ptr
      type(c_ptr), value :: ctx
    end function
    ! explicit time stepping: ivd%physicalTimeStep after the last cycle
    integer(c_int) function flite_explicit_time_step(ctx, dt) bind(C, name="flite_explicit_time_step")
      import :: c_int, c_ptr, c_double
      type(c_ptr), value :: ctx
      real(c_double), intent(out) :: dt
    end function

    ! the geometry of the next physical step of a moving mesh (flowType 2),
    ! in place of readComputationData(COMPINFILE, 1) (mg_par:525-545)
    integer(c_int) function flite_update_geometry(ctx, nlevels, levels) bind(C, name="flite_update_geometry")
      import :: c_int, c_ptr, flite_level_desc
      type(c_ptr), value :: ctx
      integer(c_int), value :: nlevels
      type(flite_level_desc), intent(in) :: levels(*)
    end function

    ! doTimeIterations (def_par:966-1000)
    integer(c_int) function flite_do_time_iterations(ctx, level, nsteps, calc_diss, calc_turb, cycle_no) &
        bind(C, name="flite_do_time_iterations")
      import :: c_int, c_ptr
      type(c_ptr), value :: ctx
      integer(c_int), value :: level, nsteps, calc_diss, calc_turb, cycle_no
    end function
    ! restrictGrid (def_par:12141-12430)
    integer(c_int) function flite_restrict(ctx, fine_level, calc_turb) bind(C, name="flite_restrict")
      import :: c_int, c_ptr
      type(c_ptr), value :: ctx
      integer(c_int), value :: fine_level, calc_turb
    end function
    ! prolongateGrid (def_par:12432-12570)
    integer(c_int) function flite_prolong(ctx, coarse_level) bind(C, name="flite_prolong")
      import :: c_int, c_ptr
      type(c_ptr), value :: ctx
      integer(c_int), value :: coarse_level
    end function
    ! mapFineToCoarse of the solution (def_par:12572-12679)
    integer(c_int) function flite_map_fine_to_coarse(ctx, fine_level) bind(C, name="flite_map_fine_to_coarse")
      import :: c_int, c_ptr
      type(c_ptr), value :: ctx
      integer(c_int), value :: fine_level
    end function
    ! oneCycle (mg_par:907-1196)
    integer(c_int) function flite_cycle(ctx, cycle_no) bind(C, name="flite_cycle")
      import :: c_int, c_ptr
      type(c_ptr), value :: ctx
      integer(c_int), value :: cycle_no
    end function
    ! writeResiduals' norms (mg_par:1299-1443); FLITE_ENAN in place of its STOP
    integer(c_int) function flite_residuals(ctx, res, maxres, maxind) bind(C, name="flite_residuals")
      import :: c_int, c_ptr, c_double, c_int32_t
      type(c_ptr), value :: ctx
      real(c_double), intent(out) :: res(7), maxres(7)
      integer(c_int32_t), intent(out) :: maxind(7)
    end function
    ! lift, drag, latF, frictionDrag, latM, longM, longMl, longMd, rollM
    ! (calculateLiftAndDrag def_par:14710-14870; the last three and the
    ! replaced lift, drag, latF, latM with forceCalcType 3, :15129-15313)
    integer(c_int) function flite_forces(ctx, out) bind(C, name="flite_forces")
      import :: c_int, c_ptr, c_double
      type(c_ptr), value :: ctx
      real(c_double), intent(out) :: out(9)
    end function

    ! makeRHS alone (def_par:1525-2590) and its adjoint product
    integer(c_int) function flite_residual_fwd(ctx, level, u, r) bind(C, name="flite_residual_fwd")
      import :: c_int, c_ptr, c_double
      type(c_ptr), value :: ctx
      integer(c_int), value :: level
      real(c_double), intent(in) :: u(*)
      real(c_double), intent(out) :: r(*)
    end function
    integer(c_int) function flite_residual_vjp(ctx, level, u, rbar, ubar) bind(C, name="flite_residual_vjp")
      import :: c_int, c_ptr, c_double
      type(c_ptr), value :: ctx
      integer(c_int), value :: level
      real(c_double), intent(in) :: u(*), rbar(*)
      real(c_double), intent(out) :: ubar(*)
    end function

    ! steady adjoint of CL or CD (no reference counterpart)
    integer(c_int) function flite_set_adjoint_method(ctx, method, restart) bind(C, name="flite_set_adjoint_method")
      import :: c_int, c_ptr
      type(c_ptr), value :: ctx
      integer(c_int), value :: method, restart
    end function
    integer(c_int) function flite_objective(ctx, objective, J) bind(C, name="flite_objective")
      import :: c_int, c_ptr, c_double
      type(c_ptr), value :: ctx
      integer(c_int), value :: objective
      real(c_double), intent(out) :: J
    end function
    integer(c_int) function flite_adjoint_solve(ctx, objective, tol, max_iter, J, side_w_bar, bnd_w_bar, &
                                                volume_bar, iterations, residual) bind(C, name="flite_adjoint_solve")
      import :: c_int, c_ptr, c_double
      type(c_ptr), value :: ctx
      integer(c_int), value :: objective, max_iter
      real(c_double), value :: tol
      real(c_double), intent(out) :: J, side_w_bar(*), bnd_w_bar(*), volume_bar(*), residual
      integer(c_int), intent(out) :: iterations
    end function

    ! several conditions in one launch per cycle (no reference counterpart)
    integer(c_int) function flite_batch_create(ncases, controls, mesh_of_case, nmeshes, nlevels, levels, batch) &
        bind(C, name="flite_batch_create")
      import :: c_int, c_int32_t, c_ptr, flite_controls
      integer(c_int), value :: ncases, nmeshes
      type(flite_controls), intent(in) :: controls(*)
      integer(c_int32_t), intent(in) :: mesh_of_case(*), nlevels(*)
      type(c_ptr), intent(in) :: levels(*)    ! c_loc of each mesh's flite_level_desc array
      type(c_ptr), intent(out) :: batch
    end function
    integer(c_int) function flite_batch_destroy(batch) bind(C, name="flite_batch_destroy")
      import :: c_int, c_ptr
      type(c_ptr), value :: batch
    end function
    integer(c_int) function flite_batch_context(batch, case_index, ctx) bind(C, name="flite_batch_context")
      import :: c_int, c_ptr
      type(c_ptr), value :: batch
      integer(c_int), value :: case_index
      type(c_ptr), intent(out) :: ctx
    end function
    integer(c_int) function flite_batch_run(batch, first_cycle, max_cycles, orders, check_every, cycles, &
                                            log10_reduction) bind(C, name="flite_batch_run")
      import :: c_int, c_int32_t, c_ptr, c_double
      type(c_ptr), value :: batch
      integer(c_int), value :: first_cycle, max_cycles, check_every
      real(c_double), value :: orders
      integer(c_int32_t), intent(out) :: cycles(*)
      real(c_double), intent(out) :: log10_reduction(*)
    end function
    ! case groups of the batch: 1 (default) on, 0 off
    integer(c_int) function flite_batch_set_grouping(batch, on) bind(C, name="flite_batch_set_grouping")
      import :: c_int, c_ptr
      type(c_ptr), value :: batch
      integer(c_int), value :: on
    end function
  end interface
end module flite_gpu
