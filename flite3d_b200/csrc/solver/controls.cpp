// Controls defaults and derived values (readInputVariables,
// SolverSource/mgnsg3d_def_par.F90:201-422).
//
// The same two functions are compiled into the host preprocessor library
// under the fp_ prefix (FLITE_CONTROLS_FP defined), so a host-only program
// can fill the controls without loading the CUDA library.
#include <cmath>
#include <cstring>

#include "flite_gpu.h"

#ifdef FLITE_CONTROLS_FP
#define FLITE_CONTROLS_FN(name) fp_##name
#else
#define FLITE_CONTROLS_FN(name) flite_##name
#endif

extern "C" int FLITE_CONTROLS_FN(controls_default)(flite_controls *c) {
    if (!c) return FLITE_EINVAL;
    std::memset(c, 0, sizeof *c);
    // def_par:217-378, in the order they appear there
    c->numberOfMGIterations = 100;
    c->numberOfCFLIncrements = 0;
    c->writeToFileInterval = 25;
    c->gamma = 1.4;
    c->MachNumber = 0.5;
    c->alpha = 0.0;
    c->beta = 0.0;
    c->CFLNumber = 1.0;
    c->ReynoldsNumber = 1.0E06;
    c->viscosityScheme = 1;
    c->inflowField[0] = 1.0;
    c->inflowField[1] = 1.0;
    c->inflowField[2] = 0.0;
    c->inflowField[3] = 0.0;
    c->inflowField[4] = 1.0;
    c->inflowField[5] = c->inflowField[0] * (c->MachNumber * c->MachNumber) / c->gamma;
    for (int i = 0; i < 6; ++i) c->inflowField[6 + i] = c->inflowField[i];
    c->inflowTemperature = 528.0;
    c->wallsAreIsentropic = 0;
    c->movingwall = 0;
    c->wallTemperature = 528.0;
    c->patchInitialization = 0;
    c->engineFlowType = 1;  // enginesFrontMassFlow, enginesRearParameters = 0
    c->numberOfEORelaxationSteps = 0;
    c->engineBCRelaxation = 1.0;
    c->dissipationScheme = 2;
    c->coarseGridDissipationScheme = 2;
    c->secondOrderDissipationFactor = 0.4;
    c->fourthOrderDissipationFactor = 0.2;
    c->coarseGridDissipationFactor = 0.75;
    c->HartensCorrectionFactor = 0.0;
    c->useMatrixDissipation = 0;
    c->residualSmoothingFactor = 0.0;
    c->multigridScheme = 3;
    c->numberOfRelaxationSteps = 1;
    c->numberOfGridsToUse = 1;
    c->numberOfRSSteps = 0;
    c->numberOfPSSteps = 0;
    c->multigridBCRelaxation = 1.0;
    c->turbulenceModel = 0;
    c->numberOfTurbulenceGrids = 1;
    c->turbulentCFLNumber = 1.0;
    c->tripFactor = 1.0;
    c->triggerRadius = 9999999.9;
    c->turbulenceTriggerValue = 0.0;
    c->referenceArea = 1.0;
    c->forceCalcType = 1;
    c->flowType = 0;
    c->timeScheme = 2;
    c->physicalTimeStep = 0.1;
    c->maximumnumberofcycles = 10000;
    c->restartNumber = 1;
    c->initialResidual = 10000;
    c->fluxType = 1;
    c->HLLCFluxOrder = 2;
    c->HLLCClipping = 1.0;
    c->Automaticlipping = 0;
    c->GradientMethod = 1;
    c->explicit_ = 0;
    c->turbProlongationRelaxation = 1.0;
    c->prolongationSmoothingFactor = 0.0;
    c->prolongationMappingScheme = 1;
    c->prolongationRelaxation = 1.0;
    c->PrandtlNumber = 0.72;
    c->turbulentPrandtlNumber = 0.9;
    c->numberOfTurbulenceSteps = 9999999;
    c->useDissipationWeighting = 0;
    c->maxTurbulenceValue = 3000;
    c->numberOfTriggerSteps = 0;
    c->maxIncrementFactor = 0.25;
    c->minimumDensity = 0.1;
    c->turbK = 0.1;
    c->boundaryTerm = 1;
    c->SAS = 0;
    c->GUSTMODEL = 0;
    c->nspan = 0;
    c->groundplane = -9999999.9;
    c->datum[0] = c->datum[1] = c->datum[2] = 0.0;
    c->numberOfProcesses = 1;
    c->precision = FLITE_FP64;
    c->reconstruction = FLITE_RECON_NONE;
    c->rungeKuttaStages = 3;
    return FLITE_OK;
}

extern "C" int FLITE_CONTROLS_FN(controls_derive)(flite_controls *c) {
    if (!c) return FLITE_EINVAL;
    // def_par:387-415
    if (c->flowType == 0) c->maximumnumberofcycles = 1000000;
    if (c->fluxType == 4) {
        c->secondOrderDissipationFactor = 0.0;
        c->fourthOrderDissipationFactor = 0.0;
    }
    const double PI = 4.0 * std::atan(1.0);
    if (!c->patchInitialization) {
        const double M = c->MachNumber, g = c->gamma;
        c->wallTemperature = (1.0 / ((g - 1.0) * (M * M))) * (c->wallTemperature / c->inflowTemperature);
        double aR = c->alpha * PI / 180., bR = c->beta * PI / 180.;
        c->inflowField[0] = 1.0;
        c->inflowField[1] = std::cos(aR) * std::cos(bR);
        c->inflowField[2] = std::sin(bR);
        c->inflowField[3] = std::sin(aR);
        c->inflowField[4] = (1. / ((g - 1.) * g * (M * M))) + 0.5;
        c->inflowField[5] = 1. / (g * (M * M));
    }
    return FLITE_OK;
}
