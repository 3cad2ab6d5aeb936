"""Controls: reference defaults, derived freestream, NAMELIST deck reader."""
import math

import pytest

from flite3d_b200 import default_controls, controls_from_inp

DECK = """&inputVariables
 ivd%numberOfProcesses = 1,
 ivd%dataDirectory = './',
 ivd%alpha =   1.25,
 ivd%MachNumber = 0.8,          ! a comment
 ivd%ReynoldsNumber = 0.0D0,
 ivd%wallsAreIsentropic = .true.,
 ivd%numberOfMGIterations = -8,
 ivd%CFLNumber = 2.0, ivd%multigridScheme = 3
 ivd%fluxType = 4,
 ivd%datum(2) = 0.5,
 ivd%inflowField(6,2) = 1.5,
 ivd%spanCor = 1
/
"""


def test_defaults_match_reference():
    # def_par:217-378
    c = default_controls()
    assert c.gamma == 1.4 and c.MachNumber == 0.5 and c.CFLNumber == 1.0
    assert c.ReynoldsNumber == 1.0e6 and c.PrandtlNumber == 0.72
    assert c.secondOrderDissipationFactor == 0.4 and c.fourthOrderDissipationFactor == 0.2
    assert c.coarseGridDissipationFactor == 0.75 and c.multigridScheme == 3
    assert c.maxIncrementFactor == 0.25 and c.minimumDensity == 0.1
    assert c.boundaryTerm == 1 and c.fluxType == 1 and c.HLLCFluxOrder == 2
    assert c.inflowTemperature == 528.0 and c.physicalTimeStep == 0.1
    # derived (def_par:387-415)
    assert c.maximumnumberofcycles == 1000000
    g, m = 1.4, 0.5
    assert c.inflowField[4] == pytest.approx(1 / ((g - 1) * g * m * m) + 0.5, rel=1e-15)
    assert c.inflowField[5] == pytest.approx(1 / (g * m * m), rel=1e-15)


def test_namelist_deck():
    c, unknown = controls_from_inp(DECK)
    assert c.MachNumber == 0.8 and c.alpha == 1.25 and c.ReynoldsNumber == 0.0
    assert c.wallsAreIsentropic == 1 and c.numberOfMGIterations == -8
    assert c.CFLNumber == 2.0 and c.fluxType == 4 and c.multigridScheme == 3
    assert c.datum[1] == 0.5
    assert c.inflowField[6 + 5] == 1.5
    # HLLC zeroes the JST factors (def_par:397-401)
    assert c.secondOrderDissipationFactor == 0.0 and c.fourthOrderDissipationFactor == 0.0
    a = math.radians(1.25)
    assert c.inflowField[1] == pytest.approx(math.cos(a), rel=1e-15)
    assert c.inflowField[3] == pytest.approx(math.sin(a), rel=1e-15)
    assert "ivd%dataDirectory" in unknown and "ivd%spanCor" in unknown


def test_extension_controls_default_to_the_reference_scheme():
    # the fields after inflowField have no reference counterpart; their
    # defaults select the reference's scheme
    c = default_controls()
    assert c.precision == 0 and c.reconstruction == 0 and c.rungeKuttaStages == 3
    assert c.useMatrixDissipation == 0 and c.dissipationScheme == 2 and c.HartensCorrectionFactor == 0.0


def test_deck_leaves_the_extension_controls_alone():
    # a reference deck cannot name them: they keep their defaults
    c, unknown = controls_from_inp(DECK)
    assert c.reconstruction == 0 and c.rungeKuttaStages == 3 and c.precision == 0


ENGINE_DECK = """&inputVariables
 ivd%engineFlowType = 2,
 ivd%enginesFrontMassFlow(1) = 0.3,
 ivd%enginesFrontMassFlow(2) = 0.25,
 ivd%enginesRearParameters(1,1) = 0.5, ivd%enginesRearParameters(2,1) = 0.9,
 ivd%enginesRearParameters(6,1) = 0.35, ivd%enginesRearParameters(7,2) = 0.1,
 ivd%engineBCRelaxation = 0.8,
 ivd%numberOfEORelaxationSteps = 20
/
"""


def test_engine_controls():
    # defaults (def_par:256-260) and the deck's array elements, stored
    # column-major as enginesRearParameters(7,2)
    c = default_controls()
    assert c.engineFlowType == 1 and c.numberOfEORelaxationSteps == 0 and c.engineBCRelaxation == 1.0
    assert list(c.enginesFrontMassFlow) == [0.0, 0.0] and not any(c.enginesRearParameters)
    c, unknown = controls_from_inp(ENGINE_DECK)
    assert not unknown
    assert c.engineFlowType == 2 and c.numberOfEORelaxationSteps == 20 and c.engineBCRelaxation == 0.8
    assert list(c.enginesFrontMassFlow) == [0.3, 0.25]
    r = list(c.enginesRearParameters)
    assert r[0] == 0.5 and r[1] == 0.9 and r[5] == 0.35 and r[7 + 6] == 0.1
