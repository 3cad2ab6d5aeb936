"""Batched solves: several meshes x flow conditions in one graph launch.

Every case of a batch must evolve exactly as the same solve run alone (the
kernels are the same and per-thread independent; the block sizes the
autotuner picks do not change any arithmetic).
"""
import numpy as np
import pytest

from flite3d_b200 import Mesh, Solver, default_controls, initial_state
from flite3d_b200.solver import Batch

pytestmark = pytest.mark.gpu


def _cases():
    meshes = [Mesh.bump_channel(12, 4, 4, 0.05, nlevels=3), Mesh.bump_channel(18, 6, 6, 0.05, nlevels=3)]
    conds = [dict(alpha=0.0, MachNumber=0.5), dict(alpha=3.0, MachNumber=0.4)]
    cases = []
    for m in meshes:
        for cd in conds:
            c = default_controls(ReynoldsNumber=0.0, fluxType=1, CFLNumber=2.0, numberOfGridsToUse=3,
                                 multigridScheme=3, **cd)
            cases.append((c, m))
    return meshes, cases


def test_batch_cases_match_single_solves(gpu):
    meshes, cases = _cases()
    batch = Batch(cases)
    singles = [Solver(c, m) for c, m in cases]
    for (c, m), bs, ss in zip(cases, batch.cases, singles):
        u0 = initial_state(c, m, perturb_seed=20261203)
        for s in (bs, ss):
            s.set_state(u0)
            s.start()
    for cyc in range(1, 4):
        batch.cycle(cyc)
        for s in singles:
            s.cycle(cyc)
    for bs, ss in zip(batch.cases, singles):
        for level in range(1, ss.nlevels + 1):
            assert np.array_equal(bs.get_state(level), ss.get_state(level))
        np.testing.assert_allclose(bs.residuals()[0], ss.residuals()[0], rtol=1e-12)


def test_batch_timing_and_autotune(gpu):
    meshes, cases = _cases()
    batch = Batch(cases)
    for (c, m), bs in zip(cases, batch.cases):
        bs.set_state(initial_state(c, m))
        bs.start()
    ms_b, launches = batch.time_cycles(3, sequential=False)
    ms_s, _ = batch.time_cycles(3, sequential=True)
    assert ms_b > 0 and ms_s > 0 and launches > 0
    e, n, best = batch.autotune(reps=2)
    assert e in (64, 128, 256) and n in (64, 128, 256) and best > 0
    lanes, ms = batch.autotune_lanes(reps=1)
    assert len(lanes) == 3 and all(u in (1, 4, 8, 16, 32) for u in lanes) and ms > 0
    batch.cycle(100)
    for bs in batch.cases:
        assert np.isfinite(bs.get_state(1)).all()


def test_batch_run_converges_every_case_like_a_single_solve(gpu):
    meshes, cases = _cases()
    batch = Batch(cases)
    for (c, m), bs in zip(cases, batch.cases):
        bs.set_state(initial_state(c, m, perturb_seed=20261203))
        bs.start()
    cycles, red = batch.run(orders=4.0, max_cycles=400)
    for (c, m), bs, n, r in zip(cases, batch.cases, cycles, red):
        assert r <= -4.0 and 1 <= n < 400
        s = Solver(c, m)
        s.set_state(initial_state(c, m, perturb_seed=20261203))
        s.start()
        r0 = None
        for cyc in range(1, n + 1):
            s.cycle(cyc)
            rr = s.residuals()[0][0]
            r0 = r0 or rr
        # the single solve reaches the target in the same cycle, with the
        # same state
        assert rr <= 1e-4 * r0
        assert np.array_equal(s.get_state(1), bs.get_state(1))


def _run_batch(cases, cycles, grouping, lanes=0, seed=7):
    batch = Batch(cases)
    batch.set_grouping(grouping)
    for (c, m), bs in zip(cases, batch.cases):
        if lanes:
            for level in range(1, bs.nlevels + 1):
                bs.set_gather_lanes(level, lanes)
        bs.set_state(initial_state(c, m, perturb_seed=seed, amplitude=0.02))
        bs.start()
    for cyc in range(1, cycles + 1):
        batch.cycle(cyc)
    return batch


@pytest.mark.parametrize("config", [
    dict(ReynoldsNumber=0.0),
    dict(ReynoldsNumber=0.0, precision=1),
    dict(ReynoldsNumber=800.0, wallsAreIsentropic=1),
    dict(ReynoldsNumber=800.0, wallsAreIsentropic=0, viscosityScheme=2, CFLNumber=1.0),
    dict(ReynoldsNumber=0.0, multigridScheme=1, rungeKuttaStages=5),
    dict(ReynoldsNumber=0.0, multigridScheme=2, numberOfRelaxationSteps=2),
    dict(ReynoldsNumber=0.0, multigridScheme=0),
    dict(ReynoldsNumber=0.0, flowType=1, physicalTimeStep=0.2, timeScheme=2),
])
@pytest.mark.parametrize("lanes", [0, 4])
def test_case_groups_match_separate_case_graphs(gpu, config, lanes):
    # every kernel of the cycle launched once for all cases on a mesh (the
    # case in the grid's y index) gives each case its own solve bit for bit
    meshes = [Mesh.bump_channel(12, 4, 4, 0.05, nlevels=3), Mesh.bump_channel(16, 6, 6, 0.05, nlevels=3)]
    conds = [dict(alpha=0.0, MachNumber=0.5), dict(alpha=2.0, MachNumber=0.45), dict(alpha=-1.0, MachNumber=0.55)]
    cases = [(default_controls(**{**dict(fluxType=1, CFLNumber=2.0, numberOfGridsToUse=3, multigridScheme=3),
                                  **config, **cd}), m) for m in meshes for cd in conds]
    grouped = _run_batch(cases, 3, True, lanes)
    assert grouped.groups() == 2
    apart = _run_batch(cases, 3, False, lanes)
    assert apart.groups() == 0
    for a, b in zip(grouped.cases, apart.cases):
        for level in range(1, a.nlevels + 1):
            assert np.array_equal(a.get_state(level), b.get_state(level)), (config, level)
        assert np.array_equal(a.residuals()[0], b.residuals()[0])
        np.testing.assert_allclose(a.forces(), b.forces(), rtol=0, atol=0)


def test_cases_without_a_group_form_run_alone(gpu):
    # the Spalart-Allmaras path has no group form: its cases keep their own
    # graphs in the batch graph, with the same results
    m = Mesh.bump_channel(12, 4, 4, 0.05, nlevels=2)
    cases = [(default_controls(ReynoldsNumber=1e5, turbulenceModel=1, wallsAreIsentropic=1, fluxType=1,
                               CFLNumber=1.0, numberOfGridsToUse=2, alpha=a), m) for a in (0.0, 2.0)]
    grouped = _run_batch(cases, 2, True)
    assert grouped.groups() == 0
    for (c, mm), bs in zip(cases, grouped.cases):
        s = Solver(c, mm)
        s.set_state(initial_state(c, mm, perturb_seed=7, amplitude=0.02))
        s.start()
        for cyc in (1, 2):
            s.cycle(cyc)
        assert np.array_equal(s.get_state(1), bs.get_state(1))
        s.close()
