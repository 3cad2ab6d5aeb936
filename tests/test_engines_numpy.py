"""An independent numpy restatement of the engine conditions of
setBCsOnSolutionField (def_par:4488-4918), checked against the CPU
restatement.  On a box whose faces are far field except the engine faces,
the start-up conditions (makePressureField, then setBCsOnSolutionField on
level 1 with cycleNumber 1, def_par:3990-3994) are the engine conditions
alone: the exhausts take the ramped exhaust state, the inlets' momenta are
scaled to the target mass flow (engineFlowType 1) or mass flow function (2)
with the internal energy kept, and engineFlowType 2 recomputes the pressure.
The state streams out through the inlets, so the no-inflow correction (which
reads the node normals) leaves it alone.
"""
import numpy as np
import pytest

from conftest import oracle_backend
from flite3d_b200 import Solver, host_controls, initial_state
from hybrid_meshes import box
from test_engines import rear_state

GAMMA = 1.4
LANES = 256  # the fixed order of the inlet sums (side s to partial s mod 256, then a pairwise tree)


def tree_sum(terms, sides):
    part = np.zeros(LANES)
    for k, s in enumerate(sides):
        part[s % LANES] += terms[k]
    w = LANES // 2
    while w >= 1:
        part[:w] = part[:w] + part[w:2 * w]
        w //= 2
    return part[0]


def pressure(u):
    ke = (u[1] * u[1] + u[2] * u[2]) + u[3] * u[3]
    return np.maximum((GAMMA - 1.0) * (u[4] - 0.5 * ke / u[0]), 0.1)


def engine_conditions(c, mesh, u, steps_done=0):
    """setBCsOnSolutionField's engine part on level 1 at cycleNumber 1."""
    u = u.copy()
    reg, ind = mesh.array(1, "node_reg"), mesh.array(1, "node_ind")
    nodes = lambda r: ind[reg[r + 20] - 1:reg[r + 21]] - 1  # noqa: E731
    p = pressure(u)
    inflow = np.array(c.inflowField[:6])
    rear = np.array(c.enginesRearParameters).reshape(2, 7)
    rp = min(0.0 / c.numberOfEORelaxationSteps, 1.0) if c.numberOfEORelaxationSteps > 0 else 1.0
    for e, r in ((0, -8), (1, -6)):
        nd = nodes(r)
        u[:, nd] = ((1.0 - rp) * inflow[:5] + rp * rear[e, :5])[:, None]
        p[nd] = (1.0 - rp) * inflow[5] + rp * rear[e, 5]
    idx, w = mesh.array(1, "engine_idx"), mesh.array(1, "engine_w")
    a, b, inlet = idx[0] - 1, idx[1] - 1, idx[2] - 1
    dot = lambda n: (u[1, n] * w[0] + u[2, n] * w[1]) + u[3, n] * w[2]  # noqa: E731
    flow_terms = dot(a) + dot(b)
    fac = [1.0, 1.0]
    scale = True
    for e in range(2):
        sel = np.nonzero(inlet == e)[0]
        flow = tree_sum(flow_terms[sel], sel)
        if c.engineFlowType == 1:
            if flow > 0.0:
                fac[e] = c.enginesFrontMassFlow[e] / flow
            continue
        ke = lambda n: (u[1, n] * u[1, n] + u[2, n] * u[2, n]) + u[3, n] * u[3, n]  # noqa: E731
        press = 0.5 * ((p[a] + 0.5 * ke(a) / u[0, a]) + (p[b] + 0.5 * ke(b) / u[0, b]))
        t1 = (GAMMA / u[0, a]) * (u[4, a] - (0.5 * ke(a)) / u[0, a])
        t2 = (GAMMA / u[0, b]) * (u[4, b] - (0.5 * ke(b)) / u[0, b])
        wn = np.sqrt((w[0] * w[0] + w[1] * w[1]) + w[2] * w[2])
        pt = tree_sum(((np.sqrt(0.5 * (t1 + t2)) / press) * 2.0 * wn)[sel], sel)
        area = tree_sum((2.0 * wn)[sel], sel)
        if scale and flow > 0.0:
            fac[e] = c.enginesFrontMassFlow[e] / (flow * (pt / area))
            if fac[e] > 99999999999.:
                scale = False
    if scale:
        g = u.copy()
        for e, r in ((0, -12), (1, -10)):
            nd = nodes(r)
            keg = (g[1, nd] * g[1, nd] + g[2, nd] * g[2, nd]) + g[3, nd] * g[3, nd]
            intE = g[4, nd] - 0.5 * keg / g[0, nd]
            u[1:4, nd] = u[1:4, nd] * fac[e]
            ke = (u[1, nd] * u[1, nd] + u[2, nd] * u[2, nd]) + u[3, nd] * u[3, nd]
            u[4, nd] = intE + 0.5 * ke / u[0, nd]
        if c.engineFlowType == 2:
            p = pressure(u)
    return u, p, fac


@pytest.mark.parametrize("ftype, front", [(1, [0.06, 0.05]), (2, [0.09, 0.07])])
@pytest.mark.parametrize("ramp", [0, 5])
def test_engine_conditions_match_numpy(ftype, front, ramp):
    m = box(8, 4, 4, kind="tet", nlevels=1, engines=2, far_only=True)
    c = host_controls(ReynoldsNumber=0.0, fluxType=1, numberOfGridsToUse=1, engineFlowType=ftype,
                      enginesFrontMassFlow=front, enginesRearParameters=rear_state(),
                      numberOfEORelaxationSteps=ramp)
    o = Solver(c, m, backend=oracle_backend())
    try:
        reg = m.array(1, "node_reg")
        # only far-field and engine nodes: wall, symmetry and inviscid-wall ranges are empty
        for r in (-20, -18, -4):
            assert reg[r + 21] < reg[r + 20]
        u0 = np.ascontiguousarray(initial_state(c, m, perturb_seed=13, amplitude=0.02))
        o.set_state(u0)
        o.start()
        want_u, want_p, fac = engine_conditions(c, m, u0)
        assert all(f != 1.0 for f in fac)  # both inlets were scaled
        got_u, got_p = o.get_state(1), o.get_pressure(1)
        assert np.array_equal(got_u, want_u)
        assert np.array_equal(got_p, want_p)
    finally:
        o.close()
        m.close()
