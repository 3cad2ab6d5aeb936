"""Moving meshes (flowType 2, ALE): the GPU library against the CPU
restatement, bit for bit on every level after each physical time step.  Each
step's geometry (coefficients, GCL weights, current and previous volumes,
coordinate movement) comes from fp_set_moving_geometry and is handed to both
through flite_update_geometry; the boundary nodes move with a rigid shift,
the interior ones also deform.  Fluxes 1-4 (HLLC of both orders), both
boundary terms, both time schemes, laminar walls moving with the mesh, the
Spalart-Allmaras model, a thread and a warp per node.
"""
import ctypes

import numpy as np
import pytest

from conftest import oracle_backend
from flite3d_b200 import Mesh, Solver, default_controls, initial_state

pytestmark = pytest.mark.gpu


def deform(x0, nb, t):
    d = np.zeros_like(x0)
    s = np.sin(np.pi * x0[0] / x0[0].max())
    d[0] = 0.04 * np.sin(2 * np.pi * x0[1]) * s * np.sin(2 * np.pi * t)
    d[1] = 0.03 * np.sin(np.pi * x0[1]) * s * np.sin(2 * np.pi * t)
    d[2] = 0.02 * np.sin(np.pi * x0[2] / x0[2].max()) * s * np.cos(2 * np.pi * t)
    d[:, :nb] = 0.0
    d[1] += 0.05 * t
    d[2] -= 0.03 * t * t
    return x0 + d


CASES = {
    "central": dict(),
    "central_bdf1": dict(timeScheme=1),
    "fv_boundary": dict(boundaryTerm=2),
    "llf": dict(fluxType=2, CFLNumber=0.5),
    "roe": dict(fluxType=3, CFLNumber=1.0),
    "hllc1": dict(fluxType=4, HLLCFluxOrder=1, CFLNumber=1.0),
    "hllc2": dict(fluxType=4, HLLCFluxOrder=2, Automaticlipping=1, CFLNumber=1.0),
    "laminar": dict(ReynoldsNumber=500.0, CFLNumber=1.0, wallsAreIsentropic=1),
    "laminar_isothermal": dict(ReynoldsNumber=500.0, CFLNumber=1.0, wallsAreIsentropic=0),
    "sa": dict(ReynoldsNumber=1.0e5, CFLNumber=1.0, turbulenceModel=1, wallsAreIsentropic=1),
}


@pytest.mark.parametrize("lanes", [0, 1])
@pytest.mark.parametrize("name", list(CASES))
def test_moving_mesh_steps_match(name, lanes):
    mesh = Mesh.bump_channel(24, 8, 8, 0.05, nlevels=3)
    x0 = mesh.array(1, "coords")
    nb = mesh.level(1).n_bnodes
    dt = 0.1
    x = lambda k: deform(x0, nb, k * dt)
    base = dict(ReynoldsNumber=0.0, fluxType=1, CFLNumber=2.0, numberOfGridsToUse=3, flowType=2,
                physicalTimeStep=dt, timeScheme=2)
    c = default_controls(**{**base, **CASES[name]})
    ts = c.timeScheme
    mesh.set_moving(x(0), x(0), x(0), ts)
    g, o = Solver(c, mesh), Solver(c, mesh, backend=oracle_backend())
    if lanes:
        for level in (1, 2, 3):
            g.set_gather_lanes(level, lanes)
    u0 = initial_state(c, mesh, perturb_seed=7, amplitude=0.03)
    for s in (g, o):
        s.set_state(u0)
        s.start()
    for step in range(1, 4):
        if step > 1:
            for s in (g, o):
                s.next_physical_step()
        mesh.set_moving(x(step), x(step - 1), x(max(step - 2, 0)), ts)
        for s in (g, o):
            s.update_geometry(mesh)
        for it in range(1, 4):
            g.cycle(it)
            o.cycle(it)
        for level in range(1, 4):
            a, b = g.get_state(level), o.get_state(level)
            assert np.all(np.isfinite(b)), (name, step, level)
            assert np.array_equal(a, b), (name, step, level, np.abs(a - b).max())
        assert np.allclose(g.residuals()[0], o.residuals()[0], rtol=1e-12, atol=0)
        assert np.allclose(g.forces(), o.forces(), rtol=1e-12, atol=1e-300)
    g.close()
    o.close()
    mesh.close()


@pytest.mark.parametrize("name", ["central", "fv_boundary", "roe", "hllc1"])
def test_moving_mesh_residual_matches(name):
    mesh = Mesh.bump_channel(24, 8, 8, 0.05, nlevels=1)
    x0 = mesh.array(1, "coords")
    nb = mesh.level(1).n_bnodes
    mesh.set_moving(deform(x0, nb, 0.3), deform(x0, nb, 0.2), deform(x0, nb, 0.1), 2)
    c = default_controls(**{**dict(ReynoldsNumber=0.0, fluxType=1, numberOfGridsToUse=1, flowType=2,
                                   physicalTimeStep=0.1), **CASES[name]})
    g, o = Solver(c, mesh), Solver(c, mesh, backend=oracle_backend())
    u = np.ascontiguousarray(initial_state(c, mesh, perturb_seed=3, amplitude=0.05))
    for s in (g, o):
        s.set_state(u)
        s.start()
    assert np.array_equal(g.residual_fwd(u), o.residual_fwd(u))
    g.close()
    o.close()
    mesh.close()


def test_moving_mesh_refusals():
    mesh = Mesh.bump_channel(12, 4, 4, 0.05, nlevels=2)
    c = default_controls(ReynoldsNumber=0.0, fluxType=1, flowType=2, physicalTimeStep=0.1, numberOfGridsToUse=2)
    # a moving run needs the GCL weights and previous volumes
    with pytest.raises(RuntimeError):
        Solver(c, mesh)
    x0 = mesh.array(1, "coords")
    mesh.set_moving(x0, x0, x0, 2)
    s = Solver(c, mesh)
    s.set_state(initial_state(c, mesh))
    s.start()
    # the adjoint products are of the static residual
    u = np.ascontiguousarray(s.get_state(1))
    r = np.zeros_like(u)
    assert s.be.residual_vjp(s._h, 1, u.ctypes.data_as(ctypes.c_void_p), r.ctypes.data_as(ctypes.c_void_p),
                             r.ctypes.data_as(ctypes.c_void_p)) == 2
    s.close()
    # a static run takes no geometry update
    st = Solver(default_controls(ReynoldsNumber=0.0, fluxType=1, flowType=1, physicalTimeStep=0.1,
                                 numberOfGridsToUse=2), mesh)
    with pytest.raises(RuntimeError):
        st.update_geometry(mesh)
    st.close()
    mesh.close()
