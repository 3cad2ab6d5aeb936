"""Meshes from other sources on the GPU: a parallel run's multi-domain .sol
files ingested into one mesh, bit for bit against the CPU restatement on the
ingested mesh and against the canonical form of the mesh the files were
written from (the two are the same mesh); meshes of hexahedra, prisms and
pyramids, bit for bit against the CPU restatement.
"""
import numpy as np
import pytest

from conftest import oracle_backend
from flite3d_b200 import Mesh, Solver, default_controls, initial_state

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("nd", [2, 4])
def test_ingested_domains_solve_like_the_canonical_mesh(tmp_path, nd):
    mesh = Mesh.bump_channel(24, 8, 8, 0.05, nlevels=3)
    mesh.write_sol_domains(tmp_path / "bump", tmp_path / "plotreg.reg", nd)
    merged = Mesh.read_sol_domains(tmp_path / "bump", tmp_path / "plotreg.reg")
    canon = mesh.canonical()
    c = default_controls(ReynoldsNumber=5000.0, wallsAreIsentropic=1, fluxType=1, CFLNumber=2.0,
                         numberOfGridsToUse=3)
    u0 = initial_state(c, merged, perturb_seed=5, amplitude=0.02)
    runs = [Solver(c, merged), Solver(c, merged, backend=oracle_backend()), Solver(c, canon)]
    for s in runs:
        s.set_state(u0)
        s.start()
        for cyc in range(1, 4):
            s.cycle(cyc)
    for level in range(1, 4):
        a = runs[0].get_state(level)
        assert np.array_equal(a, runs[1].get_state(level)), level
        assert np.array_equal(a, runs[2].get_state(level)), level
    for s in runs:
        s.close()
    for m in (merged, canon, mesh):
        m.close()


@pytest.mark.parametrize("kind", ["hex", "prism", "pyramid", "mixed"])
def test_hybrid_element_meshes_match(kind):
    # meshes of gen3d's other element types run the same device path
    from hybrid_meshes import box
    mesh = box(8, 4, 4, kind=kind, nlevels=2)
    c = default_controls(ReynoldsNumber=2000.0, wallsAreIsentropic=1, fluxType=1, CFLNumber=2.0,
                         numberOfGridsToUse=2)
    u0 = initial_state(c, mesh, perturb_seed=9, amplitude=0.02)
    g, o = Solver(c, mesh), Solver(c, mesh, backend=oracle_backend())
    for s in (g, o):
        s.set_state(u0)
        s.start()
        for cyc in range(1, 4):
            s.cycle(cyc)
    for level in (1, 2):
        assert np.array_equal(g.get_state(level), o.get_state(level)), (kind, level)
    g.close()
    o.close()
    mesh.close()
