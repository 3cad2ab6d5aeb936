"""A parallel run's multi-domain .sol files ingested into one mesh and solved
on the GPU: bit for bit against the CPU restatement on the ingested mesh, and
bit for bit against the canonical form of the mesh the files were written
from (the two are the same mesh).
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
