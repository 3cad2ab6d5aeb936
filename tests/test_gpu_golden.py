"""The GPU path against the committed regression fixtures of the CPU
restatement (tests/golden/*.npz): the same 15 growing-V cycles from the same
seeded state give the fixture's level-1 state bit for bit, and its residual
history and forces to the reduction tolerance (the GPU sums norms and forces
in another order)."""
import glob
import os

import numpy as np
import pytest

from conftest import ROOT
from flite3d_b200 import Mesh, Solver, default_controls, initial_state

pytestmark = pytest.mark.gpu

INTS = ("fluxType", "HLLCFluxOrder", "Automaticlipping", "multigridScheme", "numberOfGridsToUse",
        "wallsAreIsentropic", "turbulenceModel", "useMatrixDissipation", "dissipationScheme",
        "reconstruction", "rungeKuttaStages")
FIXTURES = sorted(os.path.splitext(os.path.basename(p))[0]
                  for p in glob.glob(os.path.join(ROOT, "tests", "golden", "*.npz")))


@pytest.mark.parametrize("name", FIXTURES)
def test_gpu_reproduces_the_fixture(name):
    g = np.load(os.path.join(ROOT, "tests", "golden", f"{name}.npz"), allow_pickle=False)
    mesh = Mesh.bump_channel(*[int(v) for v in g["mesh"]], 0.05, nlevels=3)
    ctl = dict(zip([str(k) for k in g["ctl_keys"]], [float(v) for v in g["ctl_vals"]]))
    ctl = {k: (int(v) if k in INTS else v) for k, v in ctl.items()}
    c = default_controls(**ctl)
    s = Solver(c, mesh)
    s.set_state(initial_state(c, mesh, perturb_seed=20261203))
    s.start()
    hist = []
    for cyc in range(1, len(g["res1"]) + 1):
        s.cycle(cyc)
        hist.append(s.residuals()[0][0])
    assert np.array_equal(s.get_state(1), g["u"])
    np.testing.assert_allclose(hist, g["res1"], rtol=1e-12)
    np.testing.assert_allclose(s.forces()[:6], g["forces"][:6], rtol=1e-12, atol=1e-15)
