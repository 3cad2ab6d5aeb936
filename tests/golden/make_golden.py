"""Regression fixtures for the CPU restatement (run from the repo root).

    python tests/golden/make_golden.py

Each fixture holds the mesh size, the controls, the residual history
(res1 of writeResiduals) of 15 growing-V cycles from the seeded initial
state, the final forces and the final level-1 state.  They pin the
restatement against unintended changes; they are not reference outputs
(the reference has none and cannot be run here).
"""
import ctypes
import os
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)

from flite3d_b200 import Mesh, Solver, default_controls, initial_state  # noqa: E402
from flite3d_b200.solver import Backend  # noqa: E402

CASES = {
    "central_jst": dict(ReynoldsNumber=0.0, fluxType=1, CFLNumber=2.0, numberOfGridsToUse=3,
                        multigridScheme=3),
    "hllc2": dict(ReynoldsNumber=0.0, fluxType=4, HLLCFluxOrder=2, Automaticlipping=1,
                  CFLNumber=2.0, numberOfGridsToUse=3, multigridScheme=3),
    "laminar": dict(ReynoldsNumber=5000.0, fluxType=1, CFLNumber=2.0, numberOfGridsToUse=3,
                    multigridScheme=3, wallsAreIsentropic=1),
    "sa": dict(ReynoldsNumber=1.0e5, fluxType=1, CFLNumber=1.0, numberOfGridsToUse=3,
               multigridScheme=3, wallsAreIsentropic=1, turbulenceModel=1),
    "matrix_dissipation": dict(ReynoldsNumber=0.0, fluxType=1, CFLNumber=2.0, numberOfGridsToUse=3,
                               multigridScheme=3, useMatrixDissipation=1),
    "lp_dissipation": dict(ReynoldsNumber=0.0, fluxType=1, CFLNumber=2.0, numberOfGridsToUse=3,
                           multigridScheme=3, dissipationScheme=1, fourthOrderDissipationFactor=0.05),
    # the upwind extension (no reference counterpart)
    "upwind_extension": dict(ReynoldsNumber=0.0, fluxType=3, reconstruction=1, rungeKuttaStages=5,
                             secondOrderDissipationFactor=0.0, fourthOrderDissipationFactor=0.0,
                             CFLNumber=2.0, numberOfGridsToUse=3, multigridScheme=3),
}
MESH = (12, 4, 4)


def main():
    import flite3d_b200.build as b
    b.build_prepro()
    b.build_oracle()
    lib = ctypes.CDLL(os.path.join(ROOT, "oracle", "_build", "liboracle.so"))
    mesh = Mesh.bump_channel(*MESH, 0.05, nlevels=3)
    only = sys.argv[1:] or list(CASES)
    for name, ctl in CASES.items():
        if name not in only:
            continue
        c = default_controls(**ctl)
        o = Solver(c, mesh, backend=Backend(lib, "oracle_"))
        o.set_state(initial_state(c, mesh, perturb_seed=20261203))
        o.start()
        res = []
        for cyc in range(1, 16):
            o.cycle(cyc)
            res.append(o.residuals()[0][0])
        np.savez(os.path.join(ROOT, "tests", "golden", f"{name}.npz"), mesh=np.array(MESH),
                 ctl_keys=np.array(list(ctl.keys())), ctl_vals=np.array([float(v) for v in ctl.values()]),
                 res1=np.array(res), forces=o.forces(), u=o.get_state(1))
        print(name, res[-1])


if __name__ == "__main__":
    main()
