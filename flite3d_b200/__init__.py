"""B200 (sm_100a) flow-solver hot path of FLITE3D behind a C ABI.

Native libraries (built in-tree by :mod:`flite3d_b200.build`):
  * libflite_gpu.so    -- CUDA solver, C ABI of include/flite_gpu.h
  * libflite_prepro.so -- meshes, gen3d restatement and file formats
"""
from .mesh import Mesh, read_rst, write_rst, write_res, write_unk, read_unk  # noqa: F401
from .solver import (Solver, default_controls, host_controls, controls_from_inp, initial_state,  # noqa: F401
                     run_steady, run_unsteady)

__all__ = ["Mesh", "Solver", "default_controls", "host_controls", "controls_from_inp", "initial_state",
           "run_steady", "run_unsteady", "read_rst", "write_rst", "write_res", "write_unk", "read_unk"]
