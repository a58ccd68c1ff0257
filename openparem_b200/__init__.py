"""B200-native per-frequency FEM solve stage of OpenParEM3D.

Public API:
  Fem3D(problem_dict).assemble().solve(freq)  -> S-parameters (see fem3d.py)
  meshgen                                      -> structured waveguide problems
The compute path is libopem_b200.so (CUDA, sm_100a) behind include/opem_b200.h.
"""
from .fem3d import Fem3D, Context, OpemError, default_opts  # noqa: F401
from . import meshgen  # noqa: F401
