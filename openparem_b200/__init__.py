"""B200-native per-frequency FEM solve stage of OpenParEM3D.

Public API:
  Fem3D(problem_dict).assemble().solve(freq)  -> S-parameters (see fem3d.py)
  Server(device, slots).submit(fem, freqs)     -> serving loop (admission by HBM footprint)
  meshgen                                      -> structured waveguide problems
The compute path is libopem_b200.so (CUDA, sm_100a) behind include/opem_b200.h.
"""
from .fem3d import Fem3D, Context, OpemError, Server, default_opts  # noqa: F401
from . import meshgen  # noqa: F401
