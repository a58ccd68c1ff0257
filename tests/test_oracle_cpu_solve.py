"""The oracle's iterative FP64 CPU solve (oracle/cpu_solve.py: GMRES-DR with
vertex-patch block Jacobi, OpenMP kernels) against the oracle's direct solve
(SuperLU, the reference's factorisation path) on the same small slab-loaded
guide: |dS| <= 1e-8 at rtol 1e-10, and the patches cover every DOF."""
import numpy as np

from openparem_b200 import meshgen
from oracle import fem, cpu_solve


def test_cpu_iterative_solve_matches_direct_solve():
    prob = meshgen.waveguide_problem(meshgen.WR_A, meshgen.WR_B, 50e-3, 4, 2, 10, 2, slab=(20e-3, 30e-3, 4.4, 0.02))
    ops = fem.Operators(prob)
    cs = cpu_solve.CpuSolver(ops)
    assert set(np.unique(cs.pdofs)) == set(range(ops.topo.n))
    for f in (8.5e9, 11.5e9):
        r = cs.solve_frequency(f)
        ref = fem.solve_frequency(ops, f)["S"]
        assert np.abs(r["S"] - ref).max() <= 1e-8, f
        assert all(0 < it < 10000 for it in r["iterations"])
