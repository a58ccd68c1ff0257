"""The ZZ error indicator and refinement marking (oracle/estimate.py), CPU.

Restates fem3D::calculateMeshErrors (fem3D.cpp:1162-1420) with
OPEM_L2ZZErrorEstimator (:987-1154): flux curl H / mu_r, its L2 projection onto
the edge elements, per-element L1 distances of the real and imaginary parts,
the larger over the driving sets, the floor(NE * fraction) largest marked."""
import numpy as np

from openparem_b200 import meshgen
from oracle import fem
from oracle.estimate import mesh_errors, estimator_rule


def test_rule_integrates_polynomials():
    for p in (1, 2, 3):
        X, W = estimator_rule(p)
        assert abs(W.sum() - 1 / 6) < 1e-15
        # int x^a y^b z^c over the unit tet = a! b! c! / (a+b+c+3)!  (degree <= 2p + 2)
        assert abs(np.sum(W * X[:, 0] * X[:, 1] * X[:, 2] ** 2) - 2 / 5040) < 1e-16


def test_indicator_falls_with_order_and_marks_the_largest():
    maxes = []
    for p in (1, 2, 3):
        prob = meshgen.waveguide_problem(meshgen.WR_A, meshgen.WR_B, 50e-3, 6, 3, 15, p, slab=(20e-3, 30e-3, 4.4, 0.02))
        ops = fem.Operators(prob)
        r = fem.solve_frequency(ops, 10e9, return_fields=True)
        err, marked, mx = mesh_errors(ops, [h for _, h in r["fields"]], 0.05)
        assert len(marked) == int(1620 * 0.05) and mx == err.max() == err[marked[0]]
        assert np.all(np.diff(err[marked]) <= 0) and err[marked[-1]] >= np.sort(err)[-len(marked)]
        maxes.append(mx)
    assert maxes[1] < maxes[0] / 2 and maxes[2] < maxes[1]   # the slab (eps_r 4.4) is coarse for ND1-3
    # a single driving set gives no larger errors than the merge of both
    err1, _, _ = mesh_errors(ops, [r["fields"][0][1]], 0.05)
    assert np.all(err1 <= err + 1e-30)
