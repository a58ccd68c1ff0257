"""CPU tests of the oracle's building blocks (basis, quadrature, topology counts)."""
import numpy as np
import pytest

from oracle.nd_basis import NDBasis, ndofs
from oracle.quadrature import tet_rule, tri_rule, line_rule
from oracle import fem
from openparem_b200 import meshgen


@pytest.mark.parametrize("p", [1, 2, 3, 4])
def test_dual_basis(p):
    B = NDBasis(p)
    W = B._functionals()
    D = W @ B.coef.reshape(B.ld, -1).T
    assert np.abs(D - np.eye(B.ld)).max() < 1e-11
    assert B.ld == ndofs(p)["local"] == p * (p + 2) * (p + 3) // 2


def test_whitney_order1():
    B = NDBasis(1)
    x = np.array([[0.2, 0.3, 0.1]])
    lam = np.array([0.4, 0.2, 0.3, 0.1])
    grad = np.array([[-1, -1, -1], [1, 0, 0], [0, 1, 0], [0, 0, 1.0]])
    ref = [lam[a] * grad[b] - lam[b] * grad[a] for a, b in [(0, 1), (0, 2), (0, 3), (1, 2), (1, 3), (2, 3)]]
    assert np.allclose(B.eval(x)[:, 0, :], ref, atol=1e-14)


@pytest.mark.parametrize("deg", [2, 5, 8])
def test_quadrature_exact(deg):
    from math import factorial
    X, w = tet_rule(deg)
    for a, b, c in [(deg, 0, 0), (1, deg - 1, 0), (0, 1, deg - 1)]:
        exact = factorial(a) * factorial(b) * factorial(c) / factorial(a + b + c + 3)
        assert abs(np.sum(w * X[:, 0] ** a * X[:, 1] ** b * X[:, 2] ** c) - exact) < 1e-15
    S, wt = tri_rule(deg)
    exact = factorial(deg) / factorial(deg + 2)
    assert abs(np.sum(wt * S[:, 0] ** deg) - exact) < 1e-15
    s, ws = line_rule(deg)
    assert abs(np.sum(ws * s ** deg) - 1.0 / (deg + 1)) < 1e-15


def test_config_counts():
    """DOF and nnz counts of the benchmark meshes (ND_p DOF counts incl. eliminated DOFs)."""
    prob, _ = meshgen.config1()
    assert len(prob["tets"]) == 1620
    ops = fem.Operators(prob)
    assert ops.topo.n == 2373 and ops.K.nnz == 33369
    p2 = meshgen.waveguide_problem(meshgen.WR_A, meshgen.WR_B, 50e-3, 6, 3, 15, 2)
    t2 = fem.Topology(p2)
    assert t2.n == 11838
    big = meshgen.waveguide_problem(meshgen.WR_A, meshgen.WR_B, 50e-3, 24, 12, 60, 1)
    tb = fem.Topology(big)
    assert len(big["tets"]) == 103680 and tb.nE == 128400 and tb.nF == 212256


def test_curl_of_gradient_vanishes():
    """K G = 0 for the discrete gradient of vertex hats (exact sequence property)."""
    prob = meshgen.small_case(order=2)
    ops = fem.Operators(prob)
    B = fem.basis(2)[0]
    # the gradient of a linear function is constant: its ND interpolant lies in
    # the kernel of curl-curl
    c = np.array([0.3, -0.7, 0.2])
    verts = np.asarray(prob["verts"])
    topo = ops.topo
    x = np.zeros(topo.n)
    # interpolate grad(c.x) = c through edge functionals (k=0 moment = c.t, others 0)
    # and face functionals (q_0 moments); assemble via element-local evaluation
    Wl = B._functionals()
    for e in range(len(topo.tets)):
        P = verts[topo.tets[e]]
        J = np.stack([P[1] - P[0], P[2] - P[0], P[3] - P[0]], axis=1)
        chat = J.T @ c                      # reference-frame constant field
        coef = np.zeros((3, B.nmon)); coef[:, 0] = chat
        x[topo.dof[e]] = Wl @ coef.ravel()
    assert np.abs(ops.K @ x).max() < 1e-10 * np.abs(ops.K).max() * np.abs(x).max()
