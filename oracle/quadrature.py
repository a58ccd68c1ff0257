"""Quadrature rules on the reference line, triangle and tetrahedron (oracle).

Collapsed (Duffy) tensor Gauss-Jacobi rules, exact for polynomials of the
requested total degree.  MFEM's IntRules (used by the reference's integrators,
src/OpenParEM3D/fem3D.cpp:115-123) integrate the same polynomial integrands
exactly on affine tetrahedra, so exact rules reproduce its element matrices
up to rounding.
"""
import numpy as np
from scipy.special import roots_jacobi, roots_legendre


def _npts(degree):
    return degree // 2 + 2


def line_rule(degree):
    """Points s in [0,1] and weights (sum 1)."""
    x, w = roots_legendre(_npts(degree))
    return 0.5 * (x + 1.0), 0.5 * w


def tri_rule(degree):
    """Points (s1,s2) on the unit triangle {s1,s2>=0, s1+s2<=1}; weights sum 1/2."""
    n = _npts(degree)
    xu, wu = roots_jacobi(n, 1.0, 0.0)
    xv, wv = roots_legendre(n)
    u = 0.5 * (xu + 1.0)
    v = 0.5 * (xv + 1.0)
    wu = wu * 0.25
    wv = wv * 0.5
    U, V = np.meshgrid(u, v, indexing="ij")
    W = np.outer(wu, wv)
    s1 = U
    s2 = (1.0 - U) * V
    return np.stack([s1.ravel(), s2.ravel()], axis=1), W.ravel()


def tet_rule(degree):
    """Points on the unit tetrahedron (0,0,0),(1,0,0),(0,1,0),(0,0,1); weights sum 1/6."""
    n = _npts(degree)
    xu, wu = roots_jacobi(n, 2.0, 0.0)
    xv, wv = roots_jacobi(n, 1.0, 0.0)
    xw, ww = roots_legendre(n)
    u = 0.5 * (xu + 1.0); wu = wu * 0.125
    v = 0.5 * (xv + 1.0); wv = wv * 0.25
    w = 0.5 * (xw + 1.0); ww = ww * 0.5
    U, V, Wc = np.meshgrid(u, v, w, indexing="ij")
    WT = wu[:, None, None] * wv[None, :, None] * ww[None, None, :]
    x = U
    y = (1.0 - U) * V
    z = (1.0 - U) * (1.0 - V) * Wc
    return np.stack([x.ravel(), y.ravel(), z.ravel()], axis=1), WT.ravel()


def l2_nodal_rule(p):
    """The rule the reference's port integrals amount to: a product of fields is
    interpolated at the nodes of MFEM 4.8's order-p L2 triangle (L2_FECollection
    with its default Gauss-Legendre basis; used by tangentialInnerProduct,
    src/OpenParEM3D/port.cpp:3463-3490 with the space of :5045, and at order
    p - 1 by Fields::calculatePz, src/OpenParEM2D/fem2D.cpp:395-480) and the
    interpolant is integrated exactly.  MFEM places the nodes of that element
    at (o_i, o_j) / (o_i + o_j + o_{p-i-j}) for i + j <= p, o the p + 1
    Gauss-Legendre points on [0, 1]; the weights are the integrals of the
    Lagrange polynomials of degree p on those nodes.  The node set is symmetric
    in the three vertices, so the rule does not depend on the vertex order.
    Returns points (s1, s2) on the unit triangle and weights summing to 1/2."""
    from math import factorial
    x, _ = roots_legendre(p + 1)
    o = np.sort(0.5 * (x + 1.0))
    pts = np.array([(o[i] / (o[i] + o[j] + o[p - i - j]), o[j] / (o[i] + o[j] + o[p - i - j]))
                    for j in range(p + 1) for i in range(p + 1 - j)])
    mons = [(a, b) for a in range(p + 1) for b in range(p + 1 - a)]
    V = np.array([[s ** a * t ** b for (a, b) in mons] for (s, t) in pts])
    moments = np.array([factorial(a) * factorial(b) / factorial(a + b + 2) for a, b in mons])
    return pts, np.linalg.solve(V.T, moments)
