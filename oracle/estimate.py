"""Zienkiewicz-Zhu mesh error indicator on H and refinement marking (oracle;
test infrastructure only).

Restates fem3D::calculateMeshErrors (src/OpenParEM3D/fem3D.cpp:1162-1420) with
its estimator OPEM_L2ZZErrorEstimator (:987-1154), as the reference runs them
(real and imaginary parts separately, norm_p = 1):

* flux: the element flux of CurlCurlIntegrator(1/mu_r) on the H field, i.e.
  F = (1/mu_r) curl H on each tetrahedron (curl of an order-p edge-element field
  lies in the order p-1 face-element space the reference stores it in);
* smooth flux: the L2 projection of F onto the order-p edge-element space,
  M1 s = b with b_i = int N_i . F = (Q_mu h)_i, solved to 1e-12 (the reference:
  CG with SOR, rtol 1e-12, 2000 iterations);
* error of element e: (int_e |Re s - Re F|) and (int_e |Im s - Im F|) (the L1
  norm of the Euclidean difference), combined as sqrt(re^2 + im^2);
* over the driving sets of one frequency the larger error per element is kept
  (:1258-1263);
* marking: the refinementCount = floor(NE * mesh.3D.refinement.fraction)
  (at least 1) largest errors, and maxMeshError = the largest (:1321-1350).

The integrals use the collapsed Gauss-Legendre tetrahedron rule of total
degree 2p + 2 (the integrand is not a polynomial, so the rule is part of the
definition; MFEM's own rule for ComputeElementLpDistance is not reproduced).
"""
import numpy as np
import scipy.sparse.linalg as spla

from .fem import basis, element_geometry


def estimator_rule(p):
    """x = u, y = (1-u) v, z = (1-u)(1-v) t with n-point Gauss-Legendre in u, v, t,
    n = (2p + 5) // 2 + 1; weights sum 1/6."""
    n = (2 * p + 2 + 3) // 2 + 1
    g, gw = np.polynomial.legendre.leggauss(n)
    g = 0.5 * (g + 1.0)
    gw = 0.5 * gw
    U, V, T = np.meshgrid(g, g, g, indexing="ij")
    WU, WV, WT = np.meshgrid(gw, gw, gw, indexing="ij")
    X = np.stack([U.ravel(), ((1 - U) * V).ravel(), ((1 - U) * (1 - V) * T).ravel()], axis=1)
    W = (WU * WV * WT * (1 - U) ** 2 * (1 - V)).ravel()
    return X, W


def element_errors(ops, s, h):
    """Per element: sqrt((int |Re(s - F)|)^2 + (int |Im(s - F)|)^2), F = curl h / mu_r."""
    prob, topo = ops.prob, ops.topo
    B = basis(topo.p)[0]
    X, W = estimator_rule(topo.p)
    phi = B.eval(X)           # (ld, nq, 3)
    cur = B.eval_curl(X)
    J, det, _, _ = element_geometry(np.asarray(prob["verts"], dtype=np.float64), topo.tets)
    Ji = np.linalg.inv(J)
    mu = np.asarray(prob["mu_r"], dtype=np.float64)[np.asarray(prob["tet_region"], dtype=np.int64)]
    se = s[topo.dof]          # (ne, ld)
    he = h[topo.dof]
    Sref = np.einsum("ei,iqc->eqc", se, phi)
    Cref = np.einsum("ei,iqc->eqc", he, cur)
    Sp = np.einsum("eba,eqb->eqa", Ji, Sref)                         # J^-T
    Fp = np.einsum("eab,eqb->eqa", J, Cref) / (det * mu)[:, None, None]
    D = Sp - Fp
    wq = np.abs(det)[:, None] * W[None, :]
    er = np.sum(wq * np.linalg.norm(D.real, axis=2), axis=1)
    ei = np.sum(wq * np.linalg.norm(D.imag, axis=2), axis=1)
    return np.sqrt(er ** 2 + ei ** 2)


def smooth_flux(ops, h):
    """L2 projection of curl h / mu_r onto the edge-element space."""
    lu = spla.splu(ops.M1.tocsc(), permc_spec="MMD_AT_PLUS_A", options=dict(SymmetricMode=True, DiagPivotThresh=0.0))
    b = ops.Q_mu @ h
    return lu.solve(b.real) + 1j * lu.solve(b.imag)


def mesh_errors(ops, h_list, fraction):
    """(errors per element, marked element ids (largest first), max error)."""
    ne = len(ops.topo.tets)
    err = np.zeros(ne)
    for h in h_list:
        err = np.maximum(err, element_errors(ops, smooth_flux(ops, h), h))
    count = max(1, int(ne * fraction))
    marked = np.argsort(-err, kind="stable")[:count]
    return err, marked, float(err.max())
