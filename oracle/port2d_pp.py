"""Port eigenmodes with edge elements of any order (oracle; test infrastructure only).

The reference's 2D solver discretises the port cross-section with MFEM's
ND_FECollection(order) for e_t and H1_FECollection(order) for e_z
(src/OpenParEM2D/fem2D.cpp:2188-2191), order = the project's mesh.order, on the
port's own faces.  The tangential trace of the 3D ND space of the same order
on those faces is that same 2D edge space, so a mode solved in it is carried
into the 3D problem without interpolation error.  This module restates the
modal problem of oracle.port2d (Lee-Sun-Cendes pencil, PEC outer boundary,
shift-invert about -k0^2 max(eps_r mu_r)) for any order p >= 1:

* e_t in the first-kind Nedelec space of order p on each triangle,
  R_p = P_{p-1}^2 + {(-y, x) h : h homogeneous of degree p-1} (p (p+2)
  functions), mapped by the covariant Piola map; degrees of freedom the edge
  moments int_0^1 (N . (B - A)) L_k(s) ds against shifted Legendre
  polynomials L_0..L_{p-1} along each edge from its lower to its higher global
  vertex, and the interior moments against P_{p-2}^2;
* e_z in the Lagrange space of degree p (equispaced nodes, edge nodes counted
  from the lower global vertex).
The discrete eigenvalues depend on the spaces only, not on the bases chosen
for them.  At p = 1 and p = 2 the spaces are those of port2d.solve_mode and
port2d.solve_mode_p2.
"""
from math import comb

import numpy as np
import scipy.sparse as sp
import scipy.sparse.linalg as spla

from .materials import MU0, EPS0
from .nd_basis import shifted_legendre, tri_test_polys, monomials2
from .quadrature import line_rule, tri_rule

LP = ((0, 1), (0, 2), (1, 2))           # local edges (local vertices sorted by global id)
VREF = np.array([[0.0, 0.0], [1.0, 0.0], [0.0, 1.0]])


def _mono(M, X):
    """Values (q, m) and derivatives d/dx, d/dy of the monomials M (m, 2) at X (q, 2)."""
    x, y = X[:, 0:1], X[:, 1:2]
    a, b = M[None, :, 0], M[None, :, 1]
    v = x ** a * y ** b
    dx = np.where(a > 0, a * x ** np.maximum(a - 1, 0) * y ** b, 0.0)
    dy = np.where(b > 0, b * x ** a * y ** np.maximum(b - 1, 0), 0.0)
    return v, dx, dy


class RefSpaces:
    """Nodal bases of ND_p and H1_p on the reference triangle, as coefficient
    arrays over monomials2(p): ND function i = (sum_m CX[m,i] mono_m,
    sum_m CY[m,i] mono_m); H1 function i = sum_m CL[m,i] mono_m."""

    def __init__(self, p):
        self.p = p
        M = monomials2(p)
        self.M = M
        idx = {(int(a), int(b)): i for i, (a, b) in enumerate(M)}
        nm = len(M)
        # spanning set of R_p
        FX, FY = [], []
        for a, b in monomials2(p - 1):
            e = np.zeros(nm)
            e[idx[(int(a), int(b))]] = 1.0
            FX.append(e); FY.append(np.zeros(nm))
            FX.append(np.zeros(nm)); FY.append(e.copy())
        for a in range(p):            # (-y, x) x^a y^(p-1-a)
            b = p - 1 - a
            ex, ey = np.zeros(nm), np.zeros(nm)
            ex[idx[(a, b + 1)]] = -1.0
            ey[idx[(a + 1, b)]] = 1.0
            FX.append(ex); FY.append(ey)
        FX, FY = np.array(FX).T, np.array(FY).T        # (nm, nf)
        nf = FX.shape[1]
        assert nf == p * (p + 2)
        # degrees of freedom of each spanning function
        s, ws = line_rule(2 * p + 2)
        D = []
        for a, b in LP:
            A, B = VREF[a], VREF[b]
            X = A[None, :] + s[:, None] * (B - A)[None, :]
            v = _mono(M, X)[0]
            tang = v @ FX * (B - A)[0] + v @ FY * (B - A)[1]          # (q, nf)
            for k in range(p):
                D.append((ws * shifted_legendre(k, s)) @ tang)
        if p >= 2:
            st, wt = tri_rule(2 * p + 2)
            v = _mono(M, st)[0]
            Q = _mono(monomials2(p - 2), st)[0] @ tri_test_polys(p - 2).T
            for r in range(Q.shape[1]):
                D.append((wt * Q[:, r]) @ (v @ FX))
                D.append((wt * Q[:, r]) @ (v @ FY))
        D = np.array(D)
        Ci = np.linalg.inv(D)                          # columns: nodal functions over the spanning set
        self.CX, self.CY = FX @ Ci, FY @ Ci
        self.nnd = nf
        # Lagrange nodes: vertices, edge nodes from the edge's first vertex, interior
        nodes = [VREF[0], VREF[1], VREF[2]]
        for a, b in LP:
            for k in range(1, p):
                nodes.append(VREF[a] + k / p * (VREF[b] - VREF[a]))
        for j in range(1, p):
            for i in range(1, p - j):
                nodes.append(np.array([i / p, j / p]))
        nodes = np.array(nodes)
        assert len(nodes) == comb(p + 2, 2)
        self.CL = np.linalg.inv(_mono(M, nodes)[0])      # (nm, nl): L_i(node_j) = delta
        self.nl = len(nodes)

    def nd(self, X):
        """Values (q, n, 2) and scalar curls (q, n) of the ND functions at X."""
        v, dx, dy = _mono(self.M, X)
        N = np.stack([v @ self.CX, v @ self.CY], axis=2)
        curl = dx @ self.CY - dy @ self.CX
        return N, curl

    def h1(self, X):
        """Values (q, n) and gradients (q, n, 2) of the Lagrange functions at X."""
        v, dx, dy = _mono(self.M, X)
        return v @ self.CL, np.stack([dx @ self.CL, dy @ self.CL], axis=2)


_REF = {}


def ref_spaces(p):
    if p not in _REF:
        _REF[p] = RefSpaces(p)
    return _REF[p]


def _nd_numbering(st, p):
    """Global ND_p DOFs of each triangle (T, p(p+2)): p per edge (edges of the
    sorted vertex pairs), p(p-1) per triangle; returns (tdofs, net, edges, einv)."""
    nt = len(st)
    ekey = np.concatenate([st[:, [a, b]] for a, b in LP])
    edges, einv = np.unique(ekey, axis=0, return_inverse=True)
    tedge = einv.reshape(3, nt).T
    ne = len(edges)
    nint = p * (p - 1)
    net = ne * p + nt * nint
    tdofs = np.concatenate([(tedge[:, :, None] * p + np.arange(p)[None, None, :]).reshape(nt, 3 * p),
                            ne * p + nint * np.arange(nt)[:, None] + np.arange(nint)[None, :]], axis=1)
    return tdofs, net, edges, einv


def project_nd(pts, tris, p, weight, field):
    """Weighted L2 projection of a tangential field onto ND_p of the triangles,
    as the reference's 2D solver forms H_t (Hsolve, src/OpenParEM2D/Hsolve.c:454-560:
    Mt H_t = gamma Zt E_t + Cz E_z with Mt the mass matrix weighted by omega mu,
    src/OpenParEM2D/fem2D.cpp:2297-2326; no boundary condition).  field(t, X2)
    -> (q, 2) values at points X2 of triangle t; weight (T,) per triangle.
    Returns per-triangle coefficients (T, p(p+2)) on the bases of ref_spaces(p)."""
    pts = np.asarray(pts, dtype=float)
    st = np.sort(np.asarray(tris, dtype=np.int64), axis=1)
    nt = len(st)
    tdofs, net, _, _ = _nd_numbering(st, p)
    X, w = tri_rule(2 * p + 2)
    Nh, _ = ref_spaces(p).nd(X)
    rows, cols, vals = [], [], []
    rhs = np.zeros(net, dtype=complex)
    for t in range(nt):
        P = pts[st[t]]
        J = np.array([P[1] - P[0], P[2] - P[0]]).T
        det = np.linalg.det(J)
        N = np.einsum("ij,qnj->qni", np.linalg.inv(J).T, Nh)
        wq = w * abs(det) * weight[t]
        td = tdofs[t]
        rows.append(np.repeat(td, len(td))); cols.append(np.tile(td, len(td)))
        vals.append(np.einsum("q,qai,qbi->ab", wq, N, N).ravel())
        np.add.at(rhs, td, np.einsum("q,qai,qi->a", wq, N, field(t, P[0] + X @ J.T)))
    M = sp.csc_matrix((np.concatenate(vals), (np.concatenate(rows), np.concatenate(cols))), shape=(net, net))
    return spla.spsolve(M, rhs)[tdofs]


def solve_mode_pp(pts, tris, freq, eps_r, mu_r=None, p=1, mode=0):
    """Fundamental mode (mode 0), or the mode-th mode in decreasing beta^2, with
    order-p elements: (beta, ct (T, p(p+2)), cz (T, nl), st (T,3) sorted vertex
    ids): per triangle the coefficients of e_t and e_z on the reference nodal
    bases of ref_spaces(p), the triangle's local vertices in increasing global
    order."""
    pts = np.asarray(pts, dtype=float)
    tris = np.asarray(tris, dtype=np.int64)
    nt = len(tris)
    eps_r = np.broadcast_to(np.asarray(eps_r, dtype=complex), (nt,))
    mu_r = np.ones(nt, dtype=complex) if mu_r is None else np.broadcast_to(np.asarray(mu_r, dtype=complex), (nt,))
    k0 = 2 * np.pi * freq * np.sqrt(MU0 * EPS0)
    R = ref_spaces(p)
    st = np.sort(tris, axis=1)
    tdofs, net, edges, einv = _nd_numbering(st, p)
    tedge = einv.reshape(3, nt).T
    ne, nn = len(edges), len(pts)
    nle, nli = p - 1, (p - 1) * (p - 2) // 2
    nz = nn + ne * nle + nt * nli
    zdofs = np.concatenate([st, (nn + tedge[:, :, None] * nle + np.arange(nle)[None, None, :]).reshape(nt, 3 * nle),
                            nn + ne * nle + nli * np.arange(nt)[:, None] + np.arange(nli)[None, :]], axis=1)
    X, w = tri_rule(2 * p + 1)
    Nh, ch = R.nd(X)                  # (q, n, 2), (q, n)
    Lh, gLh = R.h1(X)                 # (q, l), (q, l, 2)
    rows_ee, cols_ee, vS, vTe, vTm = [], [], [], [], []
    rows_ez, cols_ez, vG = [], [], []
    rows_zz, cols_zz, vZ = [], [], []
    for t in range(nt):
        P = pts[st[t]]
        J = np.array([P[1] - P[0], P[2] - P[0]]).T
        det = np.linalg.det(J)
        JiT = np.linalg.inv(J).T
        N = np.einsum("ij,qnj->qni", JiT, Nh)            # covariant Piola
        cu = ch / det
        gL = np.einsum("ij,qlj->qli", JiT, gLh)
        wq = w * abs(det)
        im, ie = 1.0 / mu_r[t], eps_r[t]
        S = np.einsum("q,qa,qb->ab", wq, cu, cu)
        T = np.einsum("q,qai,qbi->ab", wq, N, N)
        G = np.einsum("q,qai,qbi->ab", wq, N, gL)
        K = np.einsum("q,qai,qbi->ab", wq, gL, gL)
        M = np.einsum("q,qa,qb->ab", wq, Lh, Lh)
        td, zd = tdofs[t], zdofs[t]
        rows_ee.append(np.repeat(td, len(td))); cols_ee.append(np.tile(td, len(td)))
        vS.append((im * S).ravel()); vTe.append((ie * T).ravel()); vTm.append((im * T).ravel())
        rows_ez.append(np.repeat(td, len(zd))); cols_ez.append(np.tile(zd, len(td))); vG.append((im * G).ravel())
        rows_zz.append(np.repeat(zd, len(zd))); cols_zz.append(np.tile(zd, len(zd)))
        vZ.append((im * K - k0 ** 2 * ie * M).ravel())
    cat = np.concatenate
    Sm = sp.csr_matrix((cat(vS), (cat(rows_ee), cat(cols_ee))), shape=(net, net))
    Te = sp.csr_matrix((cat(vTe), (cat(rows_ee), cat(cols_ee))), shape=(net, net))
    Tm = sp.csr_matrix((cat(vTm), (cat(rows_ee), cat(cols_ee))), shape=(net, net))
    Gm = sp.csr_matrix((cat(vG), (cat(rows_ez), cat(cols_ez))), shape=(net, nz))
    Kz = sp.csr_matrix((cat(vZ), (cat(rows_zz), cat(cols_zz))), shape=(nz, nz))
    # PEC walls: the DOFs of boundary edges (one triangle) and their vertices
    cnt = np.bincount(einv, minlength=ne)
    bedge = np.where(cnt == 1)[0]
    bnode = np.unique(edges[bedge].ravel())
    bt = (bedge[:, None] * p + np.arange(p)[None, :]).ravel()
    bz = np.concatenate([bnode, (nn + bedge[:, None] * nle + np.arange(nle)[None, :]).ravel()])
    ke = np.setdiff1d(np.arange(net), bt)
    kn = np.setdiff1d(np.arange(nz), bz)
    A = sp.bmat([[Sm - k0 ** 2 * Te, None], [None, sp.csr_matrix((nz, nz))]]).tocsr()
    B = sp.bmat([[Tm, -Gm], [-Gm.T, Kz]]).tocsr()
    keep = np.concatenate([ke, net + kn])
    A = A[keep][:, keep].tocsc()
    B = B[keep][:, keep].tocsc()
    sigma = -k0 ** 2 * np.max(np.real(eps_r * mu_r))
    lu = spla.splu((A - sigma * B).tocsc(), permc_spec="MMD_AT_PLUS_A")
    # every (0, psi) solves A x = 0 B x: a null space between the propagating
    # (lam < 0) and the cut-off (lam > 0) modes.  Setting psi from the e_z rows of
    # B x = 0, which every eigenvector of a nonzero lam satisfies, removes it.
    nt_ = len(ke)
    Bz = B[nt_:, nt_:].tocsc()
    Bzt = B[nt_:, :nt_].tocsr()
    luz = spla.splu(Bz, permc_spec="MMD_AT_PLUS_A") if Bz.shape[0] else None

    def op_mv(x):
        y = lu.solve(B @ x)
        if luz is not None:
            y[nt_:] = luz.solve(-(Bzt @ y[:nt_]))
        return y
    op = spla.LinearOperator(A.shape, matvec=op_mv, dtype=complex)
    mu, vec = spla.eigs(op, k=mode + 1, which="LM", tol=1e-14 if mode else 0)
    order = np.argsort(-np.abs(mu))          # nearest the shift first: decreasing beta^2
    lam = sigma + 1.0 / mu[order[mode]]
    beta = np.sqrt(-lam + 0j)
    if beta.real < 0:
        beta = -beta
    x = vec[:, order[mode]]
    et = np.zeros(net, dtype=complex)
    et[ke] = x[:len(ke)]
    psi = np.zeros(nz, dtype=complex)
    psi[kn] = x[len(ke):]
    ez = -1j * beta * psi
    return beta, et[tdofs], ez[zdofs], st
