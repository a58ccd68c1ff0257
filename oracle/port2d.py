"""Port eigenmodes of a waveguide cross-section (oracle; test infrastructure only).

The reference computes port modes with its 2D solver OpenParEM2D, spawned by
OpenParEM3D (src/OpenParEM3D/port.cpp:5081-5176; the eigenproblem in
src/OpenParEM2D/fem2D.cpp with SLEPc, eigensolve.c:849-977).  This module
restates the modal problem of an inhomogeneously filled guide with PEC walls:
fields E = (e_t + z e_z) exp(-j beta z) in the weak form of
curl (1/mu_r) curl E - k0^2 eps_r E = 0, with lowest-order edge elements for
e_t and linear nodal elements for e_z.  Writing psi = j e_z / beta gives the
symmetric generalized eigenproblem (Lee, Sun and Cendes, IEEE MTT 1991)

    [S - k0^2 T_eps   0] [e_t]          [ T_mu   -G ] [e_t]
    [      0          0] [psi] = -beta^2 [ -G^T   Kz ] [psi]

S = int (1/mu_r) curl N_i curl N_j,  T_eps = int eps_r N_i . N_j,
T_mu = int (1/mu_r) N_i . N_j,  G = int (1/mu_r) N_i . grad L_j,
Kz = int (1/mu_r) grad L_i . grad L_j - k0^2 eps_r L_i L_j.
The fundamental mode has the largest beta^2; it is found by shift-invert
about -k0^2 max(eps_r mu_r).  The analytic dispersion relation of a guide
loaded by a centred full-height dielectric slab (TE_m0 family) is included
as an independent check.
"""
import numpy as np
import scipy.sparse as sp
import scipy.sparse.linalg as spla
from scipy.optimize import brentq

from .materials import MU0, EPS0


def rect_mesh(a, b, nx, ny, x_breaks=()):
    """Triangles of [-a/2, a/2] x [-b/2, b/2] with about nx cells across; the x
    grid is uniform between consecutive x_breaks (so a slab's interfaces are mesh
    lines and every segment has cells of about the same width)."""
    knots = np.unique(np.concatenate([[-a / 2, a / 2], np.asarray(x_breaks, dtype=float)]))
    h = a / nx
    segs = [np.linspace(x0, x1, max(1, int(round((x1 - x0) / h))) + 1) for x0, x1 in zip(knots[:-1], knots[1:])]
    xs = np.unique(np.concatenate(segs))
    ys = np.linspace(-b / 2, b / 2, ny + 1)
    X, Y = np.meshgrid(xs, ys, indexing="ij")
    pts = np.stack([X.ravel(), Y.ravel()], axis=1)
    nyp = len(ys)
    tris = []
    for i in range(len(xs) - 1):
        for j in range(ny):
            v00, v10, v01, v11 = i * nyp + j, (i + 1) * nyp + j, i * nyp + j + 1, (i + 1) * nyp + j + 1
            tris.append([v00, v10, v11])
            tris.append([v00, v11, v01])
    return pts, np.array(tris, dtype=np.int64)


def solve_mode(pts, tris, freq, eps_r, mu_r=None):
    """Fundamental mode: (beta (complex), e_t edge coefficients, e_z nodal values,
    edges (sorted vertex pairs)).  eps_r, mu_r: per triangle (complex allowed)."""
    pts = np.asarray(pts, dtype=float)
    tris = np.asarray(tris, dtype=np.int64)
    nt = len(tris)
    eps_r = np.broadcast_to(np.asarray(eps_r, dtype=complex), (nt,))
    mu_r = np.ones(nt, dtype=complex) if mu_r is None else np.broadcast_to(np.asarray(mu_r, dtype=complex), (nt,))
    k0 = 2 * np.pi * freq * np.sqrt(MU0 * EPS0)
    lp = [(0, 1), (0, 2), (1, 2)]
    st = np.sort(tris, axis=1)
    ekey = np.concatenate([st[:, [a, b]] for a, b in lp])
    edges, einv = np.unique(ekey, axis=0, return_inverse=True)
    tedge = einv.reshape(3, nt).T
    ne, nn = len(edges), len(pts)
    rows, cols, vS, vTe, vTm, vG, vKz = [], [], [], [], [], [], []
    Gr, Gc, Gv = [], [], []
    Zr, Zc, Zv = [], [], []
    for t in range(nt):
        v = st[t]
        P = pts[v]
        J = np.array([P[1] - P[0], P[2] - P[0]]).T
        area = 0.5 * abs(np.linalg.det(J))
        gl = np.linalg.inv(J).T @ np.array([[-1, 1, 0], [-1, 0, 1.0]])   # columns: grad lambda_i
        g = [gl[:, i] for i in range(3)]
        Mll = area / 12.0 * (np.ones((3, 3)) + np.eye(3))                # int lambda_i lambda_j
        curl = [2.0 * (g[a][0] * g[b][1] - g[a][1] * g[b][0]) for a, b in lp]

        def nn_(i, j):   # int N_i . N_j, N = l_a g_b - l_b g_a
            a, b = lp[i]
            c, d = lp[j]
            return (Mll[a, c] * g[b] @ g[d] - Mll[a, d] * g[b] @ g[c] - Mll[b, c] * g[a] @ g[d]
                    + Mll[b, d] * g[a] @ g[c])

        def ng_(i, k):   # int N_i . grad l_k = (area/3) (g_b - g_a) . g_k
            a, b = lp[i]
            return area / 3.0 * ((g[b] - g[a]) @ g[k])

        im, ie = 1.0 / mu_r[t], eps_r[t]
        for i in range(3):
            for j in range(3):
                rows.append(tedge[t, i]); cols.append(tedge[t, j])
                vS.append(im * curl[i] * curl[j] * area)
                m = nn_(i, j)
                vTe.append(ie * m); vTm.append(im * m)
            for k in range(3):
                Gr.append(tedge[t, i]); Gc.append(v[k]); Gv.append(im * ng_(i, k))
        for k in range(3):
            for l in range(3):
                Zr.append(v[k]); Zc.append(v[l])
                Zv.append(im * area * (g[k] @ g[l]) - k0 ** 2 * ie * Mll[k, l])
    S = sp.csr_matrix((vS, (rows, cols)), shape=(ne, ne))
    Te = sp.csr_matrix((vTe, (rows, cols)), shape=(ne, ne))
    Tm = sp.csr_matrix((vTm, (rows, cols)), shape=(ne, ne))
    G = sp.csr_matrix((Gv, (Gr, Gc)), shape=(ne, nn))
    Kz = sp.csr_matrix((Zv, (Zr, Zc)), shape=(nn, nn))
    # PEC walls: boundary edges (one triangle) and their nodes
    cnt = np.bincount(einv, minlength=ne)
    bedge = np.where(cnt == 1)[0]
    bnode = np.unique(edges[bedge].ravel())
    ke = np.setdiff1d(np.arange(ne), bedge)
    kn = np.setdiff1d(np.arange(nn), bnode)
    A = sp.bmat([[S - k0 ** 2 * Te, None], [None, sp.csr_matrix((nn, nn))]]).tocsr()
    B = sp.bmat([[Tm, -G], [-G.T, Kz]]).tocsr()
    keep = np.concatenate([ke, ne + kn])
    A = A[keep][:, keep].tocsc()
    B = B[keep][:, keep].tocsc()
    sigma = -k0 ** 2 * np.max(np.real(eps_r * mu_r))
    lu = spla.splu((A - sigma * B).tocsc(), permc_spec="MMD_AT_PLUS_A")
    op = spla.LinearOperator(A.shape, matvec=lambda x: lu.solve(B @ x), dtype=complex)
    mu, vec = spla.eigs(op, k=1, which="LM")
    lam = sigma + 1.0 / mu[0]
    beta = np.sqrt(-lam + 0j)
    if beta.real < 0:
        beta = -beta
    x = vec[:, 0]
    et = np.zeros(ne, dtype=complex)
    et[ke] = x[:len(ke)]
    psi = np.zeros(nn, dtype=complex)
    psi[kn] = x[len(ke):]
    ez = -1j * beta * psi
    return beta, et, ez, edges


def slab_beta(a, slab_width, eps_slab, freq, eps_air=1.0):
    """Fundamental TE_10-like beta of a guide of width a with a centred full-height
    slab: kd tan(kd w/2) = ka cot(ka (a-w)/2), kd^2 = eps_slab k0^2 - beta^2,
    ka^2 = eps_air k0^2 - beta^2."""
    k0 = 2 * np.pi * freq * np.sqrt(MU0 * EPS0)
    w = slab_width

    def F(beta):
        kd = np.sqrt(eps_slab * k0 ** 2 - beta ** 2 + 0j)
        ka = np.sqrt(eps_air * k0 ** 2 - beta ** 2 + 0j)
        return (kd * np.tan(kd * w / 2) - ka / np.tan(ka * (a - w) / 2)).real

    lo = np.sqrt(max(eps_air * k0 ** 2 - (np.pi / a) ** 2, 0.0)) * (1 + 1e-9)
    hi = k0 * np.sqrt(eps_slab) * (1 - 1e-12)
    bs = np.linspace(lo, hi, 20001)
    fv = np.array([F(b) for b in bs])
    best = None
    for i in range(len(bs) - 1):
        if np.sign(fv[i]) != np.sign(fv[i + 1]) and abs(fv[i]) < 1e4 and abs(fv[i + 1]) < 1e4:
            best = brentq(F, bs[i], bs[i + 1], xtol=1e-14, rtol=1e-15)   # largest root wins (last)
    return best


# ---------------------------------------------------------------------------
# Second-order elements: e_t in the first-kind edge space of degree 2 (8 per
# triangle), e_z in quadratic nodal elements (6 per triangle).  With the
# triangle's vertices sorted by node id and lambda_0..2 their barycentrics,
#   e_t: W_ab = l_a grad l_b - l_b grad l_a and G_ab = grad(l_a l_b) for the edges
#        (a,b) = (0,1), (0,2), (1,2), then the face functions l_2 W_01, l_0 W_12;
#   e_z: l_0, l_1, l_2, then the edge bubbles l_a l_b.
# W_ab and G_ab of an edge are shared by its triangles (global orientation: low
# to high node id); the face functions have no tangential trace.  Whitney plus
# edge gradients span the complete linear fields; the face functions complete
# the degree-2 space (Webb, IEEE TAP 47(8) 1999).
LP2 = [(0, 1), (0, 2), (1, 2)]


def p2_basis(lam, g):
    """Values at barycentric points lam (q,3) of a triangle with gradients g (3,2):
    N (q,8,2), curl N (q,8), L (q,6), grad L (q,6,2)."""
    q = len(lam)
    N = np.zeros((q, 8, 2))
    cN = np.zeros((q, 8))
    L = np.zeros((q, 6))
    dL = np.zeros((q, 6, 2))

    def cross(u, v):
        return u[..., 0] * v[..., 1] - u[..., 1] * v[..., 0]
    for i, (a, b) in enumerate(LP2):
        N[:, i] = lam[:, a:a + 1] * g[b][None, :] - lam[:, b:b + 1] * g[a][None, :]
        cN[:, i] = 2.0 * cross(g[a], g[b])
        N[:, 3 + i] = lam[:, a:a + 1] * g[b][None, :] + lam[:, b:b + 1] * g[a][None, :]
        L[:, 3 + i] = lam[:, a] * lam[:, b]
        dL[:, 3 + i] = N[:, 3 + i]
    for k, (c, (a, b)) in enumerate(((2, (0, 1)), (0, (1, 2)))):
        W = lam[:, a:a + 1] * g[b][None, :] - lam[:, b:b + 1] * g[a][None, :]
        N[:, 6 + k] = lam[:, c:c + 1] * W
        cN[:, 6 + k] = cross(np.broadcast_to(g[c], W.shape), W) + lam[:, c] * 2.0 * cross(g[a], g[b])
    for k in range(3):
        L[:, k] = lam[:, k]
        dL[:, k] = g[k][None, :]
    return N, cN, L, dL


def solve_mode_p2(pts, tris, freq, eps_r, mu_r=None):
    """Fundamental mode with second-order elements: (beta, ct (T,8), cz (T,6),
    st (T,3) sorted vertex ids) with per-triangle local coefficients."""
    from .quadrature import tri_rule
    pts = np.asarray(pts, dtype=float)
    tris = np.asarray(tris, dtype=np.int64)
    nt = len(tris)
    eps_r = np.broadcast_to(np.asarray(eps_r, dtype=complex), (nt,))
    mu_r = np.ones(nt, dtype=complex) if mu_r is None else np.broadcast_to(np.asarray(mu_r, dtype=complex), (nt,))
    k0 = 2 * np.pi * freq * np.sqrt(MU0 * EPS0)
    st = np.sort(tris, axis=1)
    ekey = np.concatenate([st[:, [a, b]] for a, b in LP2])
    edges, einv = np.unique(ekey, axis=0, return_inverse=True)
    tedge = einv.reshape(3, nt).T
    ne, nn = len(edges), len(pts)
    # global numbering: e_t = [W (ne), G (ne), face (2 nt)], e_z = [vertex (nn), bubble (ne)]
    net = 2 * ne + 2 * nt
    tdofs = np.concatenate([tedge, ne + tedge, 2 * ne + 2 * np.arange(nt)[:, None] + np.arange(2)[None, :]], axis=1)
    zdofs = np.concatenate([st, nn + tedge], axis=1)
    s, wq = tri_rule(4)
    lam = np.stack([1 - s[:, 0] - s[:, 1], s[:, 0], s[:, 1]], axis=1)
    rows_ee, cols_ee, vA, vT = [], [], [], []
    rows_ez, cols_ez, vG = [], [], []
    rows_zz, cols_zz, vZ = [], [], []
    for t in range(nt):
        P = pts[st[t]]
        J = np.array([P[1] - P[0], P[2] - P[0]]).T
        area = 0.5 * abs(np.linalg.det(J))
        gl = np.linalg.inv(J).T @ np.array([[-1, 1, 0], [-1, 0, 1.0]])
        g = [gl[:, i] for i in range(3)]
        N, cN, L, dL = p2_basis(lam, g)
        w = 2 * area * wq
        im, ie = 1.0 / mu_r[t], eps_r[t]
        M = np.einsum("q,qia,qja->ij", w, N, N)
        C = np.einsum("q,qi,qj->ij", w, cN, cN)
        Gm = np.einsum("q,qia,qja->ij", w, N, dL)
        Kg = np.einsum("q,qia,qja->ij", w, dL, dL)
        Ml = np.einsum("q,qi,qj->ij", w, L, L)
        rows_ee.append(np.repeat(tdofs[t], 8)); cols_ee.append(np.tile(tdofs[t], 8))
        vA.append((im * C - k0 ** 2 * ie * M).ravel()); vT.append((im * M).ravel())
        rows_ez.append(np.repeat(tdofs[t], 6)); cols_ez.append(np.tile(zdofs[t], 8)); vG.append((im * Gm).ravel())
        rows_zz.append(np.repeat(zdofs[t], 6)); cols_zz.append(np.tile(zdofs[t], 6))
        vZ.append((im * Kg - k0 ** 2 * ie * Ml).ravel())
    cat = np.concatenate
    A_ee = sp.csr_matrix((cat(vA), (cat(rows_ee), cat(cols_ee))), shape=(net, net))
    T_mu = sp.csr_matrix((cat(vT), (cat(rows_ee), cat(cols_ee))), shape=(net, net))
    G = sp.csr_matrix((cat(vG), (cat(rows_ez), cat(cols_ez))), shape=(net, nn + ne))
    Kz = sp.csr_matrix((cat(vZ), (cat(rows_zz), cat(cols_zz))), shape=(nn + ne, nn + ne))
    # PEC: both edge functions of boundary edges, boundary vertices and bubbles
    cnt = np.bincount(einv, minlength=ne)
    bedge = np.where(cnt == 1)[0]
    bnode = np.unique(edges[bedge].ravel())
    kt = np.setdiff1d(np.arange(net), np.concatenate([bedge, ne + bedge]))
    kz = np.setdiff1d(np.arange(nn + ne), np.concatenate([bnode, nn + bedge]))
    nz = nn + ne
    A = sp.bmat([[A_ee, None], [None, sp.csr_matrix((nz, nz))]]).tocsr()
    B = sp.bmat([[T_mu, -G], [-G.T, Kz]]).tocsr()
    keep = np.concatenate([kt, net + kz])
    A = A[keep][:, keep].tocsc()
    B = B[keep][:, keep].tocsc()
    sigma = -k0 ** 2 * np.max(np.real(eps_r * mu_r))
    lu = spla.splu((A - sigma * B).tocsc(), permc_spec="MMD_AT_PLUS_A")
    op = spla.LinearOperator(A.shape, matvec=lambda x: lu.solve(B @ x), dtype=complex)
    mu_, vec = spla.eigs(op, k=1, which="LM")
    lam_ = sigma + 1.0 / mu_[0]
    beta = np.sqrt(-lam_ + 0j)
    if beta.real < 0:
        beta = -beta
    x = vec[:, 0]
    et = np.zeros(net, dtype=complex)
    et[kt] = x[:len(kt)]
    psi = np.zeros(nz, dtype=complex)
    psi[kz] = x[len(kt):]
    ez = -1j * beta * psi
    return beta, et[tdofs], ez[zdofs], st
