"""Nedelec (first kind) order-p basis on the reference tetrahedron (oracle).

The space is ND_p = P_{p-1}^3 + x cross P~_{p-1}^3, the space of MFEM's
``ND_FECollection(p, 3)`` that the reference builds at
src/OpenParEM3D/fem3D.cpp:65-66.  The basis is the dual basis of moment
degrees of freedom defined on the reference tetrahedron whose vertices are
the element's vertices sorted by global index:

* edge (a,b), a<b, tangent t=v_b-v_a:      int_0^1 u(v_a+s t).t  P_k(2s-1) ds,      k<p
* face (a,b,c), a<b<c, t1=v_b-v_a, t2=v_c-v_a:
                                            int_unit-tri u.t_m  q_r(s1,s2)  ds1 ds2,  r<dim P_{p-2}, m=1,2
* interior:                                 int_T u_d  w_r(x,y,z)  dx,                r<dim P_{p-3}, d=x,y,z

q_r and w_r are the monomials (ordered by degree, leading exponent
descending) orthonormalised by the Cholesky factor of their exact Gram
matrix on the unit triangle / reference tetrahedron.

Because every shared edge and face is parameterised from its lowest global
vertex on both sides, the same functional is used by every element that
touches it, so the global space is H(curl)-conforming with no sign flips.

Local DOF order: 6 edges (01,02,03,12,13,23) x p, then 4 faces
(012,013,023,123) x [monomials by degree, i descending] x [t1,t2], then
interior x [monomials] x [x,y,z].
"""
import numpy as np
from .quadrature import line_rule, tri_rule, tet_rule

VERTS = np.array([[0.0, 0, 0], [1.0, 0, 0], [0.0, 1, 0], [0.0, 0, 1]])
EDGES = [(0, 1), (0, 2), (0, 3), (1, 2), (1, 3), (2, 3)]
FACES = [(0, 1, 2), (0, 1, 3), (0, 2, 3), (1, 2, 3)]
# edges of each face, as indices into EDGES, in the face's (ab, ac, bc) order
FACE_EDGES = [[EDGES.index((f[0], f[1])), EDGES.index((f[0], f[2])), EDGES.index((f[1], f[2]))]
              for f in FACES]


def monomials3(P):
    E = []
    for d in range(P + 1):
        for a in range(d, -1, -1):
            for b in range(d - a, -1, -1):
                E.append((a, b, d - a - b))
    return np.array(E, dtype=np.int64).reshape(-1, 3)


def monomials2(P):
    E = []
    for d in range(P + 1):
        for i in range(d, -1, -1):
            E.append((i, d - i))
    return np.array(E, dtype=np.int64).reshape(-1, 2)


def vander3(X, E):
    X = np.atleast_2d(X)
    return (X[:, 0:1] ** E[None, :, 0]) * (X[:, 1:2] ** E[None, :, 1]) * (X[:, 2:3] ** E[None, :, 2])


def _gram_cholesky_inv(G):
    L = np.linalg.cholesky(G)
    return np.linalg.solve(L, np.eye(len(G)))


def tri_test_polys(P):
    """Coefficients T (n,n) over monomials2(P): q_r = sum_c T[r,c] s1^i_c s2^j_c are
    orthonormal on the unit triangle (Cholesky of the exact Gram matrix
    int s1^a s2^b = a! b! / (a+b+2)!)."""
    from math import factorial
    M = monomials2(P)
    G = np.array([[factorial(a[0] + b[0]) * factorial(a[1] + b[1]) / factorial(a[0] + b[0] + a[1] + b[1] + 2)
                   for b in M] for a in M])
    return _gram_cholesky_inv(G)


def tet_test_polys(P):
    """As tri_test_polys on the reference tet (int x^a y^b z^c = a! b! c! / (a+b+c+3)!)."""
    from math import factorial
    M = monomials3(P)
    G = np.array([[factorial(a[0] + b[0]) * factorial(a[1] + b[1]) * factorial(a[2] + b[2])
                   / factorial(int((a + b).sum()) + 3) for b in M] for a in M])
    return _gram_cholesky_inv(G)


def shifted_legendre(k, s):
    return np.polynomial.legendre.legval(2.0 * s - 1.0, [0] * k + [1])


def ndofs(p):
    return {"edge": p, "face": p * (p - 1), "interior": p * (p - 1) * (p - 2) // 2,
            "local": 6 * p + 4 * p * (p - 1) + p * (p - 1) * (p - 2) // 2}


class NDBasis:
    """Order-p basis: coefficients over monomials of degree <= p."""

    def __init__(self, p):
        assert p >= 1
        self.p = p
        self.E = monomials3(p)
        nm = len(self.E)
        self.nmon = nm
        idx = {tuple(e): i for i, e in enumerate(self.E)}
        # derivative matrices D[d] : coef -> coef of d/dx_d
        D = np.zeros((3, nm, nm))
        for j, e in enumerate(self.E):
            for d in range(3):
                if e[d] > 0:
                    f = list(e); f[d] -= 1
                    D[d, idx[tuple(f)], j] = e[d]
        self.D = D
        # spanning set of ND_p
        span = []
        for j, e in enumerate(self.E):
            if e.sum() <= p - 1:
                for c in range(3):
                    v = np.zeros((3, nm)); v[c, j] = 1.0; span.append(v)
        for j, e in enumerate(self.E):
            if e.sum() == p - 1:
                for c in range(3):
                    # x cross (e_c m)
                    v = np.zeros((3, nm))
                    for r in range(3):
                        # (x cross e_c)_r = eps_{r s c} x_s
                        for s in range(3):
                            eps = _levi(r, s, c)
                            if eps != 0:
                                f = list(e); f[s] += 1
                                v[r, idx[tuple(f)]] += eps
                    span.append(v)
        S = np.array(span).reshape(len(span), -1)
        _, sv, Vt = np.linalg.svd(S, full_matrices=False)
        ld = ndofs(p)["local"]
        rank = int((sv > 1e-10 * sv[0]).sum())
        assert rank == ld, (rank, ld)
        Psi = Vt[:ld]                      # (ld, 3*nm)
        W = self._functionals()            # (ld, 3*nm)
        Dm = W @ Psi.T                     # D_ij = l_i(psi_j)
        C = np.linalg.solve(Dm, np.eye(ld)).T   # phi_k = sum_j C_kj psi_j
        self.coef = (C @ Psi).reshape(ld, 3, nm)
        self.ld = ld
        # curl coefficients
        cc = np.zeros_like(self.coef)
        u = self.coef
        cc[:, 0] = np.einsum("mn,in->im", D[1], u[:, 2]) - np.einsum("mn,in->im", D[2], u[:, 1])
        cc[:, 1] = np.einsum("mn,in->im", D[2], u[:, 0]) - np.einsum("mn,in->im", D[0], u[:, 2])
        cc[:, 2] = np.einsum("mn,in->im", D[0], u[:, 1]) - np.einsum("mn,in->im", D[1], u[:, 0])
        self.curl_coef = cc

    def _functionals(self):
        p, E, nm = self.p, self.E, self.nmon
        rows = []
        s, ws = line_rule(2 * p)
        for (a, b) in EDGES:
            t = VERTS[b] - VERTS[a]
            X = VERTS[a][None, :] + s[:, None] * t[None, :]
            V = vander3(X, E)
            for k in range(p):
                L = shifted_legendre(k, s)
                w = np.einsum("q,q,c,qm->cm", ws, L, t, V)
                rows.append(w.ravel())
        if p >= 2:
            st, wt = tri_rule(2 * p + 2)
            M2 = monomials2(p - 2)
            T2 = tri_test_polys(p - 2)
            Q2 = (st[:, 0:1] ** M2[None, :, 0]) * (st[:, 1:2] ** M2[None, :, 1]) @ T2.T
            for (a, b, c) in FACES:
                t1 = VERTS[b] - VERTS[a]; t2 = VERTS[c] - VERTS[a]
                X = VERTS[a][None, :] + st[:, 0:1] * t1[None, :] + st[:, 1:2] * t2[None, :]
                V = vander3(X, E)
                for r in range(len(M2)):
                    q = Q2[:, r]
                    for t in (t1, t2):
                        w = np.einsum("q,q,c,qm->cm", wt, q, t, V)
                        rows.append(w.ravel())
        if p >= 3:
            X, wq = tet_rule(2 * p + 2)
            V = vander3(X, E)
            M3 = monomials3(p - 3)
            Q3 = vander3(X, M3) @ tet_test_polys(p - 3).T
            for r in range(len(M3)):
                q = Q3[:, r]
                for d in range(3):
                    w = np.zeros((3, nm))
                    w[d] = np.einsum("q,q,qm->m", wq, q, V)
                    rows.append(w.ravel())
        return np.array(rows)

    def eval(self, X):
        """Values (ld, npts, 3) at reference points X (npts, 3)."""
        V = vander3(X, self.E)
        return np.einsum("icm,qm->iqc", self.coef, V)

    def eval_curl(self, X):
        V = vander3(X, self.E)
        return np.einsum("icm,qm->iqc", self.curl_coef, V)

    # ---- reference tensors -------------------------------------------------
    def reference_tensors(self):
        """Mhat[a,b] = int phi_i,a phi_j,b ; Khat[a,b] = int curl_i,a curl_j,b ;
        Qhat = int phi_i . curl phi_j  (all over the reference tet)."""
        X, w = tet_rule(2 * self.p + 1)
        P = self.eval(X)
        C = self.eval_curl(X)
        Mh = np.einsum("q,iqa,jqb->abij", w, P, P)
        Kh = np.einsum("q,iqa,jqb->abij", w, C, C)
        Qh = np.einsum("q,iqa,jqa->ij", w, P, C)
        return Mh, Kh, Qh

    def face_tensors(self, f, rule=None):
        """For local face f: (dofs, Fhat[k,l] (2,2,nf,nf), Chat (nf,nf)).

        Fhat[k,l]_ij = int_unit-tri (phi_i . t_k)(phi_j . t_l) ds,
        Chat_ij      = int_unit-tri (curl phi_i . N)(curl phi_j . N) ds, N = t1 x t2;
        exactly, or with rule = (points, weights) on the unit triangle.
        """
        a, b, c = FACES[f]
        t1 = VERTS[b] - VERTS[a]; t2 = VERTS[c] - VERTS[a]
        N = np.cross(t1, t2)
        st, wt = tri_rule(2 * self.p + 1) if rule is None else rule
        X = VERTS[a][None, :] + st[:, 0:1] * t1[None, :] + st[:, 1:2] * t2[None, :]
        dofs = self.face_dofs(f)
        P = self.eval(X)[dofs]
        Cu = self.eval_curl(X)[dofs]
        Pt = np.stack([P @ t1, P @ t2], axis=0)  # (2, nf, q)
        Fh = np.einsum("q,kiq,ljq->klij", wt, Pt, Pt)
        Cn = Cu @ N
        Ch = np.einsum("q,iq,jq->ij", wt, Cn, Cn)
        return dofs, Fh, Ch

    def face_dofs(self, f):
        """Local DOF indices whose tangential trace lives on local face f, in the
        order: the face's edges (ab, ac, bc) x p, then the face's own DOFs."""
        p = self.p
        out = []
        for e in FACE_EDGES[f]:
            out += [e * p + k for k in range(p)]
        nfd = p * (p - 1)
        out += [6 * p + f * nfd + k for k in range(nfd)]
        return np.array(out, dtype=np.int64)


def _levi(i, j, k):
    return int(np.sign((j - i) * (k - i) * (k - j))) if len({i, j, k}) == 3 else 0
