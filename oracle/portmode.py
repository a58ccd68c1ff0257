"""Port modes computed on the port's own faces (oracle; test infrastructure only).

The reference drives every port with the mode its 2D solver finds on the port's
cross-section: OpenParEM3D writes the port faces out as a 2D mesh, spawns
OpenParEM2D (src/OpenParEM3D/port.cpp:5081-5176), reads back the modal fields
and metrics (load_modeMetrics, port.cpp:5302-5453) and interpolates the fields
onto the 3D port trace (Mode::fillX, port.cpp:3234-3341).  This module restates
that chain for one mode per port:

* the 2D mesh is the port's faces, each split into nsub x nsub similar triangles
  (nodes on shared edges are shared, so the mesh is conforming), with each
  sub-triangle's material taken from the tetrahedron that owns its face;
* the fundamental mode is the Lee-Sun-Cendes eigenpair of oracle.port2d
  (lowest-order edge elements for e_t, linear nodal e_z, PEC on the outer
  boundary), gamma = j beta;
* for propagation along the port's outward normal n (the convention of the
  analytic modes), H_t = n x (gamma e_t + grad_t e_z) / (j w mu);
* V = -int E . dl along the voltage path (composite 4-point Gauss on 16 nsub
  pieces), Pz = 1/2 int (E x H*) . n over the sub-triangles (exact rule for the
  piecewise-quadratic integrand), and where the mode gives a current path
  ("ipath", closed unless "ipath_closed" is False) I = int H . dl along it (the
  same composite rule per segment);
* Z by the mode's impedance definition ("zdef", OpenParEM2D
  Mode::calculateImpedance, src/OpenParEM2D/fem2D.cpp:1803-1824): PV
  V V* / (2 Pz*) (the default), VI V / I, PI 2 Pz / (I I*).

On unsplit port faces (nsub = 1) the mode is solved with the order-p elements
of oracle.port2d_pp, so it lies in the 3D trace space, and it follows the
reference's 2D solver further: H_t is the mu-weighted L2 projection of the
expression above onto ND_p (Hsolve), Pz integrates E_t x H_t* interpolated on
the order-(p-1) L2 triangle (Fields::calculatePz), and the 3D overlaps use the
order-p nodal rule (oracle.fem, quadrature.l2_nodal_rule).
"""
import numpy as np

from .materials import MU0, EPS0, relative_eps
from .modes import _frame
from .nd_basis import FACES
from .port2d import solve_mode, solve_mode_p2, LP2
from .port2d_pp import solve_mode_pp, ref_spaces, project_nd
from .quadrature import tri_rule, l2_nodal_rule


def port_submesh(verts, face_verts, nsub, origin, uh, vh):
    """Conforming split of the port faces.  face_verts: (F,3) global vertex ids in
    each face's local order (P0, P1, P2).  Returns nodes (N,3), xy (N,2),
    tris (T,3), tri_face (T,)."""
    n = int(nsub)
    key_id = {}
    nodes = []

    def node(key, X):
        if key not in key_id:
            key_id[key] = len(nodes)
            nodes.append(X)
        return key_id[key]

    def edge_node(ga, gb, m):   # m/n of the way from ga to gb
        if m == 0:
            return node(("v", ga), verts[ga])
        if m == n:
            return node(("v", gb), verts[gb])
        lo, hi, mm = (ga, gb, m) if ga < gb else (gb, ga, n - m)
        return node(("e", lo, hi, mm), verts[lo] + (mm / n) * (verts[hi] - verts[lo]))

    tris, tri_face = [], []
    sub = np.full((len(face_verts), n + 1, n + 1, 2), -1, dtype=np.int64)   # (face, i, j, upper) -> sub-triangle
    for f, (g0, g1, g2) in enumerate(face_verts):
        P0, P1, P2 = verts[g0], verts[g1], verts[g2]
        ids = {}
        for i in range(n + 1):
            for j in range(n + 1 - i):
                if j == 0:
                    ids[i, j] = edge_node(g0, g1, i)
                elif i == 0:
                    ids[i, j] = edge_node(g0, g2, j)
                elif i + j == n:
                    ids[i, j] = edge_node(g1, g2, j)
                else:
                    ids[i, j] = node(("f", f, i, j), P0 + (i / n) * (P1 - P0) + (j / n) * (P2 - P0))
        for i in range(n):
            for j in range(n - i):
                sub[f, i, j, 0] = len(tris)
                tris.append([ids[i, j], ids[i + 1, j], ids[i, j + 1]])
                tri_face.append(f)
                if i + j <= n - 2:
                    sub[f, i, j, 1] = len(tris)
                    tris.append([ids[i + 1, j], ids[i + 1, j + 1], ids[i, j + 1]])
                    tri_face.append(f)
    X = np.array(nodes, dtype=np.float64)
    xy = np.stack([(X - origin) @ uh, (X - origin) @ vh], axis=1)
    return X, xy, np.array(tris, dtype=np.int64), np.array(tri_face, dtype=np.int64), sub


class Fem2DMode:
    """The fundamental mode of one port on its split faces at one frequency."""

    def __init__(self, prob, topo, faces, mode, freq):
        verts = np.asarray(prob["verts"], dtype=np.float64)
        o, uh, vh, nh = _frame(mode)
        self.o, self.uh, self.vh, self.nh = o, uh, vh, nh
        fv = np.array([topo.tets[topo.face_owner[f]][list(FACES[topo.face_lface[f]])] for f in faces], dtype=np.int64)
        X, xy, tris, tri_face, self.sub = port_submesh(verts, fv, mode["nsub"], o, uh, vh)
        self.nsub = int(mode["nsub"])
        reg = np.asarray(prob["tet_region"], dtype=np.int64)[topo.face_owner[np.asarray(faces)]][tri_face]
        eps = relative_eps(freq, np.asarray(prob["eps_r"], dtype=np.float64)[reg],
                           np.asarray(prob["tand"], dtype=np.float64)[reg],
                           np.asarray(prob["sigma"], dtype=np.float64)[reg])
        mu = np.asarray(prob["mu_r"], dtype=np.float64)[reg].astype(np.complex128)
        self.order = int(mode.get("order2d", 1))
        mode_index = int(mode.get("mode_index", 0))   # 0: the fundamental mode; k: the k-th in decreasing beta^2
        # order-p edge / Lagrange elements (oracle.port2d_pp): on unsplit port faces
        # (the mode then lies in the 3D trace space), at orders above 2 and for
        # higher modes; the split faces of the earlier path keep its solvers
        if self.order >= 3 or mode_index > 0 or self.nsub == 1:
            beta, ct, cz, _ = solve_mode_pp(xy, tris, freq, eps, mu, self.order, mode_index)
            e0 = ct[:, :3 * self.order].ravel()
            big = e0[np.argmax(np.abs(e0))]
            self.ctp, self.czp = ct / big, cz / big
            self.ref = ref_spaces(self.order)
            self.pp = True
        elif self.order == 2:
            beta, ct, cz, _ = solve_mode_p2(xy, tris, freq, eps, mu)
            big = ct[:, :3].ravel()[np.argmax(np.abs(ct[:, :3]).ravel())]   # largest Whitney coefficient
            self.ct, self.cz2 = ct / big, cz / big
        else:
            beta, et, ez, edges = solve_mode(xy, tris, freq, eps, mu)
            big = et[np.argmax(np.abs(et))]
            et, ez = et / big, ez / big
        self.freq, self.beta, self.gamma = freq, beta, 1j * beta
        self.xy, self.tris, self.mu = xy, tris, mu
        self.mu_port = float(np.real(mu[0]))
        # per sub-triangle: vertex order sorted by node id, gradients, edge coefficients
        st = np.sort(tris, axis=1)
        P = xy[st]                                           # (T,3,2)
        J = np.stack([P[:, 1] - P[:, 0], P[:, 2] - P[:, 0]], axis=2)   # columns
        det = J[:, 0, 0] * J[:, 1, 1] - J[:, 0, 1] * J[:, 1, 0]
        Jinv = np.stack([np.stack([J[:, 1, 1], -J[:, 0, 1]], 1), np.stack([-J[:, 1, 0], J[:, 0, 0]], 1)], 1) / det[:, None, None]
        r = np.array([[-1.0, -1.0], [1.0, 0.0], [0.0, 1.0]])
        self.g = np.einsum("tji,kj->tki", Jinv, r)          # grad lambda_k = J^-T r_k : (T,3,2)
        self.area = 0.5 * np.abs(det)
        self.st, self.P0, self.Jinv = st, P[:, 0], Jinv
        if self.order == 1 and not getattr(self, "pp", False):
            eid = {(int(a), int(b)): e for e, (a, b) in enumerate(edges)}
            lp = [(0, 1), (0, 2), (1, 2)]
            self.ce = np.array([[et[eid[(int(t[a]), int(t[b]))]] for a, b in lp] for t in st])   # (T,3)
            self.cz = ez[st]                                     # (T,3)
            self.gz = np.einsum("tk,tki->ti", self.cz, self.g)   # grad e_z (T,2)
        self.w = 2 * np.pi * freq
        self.chp = None
        if getattr(self, "pp", False):
            # H_t as the reference's 2D solver forms it: the mu-weighted L2
            # projection of n x (gamma e_t + grad e_z) / (j w mu) onto ND_p
            def h2d(t, X2):
                _, H = self._eval(np.full(len(X2), t), X2)
                return np.stack([H @ self.uh, H @ self.vh], axis=1)
            self.chp = project_nd(xy, tris, self.order, mu, h2d)
        # metrics
        p0 = np.asarray(mode["vpath"][0], dtype=np.float64)
        p1 = np.asarray(mode["vpath"][1], dtype=np.float64)
        K = 16 * int(mode["nsub"])
        xg, wg = np.polynomial.legendre.leggauss(4)
        s = ((np.arange(K)[:, None] + 0.5 * (xg[None, :] + 1)) / K).ravel()
        ws = np.tile(0.5 * wg / K, K)
        Xp = p0[None, :] + s[:, None] * (p1 - p0)[None, :]
        self.V = -np.sum(ws * (self.Et(Xp) @ (p1 - p0)))
        if self.chp is not None:
            # the reference's Pz (Fields::calculatePz, src/OpenParEM2D/fem2D.cpp:395-480):
            # E_t x H_t* interpolated on the order-(p-1) L2 triangle and integrated
            q, wq = l2_nodal_rule(self.order - 1)
        else:
            q, wq = tri_rule(max(4, 2 * self.order))   # exact for the degree-2p integrand
        T, nq = len(st), len(wq)
        tt = np.repeat(np.arange(T), nq)
        X2 = (self.P0[tt] + np.tile(q[:, 0], T)[:, None] * (P[tt, 1] - P[tt, 0])
              + np.tile(q[:, 1], T)[:, None] * (P[tt, 2] - P[tt, 0]))
        E, H = self._eval(tt, X2)
        # weights sum to 1/2 on the unit triangle: int = 2 area sum(w f)
        self.Pz = 0.5 * np.sum(2 * self.area[tt] * np.tile(wq, T) * (np.cross(E, np.conj(H)) @ nh))
        self.I = 0j
        ip = mode.get("ipath")
        if ip is not None:
            ip = np.asarray(ip, dtype=np.float64).reshape(-1, 3)
            nseg = len(ip) if mode.get("ipath_closed", True) else len(ip) - 1
            for k in range(nseg):
                a, b = ip[k], ip[(k + 1) % len(ip)]
                self.I += np.sum(ws * (self.Ht(a[None, :] + s[:, None] * (b - a)[None, :]) @ (b - a)))
        zdef = mode.get("zdef", "PV")
        if zdef == "VI":
            self.Z = self.V / self.I
        elif zdef == "PI":
            self.Z = 2 * self.Pz / (self.I * np.conj(self.I))
        else:
            self.Z = 0.5 * self.V * np.conj(self.V) / np.conj(self.Pz)

    def _locate(self, X2):
        """Sub-triangle of each 2D point: the one it is deepest inside."""
        out = np.empty(len(X2), dtype=np.int64)
        for c in range(0, len(X2), 256):
            d = X2[c:c + 256, None, :] - self.P0[None, :, :]            # (p,T,2)
            lam = np.einsum("tij,ptj->pti", self.Jinv, d)              # (p,T,2): lambda_1, lambda_2
            l0 = 1 - lam[..., 0] - lam[..., 1]
            out[c:c + 256] = np.argmax(np.minimum(l0, np.minimum(lam[..., 0], lam[..., 1])), axis=1)
        return out

    def _eval(self, t, X2):
        d = X2 - self.P0[t]
        lam12 = np.einsum("pij,pj->pi", self.Jinv[t], d)
        lam = np.stack([1 - lam12[:, 0] - lam12[:, 1], lam12[:, 0], lam12[:, 1]], axis=1)   # (p,3)
        g = self.g[t]                                               # (p,3,2)
        e2 = np.zeros((len(t), 2), dtype=np.complex128)
        if getattr(self, "pp", False):
            Nh, _ = self.ref.nd(lam12)                              # reference coordinates = (lambda_1, lambda_2)
            _, gLh = self.ref.h1(lam12)
            JiT = np.transpose(self.Jinv[t], (0, 2, 1))
            e2 = np.einsum("pij,pj->pi", JiT, np.einsum("pn,pni->pi", self.ctp[t], Nh))
            gz = np.einsum("pij,pj->pi", JiT, np.einsum("pl,pli->pi", self.czp[t], gLh))
            if self.chp is not None:
                h2 = np.einsum("pij,pj->pi", JiT, np.einsum("pn,pni->pi", self.chp[t], Nh))
                E = e2[:, 0:1] * self.uh[None, :] + e2[:, 1:2] * self.vh[None, :]
                return E, h2[:, 0:1] * self.uh[None, :] + h2[:, 1:2] * self.vh[None, :]
        elif self.order == 2:
            gz = np.zeros((len(t), 2), dtype=np.complex128)
            for i, (a, b) in enumerate(LP2):
                W = lam[:, a:a + 1] * g[:, b] - lam[:, b:b + 1] * g[:, a]
                Gr = lam[:, a:a + 1] * g[:, b] + lam[:, b:b + 1] * g[:, a]
                e2 += self.ct[t, i][:, None] * W + self.ct[t, 3 + i][:, None] * Gr
                gz += self.cz2[t, 3 + i][:, None] * Gr
            for k, (c, (a, b)) in enumerate(((2, (0, 1)), (0, (1, 2)))):
                W = lam[:, a:a + 1] * g[:, b] - lam[:, b:b + 1] * g[:, a]
                e2 += self.ct[t, 6 + k][:, None] * lam[:, c:c + 1] * W
            for k in range(3):
                gz += self.cz2[t, k][:, None] * g[:, k]
        else:
            for i, (a, b) in enumerate([(0, 1), (0, 2), (1, 2)]):
                Ni = lam[:, a:a + 1] * g[:, b] - lam[:, b:b + 1] * g[:, a]
                e2 += self.ce[t, i][:, None] * Ni
            gz = self.gz[t]
        E = e2[:, 0:1] * self.uh[None, :] + e2[:, 1:2] * self.vh[None, :]
        G = self.gamma * e2 + gz
        G3 = G[:, 0:1] * self.uh[None, :] + G[:, 1:2] * self.vh[None, :]
        H = np.cross(self.nh[None, :], G3) / (1j * self.w * MU0 * self.mu[t][:, None])
        return E, H

    def _xy(self, X):
        X = np.atleast_2d(np.asarray(X, dtype=np.float64))
        return np.stack([(X - self.o) @ self.uh, (X - self.o) @ self.vh], axis=1)

    def Et(self, X):
        X2 = self._xy(X)
        return self._eval(self._locate(X2), X2)[0]

    def Ht(self, X):
        X2 = self._xy(X)
        return self._eval(self._locate(X2), X2)[1]

    def face_tri(self, f, S12):
        """Sub-triangle of port face f holding the points of face parameters
        S12 = (s1, s2): cell (i, j) of the split, its upper half when the
        fractional parts add up to more than one."""
        n = self.nsub
        s1, s2 = S12[:, 0], S12[:, 1]
        i = np.minimum(np.floor(n * np.maximum(0.0, s1)).astype(np.int64), n - 1)
        j = np.minimum(np.floor(n * np.maximum(0.0, s2)).astype(np.int64), n - 1 - i)
        up = ((n * s1 - i) + (n * s2 - j) > 1.0) & (i + j <= n - 2)
        return self.sub[f, i, j, up.astype(np.int64)]

    def metrics(self):
        mode = self

        class _Field:
            def __init__(self, which):
                self.which = which
                self.nsub = mode.nsub

            def __call__(self, X):
                X2 = mode._xy(X)
                return mode._eval(mode._locate(X2), X2)[self.which]

            def at_face(self, f, S12, X):
                return mode._eval(mode.face_tri(f, S12), mode._xy(X))[self.which]

        # unsplit faces: the mode lies in the 3D trace space and the overlaps follow
        # the reference's nodal rule (oracle.fem)
        return {"gamma": self.gamma, "Z": self.Z, "V": self.V, "Pz": self.Pz, "I": self.I, "Et": _Field(0),
                "Ht": _Field(1), "nodal": self.chp is not None and self.nsub == 1}
