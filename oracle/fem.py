"""FP64 CPU restatement of OpenParEM3D's per-frequency solve stage (oracle).

TEST INFRASTRUCTURE: used by tests/, smoke() and bench.py's CPU legs only.

Problem dictionary (the same fields the C ABI takes):
  verts (nv,3) m, tets (ne,4), tet_region (ne,), bdr_tris (nb,3), bdr_attr (nb,)
  order p
  region arrays eps_r, tand, sigma, mu_r  (indexed by tet_region)
  boundaries: {attr: {"type": "pec"|"pmc"|"port"|"impedance"|"radiation", ...}}
     port:       {"port": k}
     impedance:  {"sigma": S/m, "Rz": m, "mu_r": 1}
     radiation:  {"wave_impedance": ohm (default sqrt(mu0/eps0))}
  ports: list of {"mode": dict} (one mode per port, the "single" driving set)
"""
import numpy as np
import scipy.sparse as sp
import scipy.sparse.linalg as spla

from .nd_basis import NDBasis, EDGES, FACES, ndofs
from .quadrature import line_rule, tri_rule, l2_nodal_rule
from . import materials, modes

EPS0 = materials.EPS0
MU0 = materials.MU0

_BASIS_CACHE = {}


def basis(p):
    if p not in _BASIS_CACHE:
        B = NDBasis(p)
        Mh, Kh, Qh = B.reference_tensors()
        faces = [B.face_tensors(f) for f in range(4)]
        _BASIS_CACHE[p] = (B, Mh, Kh, Qh, faces)
    return _BASIS_CACHE[p]


# --------------------------------------------------------------------------
# topology and DOF numbering   (replaces MFEM ND_FECollection numbering,
# src/OpenParEM3D/fem3D.cpp:65-66)
# --------------------------------------------------------------------------
class Topology:
    def __init__(self, prob):
        p = prob["order"]
        self.p = p
        tets = np.sort(np.asarray(prob["tets"], dtype=np.int64), axis=1)
        self.tets = tets
        ne = len(tets)
        ep = np.array(EDGES)
        fp = np.array(FACES)
        e_all = tets[:, ep].reshape(-1, 2)
        ekey = e_all[:, 0] * (tets.max() + 1) + e_all[:, 1]
        uk, einv = np.unique(ekey, return_inverse=True)
        self.nE = len(uk)
        self.tet_edges = einv.reshape(ne, 6)
        nv1 = tets.max() + 1
        f_all = tets[:, fp].reshape(-1, 3)
        fkey = (f_all[:, 0] * nv1 + f_all[:, 1]) * nv1 + f_all[:, 2]
        ufk, finv = np.unique(fkey, return_inverse=True)
        self.nF = len(ufk)
        self.tet_faces = finv.reshape(ne, 4)
        self._fkey_sorted = ufk
        self._nv1 = nv1
        nd = ndofs(p)
        ne_d, nf_d, ni_d = nd["edge"], nd["face"], nd["interior"]
        self.ld = nd["local"]
        dof = np.zeros((ne, self.ld), dtype=np.int64)
        c = 0
        for le in range(6):
            for k in range(ne_d):
                dof[:, c] = self.tet_edges[:, le] * ne_d + k; c += 1
        base_f = self.nE * ne_d
        for lf in range(4):
            for k in range(nf_d):
                dof[:, c] = base_f + self.tet_faces[:, lf] * nf_d + k; c += 1
        base_i = base_f + self.nF * nf_d
        for k in range(ni_d):
            dof[:, c] = base_i + np.arange(ne) * ni_d + k; c += 1
        self.dof = dof
        self.n = base_i + ne * ni_d
        # face -> (tet, local face) for one adjacent tet
        owner = np.full(self.nF, -1, dtype=np.int64)
        lface = np.full(self.nF, -1, dtype=np.int64)
        fl = self.tet_faces.ravel()
        owner[fl] = np.repeat(np.arange(ne), 4)
        lface[fl] = np.tile(np.arange(4), ne)
        self.face_owner = owner
        self.face_lface = lface
        # boundary triangles -> global face id
        bt = np.sort(np.asarray(prob["bdr_tris"], dtype=np.int64).reshape(-1, 3), axis=1)
        bkey = (bt[:, 0] * nv1 + bt[:, 1]) * nv1 + bt[:, 2]
        pos = np.searchsorted(ufk, bkey)
        assert np.all(ufk[np.minimum(pos, len(ufk) - 1)] == bkey), "boundary triangle is not a mesh face"
        self.bdr_face = pos
        self.bdr_tris_sorted = bt

    def face_global_dofs(self, faces):
        """Global DOFs of the tangential trace on each face (nfaces, p(p+2))."""
        B = basis(self.p)[0]
        out = []
        for f in faces:
            t, lf = self.face_owner[f], self.face_lface[f]
            out.append(self.dof[t, B.face_dofs(lf)])
        return np.array(out, dtype=np.int64).reshape(len(faces), -1)


# --------------------------------------------------------------------------
# element matrices (CurlCurlIntegrator / VectorFEMassIntegrator /
# MixedVectorCurlIntegrator restated, src/OpenParEM3D/fem3D.cpp:115-123,195-216)
# --------------------------------------------------------------------------
def element_geometry(verts, tets_sorted):
    P = verts[tets_sorted]                       # (ne,4,3)
    J = np.stack([P[:, 1] - P[:, 0], P[:, 2] - P[:, 0], P[:, 3] - P[:, 0]], axis=2)  # columns
    det = np.linalg.det(J)
    Ji = np.linalg.inv(J)
    G = Ji @ np.transpose(Ji, (0, 2, 1))          # J^-1 J^-T
    C = np.transpose(J, (0, 2, 1)) @ J            # J^T J
    return J, det, G, C


def element_matrices(prob, topo):
    B, Mh, Kh, Qh, _ = basis(topo.p)
    verts = np.asarray(prob["verts"], dtype=np.float64)
    _, det, G, C = element_geometry(verts, topo.tets)
    ad = np.abs(det)
    Me = np.einsum("e,eab,abij->eij", ad, G, Mh)
    Ke = np.einsum("e,eab,abij->eij", 1.0 / ad, C, Kh)
    Qe = np.sign(det)[:, None, None] * Qh[None]
    return Me, Ke, Qe


def nodal_face_tables(p):
    """Face tables of basis(p) with the port integrals' nodal rule
    (quadrature.l2_nodal_rule(p)) in place of exact integration."""
    key = ("nodal", p)
    if key not in _BASIS_CACHE:
        B = basis(p)[0]
        rule = l2_nodal_rule(p)
        _BASIS_CACHE[key] = [B.face_tensors(f, rule) for f in range(4)]
    return _BASIS_CACHE[key]


def face_matrices(prob, topo, faces, nodal=False):
    """(dofs, Bm, Bcc) for boundary faces: tangential mass and surface curl-curl
    (Bm with the port integrals' nodal rule when nodal is set)."""
    B, _, _, _, ftabs = basis(topo.p)
    if nodal:
        ftabs = nodal_face_tables(topo.p)
    verts = np.asarray(prob["verts"], dtype=np.float64)
    dofs, Bm, Bcc = [], [], []
    for f in faces:
        t, lf = topo.face_owner[f], topo.face_lface[f]
        a, b, c = FACES[lf]
        Pv = verts[topo.tets[t]]
        t1 = Pv[b] - Pv[a]; t2 = Pv[c] - Pv[a]
        g = np.array([[t1 @ t1, t1 @ t2], [t2 @ t1, t2 @ t2]])
        gi = np.linalg.inv(g)
        A2 = np.linalg.norm(np.cross(t1, t2))
        ldofs, Fh, Ch = ftabs[lf]
        Bm.append(A2 * np.einsum("kl,klij->ij", gi, Fh))
        Bcc.append(Ch / A2)
        dofs.append(topo.dof[t, ldofs])
    return np.array(dofs), np.array(Bm), np.array(Bcc)


def _coo(n, dofs, mats, weights=None):
    if weights is not None:
        mats = mats * weights[:, None, None]
    ld = dofs.shape[1]
    r = np.repeat(dofs, ld, axis=1).ravel()
    c = np.tile(dofs, (1, ld)).ravel()
    return sp.csr_matrix((mats.ravel(), (r, c)), shape=(n, n))


class Operators:
    """Frequency-independent real operators on the shared pattern."""

    def __init__(self, prob):
        self.prob = prob
        topo = Topology(prob)
        self.topo = topo
        n = topo.n
        reg = np.asarray(prob["tet_region"], dtype=np.int64)
        eps_r = np.asarray(prob["eps_r"], dtype=np.float64)[reg]
        tand = np.asarray(prob["tand"], dtype=np.float64)[reg]
        sigma = np.asarray(prob["sigma"], dtype=np.float64)[reg]
        mu_r = np.asarray(prob["mu_r"], dtype=np.float64)[reg]
        Me, Ke, Qe = element_matrices(prob, topo)
        d = topo.dof
        self.K = _coo(n, d, Ke, 1.0 / mu_r)
        self.M_eps = _coo(n, d, Me, eps_r)
        self.M_tand = _coo(n, d, Me, eps_r * tand)
        self.M_sig = _coo(n, d, Me, sigma)
        self.M1 = _coo(n, d, Me)
        self.Q_mu = _coo(n, d, Qe, 1.0 / mu_r)
        # boundaries
        battr = np.asarray(prob["bdr_attr"], dtype=np.int64)
        bnd = prob["boundaries"]
        self.pec_faces = topo.bdr_face[np.isin(battr, [a for a, v in bnd.items() if v["type"] == "pec"])]
        self.port_faces = {}
        self.imp = []       # (kind, spec, matrix)
        reg_of_face = reg[topo.face_owner]
        for attr, spec in bnd.items():
            faces = topo.bdr_face[battr == attr]
            if spec["type"] == "port":
                self.port_faces.setdefault(spec["port"], []).extend(faces.tolist())
            elif spec["type"] in ("impedance", "radiation"):
                fd, Bm, _ = face_matrices(prob, topo, faces)
                self.imp.append((spec, _coo(n, fd, Bm)))
        self.ports = []
        for k in range(len(prob["ports"])):
            faces = np.array(sorted(self.port_faces.get(k, [])), dtype=np.int64)
            fd, Bm, Bcc = face_matrices(prob, topo, faces)
            _, Bmn, _ = face_matrices(prob, topo, faces, nodal=True)
            rf = reg_of_face[faces]
            w_mu = 1.0 / np.asarray(prob["mu_r"], dtype=np.float64)[rf]
            w_eps = np.asarray(prob["eps_r"], dtype=np.float64)[rf]
            w_tand = w_eps * np.asarray(prob["tand"], dtype=np.float64)[rf]
            w_sig = np.asarray(prob["sigma"], dtype=np.float64)[rf]
            self.ports.append({
                "faces": faces,
                "dofs": np.unique(fd),
                "Bcc": _coo(n, fd, Bcc, w_mu),
                "Bm_eps": _coo(n, fd, Bm, w_eps),
                "Bm_tand": _coo(n, fd, Bm, w_tand),
                "Bm_sig": _coo(n, fd, Bm, w_sig),
                "Bm1": _coo(n, fd, Bm),
                # the reference's overlap integrals (tangentialInnerProduct,
                # port.cpp:3463-3490): the product interpolated at the nodes of the
                # order-p L2 triangle and integrated, i.e. the nodal rule
                "Bm1n": _coo(n, fd, Bmn),
                "region": int(reg_of_face[faces[0]]) if len(faces) else 0,
            })
        self.pec_dofs = np.unique(topo.face_global_dofs(self.pec_faces)) if len(self.pec_faces) else np.zeros(0, np.int64)

    # ---------------------------------------------------------------------
    def port_trace(self, k, field):
        """Interpolate a tangential field on port k into its trace DOFs
        (the role of Mode::fillX / 2D->3D transfer, src/OpenParEM3D/port.cpp:3234-3341,
        applied to the mode's field).  ``field(X) -> (npts,3) complex``."""
        topo = self.topo
        p = topo.p
        verts = np.asarray(self.prob["verts"], dtype=np.float64)
        x = np.zeros(topo.n, dtype=np.complex128)
        B = basis(p)[0]
        s, ws = line_rule(2 * p + 4)
        from .nd_basis import shifted_legendre, tri_test_polys, monomials2
        L = np.array([shifted_legendre(k_, s) for k_ in range(p)])  # (p, q)
        if p >= 2:
            st, wt = tri_rule(2 * p + 4)
            M2 = monomials2(p - 2)
            Q2 = ((st[:, 0:1] ** M2[None, :, 0]) * (st[:, 1:2] ** M2[None, :, 1])) @ tri_test_polys(p - 2).T
        # A field known per port face (a 2D mode, linear on each sub-triangle of
        # the face's nsub x nsub split) is evaluated on the face being traced,
        # with the rules applied cell by cell.  The two faces of an edge inside
        # the port give its edge moments as their mean (equal for a continuous
        # field; a 2D mode's H_t, a normal component of an edge-element field,
        # jumps between cells).
        at_face = getattr(field, "at_face", None)
        if at_face is not None:
            N = field.nsub
            sp = ((np.arange(N)[:, None] + s[None, :]) / N).ravel()
            wsp = np.tile(ws / N, N)
            Lc = np.array([shifted_legendre(k_, sp) for k_ in range(p)])
            zero = np.zeros_like(sp)
            edge_par = (np.stack([sp, zero], 1), np.stack([zero, sp], 1), np.stack([1 - sp, sp], 1))
            if p >= 2:
                cells = [(i, j, up) for i in range(N) for j in range(N - i) for up in (0, 1)
                         if not (up and i + j > N - 2)]
                A1 = np.concatenate([((i + 1 - st[:, 0]) if up else (i + st[:, 0])) / N for i, j, up in cells])
                A2 = np.concatenate([((j + 1 - st[:, 1]) if up else (j + st[:, 1])) / N for i, j, up in cells])
                wc = np.tile(wt / N ** 2, len(cells))
                Qc = ((A1[:, None] ** M2[None, :, 0]) * (A2[:, None] ** M2[None, :, 1])) @ tri_test_polys(p - 2).T
        cnt = np.zeros(topo.n)
        for fi, f in enumerate(self.ports[k]["faces"]):
            t, lf = topo.face_owner[f], topo.face_lface[f]
            a, b, c = FACES[lf]
            Pv = verts[topo.tets[t]]
            gd = topo.dof[t, B.face_dofs(lf)]
            vals = []
            for e, (i, j) in enumerate(((a, b), (a, c), (b, c))):
                tv = Pv[j] - Pv[i]
                if at_face is not None:
                    X = Pv[i][None, :] + sp[:, None] * tv[None, :]
                    Et = at_face(fi, edge_par[e], X) @ tv
                    vals.extend((Lc * (wsp * Et)[None, :]).sum(axis=1))
                else:
                    X = Pv[i][None, :] + s[:, None] * tv[None, :]
                    Et = field(X) @ tv
                    vals.extend((L * (ws * Et)[None, :]).sum(axis=1))
            if p >= 2:
                t1 = Pv[b] - Pv[a]; t2 = Pv[c] - Pv[a]
                if at_face is not None:
                    X = Pv[a][None, :] + A1[:, None] * t1[None, :] + A2[:, None] * t2[None, :]
                    F = at_face(fi, np.stack([A1, A2], 1), X)
                    for r in range(Qc.shape[1]):
                        for tv in (t1, t2):
                            vals.append(np.sum(wc * Qc[:, r] * (F @ tv)))
                else:
                    X = Pv[a][None, :] + st[:, 0:1] * t1[None, :] + st[:, 1:2] * t2[None, :]
                    F = field(X)
                    for r in range(Q2.shape[1]):
                        for tv in (t1, t2):
                            vals.append(np.sum(wt * Q2[:, r] * (F @ tv)))
            x[gd] += np.array(vals)
            cnt[gd] += 1
        x[cnt > 1] /= cnt[cnt > 1]
        return x


# --------------------------------------------------------------------------
def eliminate(A, dofs):
    """MatZeroRowsColumns(A, dofs, diag=1) (src/OpenParEM3D/solveComplexLinearSystem.c:61-65,129)."""
    n = A.shape[0]
    keep = np.ones(n)
    keep[dofs] = 0.0
    D = sp.diags(keep)
    I = sp.diags(1.0 - keep)
    return (D @ A @ D + I).tocsr()


def assemble_A(ops, freq, driven):
    """Complex A(omega) for driving set ``driven`` (0-based driven port),
    src/OpenParEM3D/fem3D.cpp:103-190 with port.cpp:5783-5875 and port.cpp:1009-1041."""
    prob = ops.prob
    w = 2 * np.pi * freq
    k0 = w * np.sqrt(MU0 * EPS0)
    A = (ops.K - k0 ** 2 * ops.M_eps + 1j * k0 ** 2 * ops.M_tand + 1j * w * MU0 * ops.M_sig).astype(np.complex128)
    for k, port in enumerate(ops.ports):
        if k == driven:
            continue
        g = robin_gamma(ops, k, freq)
        A = A + (1.0 / g) * port["Bcc"] + (1.0 / g) * (-k0 ** 2 * port["Bm_eps"] + 1j * k0 ** 2 * port["Bm_tand"]
                                                      + 1j * w * MU0 * port["Bm_sig"])
    for spec, Bm in ops.imp:
        if spec["type"] == "impedance":
            Rs = materials.surface_resistance(freq, spec["sigma"], spec.get("mu_r", 1.0), spec.get("Rz", 0.0))
        else:
            Rs = spec.get("wave_impedance", np.sqrt(MU0 / EPS0))
        A = A + 1j * (w * MU0 / Rs) * Bm
    return A.tocsr()


def port_mode(ops, k, freq):
    prob = ops.prob
    port = ops.ports[k]
    mode = prob["ports"][k]["mode"]
    if mode.get("kind") == "FEM2D":
        # the port's own 2D eigenmode (oracle.portmode), cached per frequency
        cache = ops.__dict__.setdefault("_fem2d", {})
        if (k, freq) not in cache:
            from .portmode import Fem2DMode
            cache[(k, freq)] = Fem2DMode(prob, ops.topo, port["faces"], mode, freq).metrics()
        return cache[(k, freq)]
    r = port["region"]
    eps_c = materials.relative_eps(freq, prob["eps_r"][r], prob["tand"][r], prob["sigma"][r])
    return modes.mode_metrics(prob["ports"][k]["mode"], freq, eps_c, prob["mu_r"][r])


def sports(prob):
    """The S-ports: (port, extra) pairs, every port's first mode in port order,
    then the further modes of ports driven by their own 2D modes ("extra_modes"
    of the port's mode: dicts with "index" (mode number in decreasing beta^2),
    "vpath" and optionally "zdef", "ipath", "ipath_closed"), in port order."""
    out = [(k, None) for k in range(len(prob["ports"]))]
    for k, p in enumerate(prob["ports"]):
        for x in p["mode"].get("extra_modes", ()):
            out.append((k, x))
    return out


def sport_mode(ops, s, freq):
    """Metrics of S-port s (sports order) at freq."""
    k, x = sports(ops.prob)[s]
    if x is None:
        return port_mode(ops, k, freq)
    cache = ops.__dict__.setdefault("_fem2d_x", {})
    if (s, freq) not in cache:
        from .portmode import Fem2DMode
        mode = dict(ops.prob["ports"][k]["mode"])
        mode.pop("extra_modes", None)
        mode.update(mode_index=int(x["index"]), vpath=x["vpath"], zdef=x.get("zdef", "PV"))
        mode.pop("ipath", None)
        if x.get("ipath") is not None:
            mode.update(ipath=x["ipath"], ipath_closed=x.get("ipath_closed", True))
        cache[(s, freq)] = Fem2DMode(ops.prob, ops.topo, ops.ports[k]["faces"], mode, freq).metrics()
    return cache[(s, freq)]


def robin_gamma(ops, k, freq):
    """gamma of port k's absorbing condition when another port drives: with
    several modes on the port, the one of largest |gamma| (Port::addPortIntegrators,
    src/OpenParEM3D/port.cpp:5790-5806, "to avoid passivity violations")."""
    g = port_mode(ops, k, freq)["gamma"]
    for s, (q, x) in enumerate(sports(ops.prob)):
        if x is not None and q == k:
            gx = sport_mode(ops, s, freq)["gamma"]
            if abs(gx) > abs(g):
                g = gx
    return g


def solve_frequency(ops, freq, return_fields=False, reciprocal=True):
    """One frequency point: every driving set, E and H, overlaps, S.
    Mirrors the driving-set loop src/OpenParEM3D/OpenParEM3D.cpp:497-566; a port
    with several modes contributes one S-port (and one driving set) per mode."""
    topo = ops.topo
    prob = ops.prob
    w = 2 * np.pi * freq
    sp_ = sports(prob)
    N = len(sp_)
    pk = [k for k, _ in sp_]
    mm = [sport_mode(ops, s, freq) for s in range(N)]
    Et = [ops.port_trace(pk[s], mm[s]["Et"]) for s in range(N)]
    Ht = [ops.port_trace(pk[s], mm[s]["Ht"]) for s in range(N)]
    Cp = np.zeros((N, N), dtype=np.complex128)   # [driving set, S-port]
    Cm = np.zeros((N, N), dtype=np.complex128)
    fields = []
    P = ops.M1.tocsc()
    # minimum degree on A+A^T (FEM matrices are structurally symmetric); the
    # mass matrix is symmetric positive definite, so no pivoting is needed
    Plu = spla.splu(P, permc_spec="MMD_AT_PLUS_A", options=dict(SymmetricMode=True, DiagPivotThresh=0.0))
    for d in range(N):
        A = assemble_A(ops, freq, pk[d])
        A = eliminate(A, ops.pec_dofs)
        x0 = np.zeros(topo.n, dtype=np.complex128)
        pd = ops.ports[pk[d]]["dofs"]
        x0[pd] = Et[d][pd]
        b = -(A @ x0)
        b[pd] = x0[pd]
        A = eliminate(A, pd)
        # threshold partial pivoting (0.1) keeps the minimum-degree order: without it the
        # lossy ND6 systems fill in 3x and factor 9x slower, at the same residual
        e = spla.splu(A.tocsc(), permc_spec="MMD_AT_PLUS_A", options=dict(DiagPivotThresh=0.1)).solve(b)
        qe = (ops.Q_mu @ e) / (w * MU0)
        h = 1j * (Plu.solve(qe.real) + 1j * Plu.solve(qe.imag))
        for k in range(N):
            # ports driven by their own 2D mode carry it exactly in the trace space:
            # their overlaps follow the reference's rule; analytic modes are
            # integrated exactly
            Bm = ops.ports[pk[k]]["Bm1n" if mm[k].get("nodal") else "Bm1"]
            e0 = np.vdot(Et[k], Bm @ e)
            e2 = np.vdot(Et[k], Bm @ Et[k])
            h0 = np.vdot(Ht[k], Bm @ h)
            h2 = np.vdot(Ht[k], Bm @ Ht[k])
            Cp[d, k] = 0.5 * (e0 / e2 + h0 / h2)
            Cm[d, k] = 0.5 * (e0 / e2 - h0 / h2)
        if return_fields:
            fields.append((e, h))
    S = s_matrix(Cp, Cm, [m["V"] for m in mm], [m["Z"] for m in mm])
    if reciprocal:
        S = 0.5 * (S + S.T)
    out = {"S": S, "Cp": Cp, "Cm": Cm, "Z": np.array([m["Z"] for m in mm])}
    if return_fields:
        out["fields"] = fields
    return out


def s_matrix(Cp, Cm, V, Z):
    """BoundaryDatabase::calculateS (src/OpenParEM3D/port.cpp:7499-7606): a S = b."""
    N = Cp.shape[0]
    a = np.zeros((N * N, N * N), dtype=np.complex128)
    b = np.zeros(N * N, dtype=np.complex128)
    s = np.array(V) / np.sqrt(np.array(Z, dtype=np.complex128))
    for i in range(N):
        for j in range(N):
            b[i * N + j] = Cp[i, j] * s[j]
            for k in range(N):
                a[i * N + j, j * N + k] = Cm[i, k] * s[k]
    return np.linalg.solve(a, b).reshape(N, N)
