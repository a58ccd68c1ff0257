"""Host-side mirror of OpenParEM3D's per-frequency solve interface.

``Fem3D`` plays the role of the reference's ``fem3D`` object for one mesh
(src/OpenParEM3D/fem3D.hpp:70-192): ``build_fe_spaces``/``assemble`` set up
the Nedelec space and operators, ``solve`` runs one frequency over every
driving set (fem3D::solve + Mode::calculateSplits + BoundaryDatabase::calculateS),
and ``fields`` returns the E and H DOF vectors.  Everything runs through the
C ABI of libopem_b200.so on one CUDA device; errors raise ``OpemError``
carrying the ABI status code, the way the reference returns a PetscErrorCode
or ``true`` on failure.
"""
import ctypes as C
import weakref

import numpy as np
import scipy.sparse as sp

from . import _lib
from ._lib import SolverOpts, SolveStats


class OpemError(RuntimeError):
    def __init__(self, code, msg):
        super().__init__(f"{_lib.ERROR_NAMES.get(code, code)}: {msg}")
        self.code = code


def _dp(a):
    return a.ctypes.data_as(_lib.DP)


def _chk(ctx, rc, what):
    if rc != _lib.OK:
        msg = _lib.lib().opem_context_last_error(ctx).decode() if ctx else ""
        raise OpemError(rc, f"{what}: {msg}")


class Context:
    """One CUDA device + stream (opem_context)."""

    def __init__(self, device=0):
        self.h = C.c_void_p()
        self._problems = weakref.WeakSet()   # problems created on this context
        rc = _lib.lib().opem_context_create(int(device), C.byref(self.h))
        if rc != _lib.OK:
            raise OpemError(rc, "opem_context_create")

    def close(self):
        """Destroys the context; problems created on it are closed first (a
        problem must not outlive its context)."""
        if self.h:
            for F in list(getattr(self, "_problems", ())):
                F.close()
            _lib.lib().opem_context_destroy(self.h)
            self.h = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def default_opts(**kw):
    o = SolverOpts()
    _lib.lib().opem_default_opts(C.byref(o))
    for k, v in kw.items():
        if not hasattr(o, k):
            raise KeyError(k)
        setattr(o, k, v)
    return o


def te_descriptor(mode):
    """Pack a rectangular TE_mn mode dict into the ABI's 22 doubles."""
    d = np.zeros(22)
    d[0:3] = mode["origin"]; d[3:6] = mode["u"]; d[6:9] = mode["v"]; d[9:12] = mode["normal"]
    d[12] = mode.get("a", 0.0); d[13] = mode.get("b", 0.0); d[14] = mode.get("m", 0); d[15] = mode.get("n", 0)
    d[16:19] = mode["vpath"][0]; d[19:22] = mode["vpath"][1]
    return d


_BTYPES = {"pec": _lib.BDR_PEC, "pmc": _lib.BDR_PMC, "port": _lib.BDR_PORT, "impedance": _lib.BDR_IMPEDANCE,
           "radiation": _lib.BDR_RADIATION}


def project_info(proj_path, order=0):
    """Host-only reading of an OpenParEM3D project (opem_project_info) -> (counts, freqs)."""
    a = np.zeros(10, dtype=np.int64)
    fr = np.zeros(4096)
    msg = C.create_string_buffer(512)
    rc = _lib.lib().opem_project_info(str(proj_path).encode(), int(order), a.ctypes.data_as(_lib.I64P), 10, _dp(fr),
                                      len(fr), msg, 512)
    if rc != _lib.OK:
        raise OpemError(rc, f"opem_project_info: {msg.value.decode()}")
    keys = ["vertices", "tets", "regions", "exterior_faces", "port_faces", "boundary_faces", "pec_faces", "ports",
            "frequencies", "order"]
    info = dict(zip(keys, (int(v) for v in a)))
    return info, fr[:min(info["frequencies"], len(fr))]


_ZDEF = {"PV": 0, "VI": 1, "PI": 2}


def port_mode_faces_z(verts, face_verts, eps_face, mode, nsub, freq, zdef="PV", ipath=None, closed=True,
                      mu_face=None, order=2, mode_index=0):
    """The 2D mode's metrics under an impedance definition (opem_port_mode_faces_z,
    host only): zdef "PV" | "VI" | "PI", ipath (k, 3) the current path's points,
    mode_index the mode in decreasing beta^2 (0: the fundamental) ->
    {gamma, Z, V, Pz, I}."""
    verts = np.ascontiguousarray(verts, dtype=np.float64)
    fv = np.ascontiguousarray(face_verts, dtype=np.int64)
    eps = np.ascontiguousarray(np.stack([np.real(eps_face), np.imag(eps_face)], axis=1), dtype=np.float64)
    mu = None if mu_face is None else np.ascontiguousarray(np.stack([np.real(mu_face), np.imag(mu_face)], axis=1))
    d = te_descriptor(mode)
    ip = None if ipath is None else np.ascontiguousarray(ipath, dtype=np.float64).reshape(-1, 3)
    m = np.zeros(10)
    rc = _lib.lib().opem_port_mode_faces_z(len(verts), _dp(verts), len(fv), fv.ctypes.data_as(_lib.I64P), _dp(eps),
                                           None if mu is None else _dp(mu), _dp(d), int(nsub), int(order),
                                           float(freq), _ZDEF[zdef], 0 if ip is None else len(ip),
                                           None if ip is None else _dp(ip), int(closed), int(mode_index), _dp(m))
    if rc != _lib.OK:
        raise OpemError(rc, "opem_port_mode_faces_z")
    c = m[0::2] + 1j * m[1::2]
    return {"gamma": c[0], "Z": c[1], "V": c[2], "Pz": c[3], "I": c[4]}


def port_mode_faces(verts, face_verts, eps_face, mode, nsub, freq, pt_face=None, pt_s=None, mu_face=None, order=1):
    """The 2D mode of a port given by its faces (opem_port_mode_faces, host only):
    -> (metrics {gamma, Z, V, Pz}, E_t (npts,3), H_t / y (npts,3)) at the points
    (pt_face, pt_s = (s1, s2) face parameters)."""
    verts = np.ascontiguousarray(verts, dtype=np.float64)
    fv = np.ascontiguousarray(face_verts, dtype=np.int64)
    eps = np.ascontiguousarray(np.stack([np.real(eps_face), np.imag(eps_face)], axis=1), dtype=np.float64)
    mu = None if mu_face is None else np.ascontiguousarray(np.stack([np.real(mu_face), np.imag(mu_face)], axis=1))
    d = te_descriptor(mode)
    npts = 0 if pt_face is None else len(pt_face)
    pf = np.ascontiguousarray(pt_face if npts else np.zeros(1), dtype=np.int64)
    ps = np.ascontiguousarray(pt_s if npts else np.zeros((1, 2)), dtype=np.float64)
    m = np.zeros(8)
    E = np.zeros((max(npts, 1), 6))
    Hy = np.zeros((max(npts, 1), 6))
    rc = _lib.lib().opem_port_mode_faces(len(verts), _dp(verts), len(fv), fv.ctypes.data_as(_lib.I64P), _dp(eps),
                                         None if mu is None else _dp(mu), _dp(d), int(nsub), int(order), float(freq),
                                         _dp(m),
                                         npts, pf.ctypes.data_as(_lib.I64P), _dp(ps), _dp(E), _dp(Hy))
    if rc != _lib.OK:
        raise OpemError(rc, "opem_port_mode_faces")
    c = m[0::2] + 1j * m[1::2]
    E = (E[:, 0::2] + 1j * E[:, 1::2])[:npts]
    Hy = (Hy[:, 0::2] + 1j * Hy[:, 1::2])[:npts]
    return {"gamma": c[0], "Z": c[1], "V": c[2], "Pz": c[3]}, E, Hy


def project_problem(proj_path, order=0):
    """An OpenParEM3D project read on the host (opem_project_read) as a problem
    dict (the format of meshgen's problems, accepted by Fem3D and by the oracle)
    plus its frequency plan."""
    L = _lib.lib()
    cnt = np.zeros(8, dtype=np.int64)
    msg = C.create_string_buffer(512)
    path = str(proj_path).encode()
    nul = None
    rc = L.opem_project_read(path, int(order), cnt.ctypes.data_as(_lib.I64P), nul, nul, nul, nul, nul, nul, nul, nul,
                             nul, nul, nul, msg, 512)
    if rc != _lib.OK:
        raise OpemError(rc, f"opem_project_read: {msg.value.decode()}")
    nv, ne, nr, nf, na, npt, nq, p = (int(v) for v in cnt)
    verts = np.zeros((nv, 3)); tets = np.zeros((ne, 4), dtype=np.int64); reg = np.zeros(ne, dtype=np.int32)
    mat = np.zeros((nr, 4)); tris = np.zeros((nf, 3), dtype=np.int64); attr = np.zeros(nf, dtype=np.int32)
    bt = np.zeros(na, dtype=np.int32); bp = np.zeros((na, 3)); pd = np.zeros((max(npt, 1), 22)); fr = np.zeros(max(nq, 1))
    ns = np.zeros(max(npt, 1), dtype=np.int32)
    rc = L.opem_project_read(path, int(order), cnt.ctypes.data_as(_lib.I64P), _dp(verts), tets.ctypes.data_as(_lib.I64P),
                             reg.ctypes.data_as(_lib.I32P), _dp(mat), tris.ctypes.data_as(_lib.I64P),
                             attr.ctypes.data_as(_lib.I32P), bt.ctypes.data_as(_lib.I32P), _dp(bp), _dp(pd),
                             ns.ctypes.data_as(_lib.I32P), _dp(fr), msg, 512)
    if rc != _lib.OK:
        raise OpemError(rc, f"opem_project_read: {msg.value.decode()}")
    names = {v: k for k, v in _BTYPES.items()}
    bnd = {}
    for a in range(na):
        t = names[int(bt[a])]
        if t == "port":
            bnd[a + 1] = {"type": "port", "port": int(bp[a, 0])}
        elif t == "impedance":
            bnd[a + 1] = {"type": "impedance", "sigma": bp[a, 0], "Rz": bp[a, 1], "mu_r": bp[a, 2]}
        elif t == "radiation":
            bnd[a + 1] = {"type": "radiation", "wave_impedance": bp[a, 0]}
        else:
            bnd[a + 1] = {"type": t}
    ports = []
    for k in range(npt):
        d = pd[k]
        mode = {"kind": "TE", "m": int(d[14]), "n": int(d[15]), "a": d[12], "b": d[13],
                "origin": d[0:3].tolist(), "u": d[3:6].tolist(), "v": d[6:9].tolist(),
                "normal": d[9:12].tolist(), "vpath": (d[16:19].tolist(), d[19:22].tolist())}
        if ns[k] > 0:   # the port's own 2D mode (the reader: 2D elements of the problem's order)
            mode.update(kind="FEM2D", nsub=int(ns[k]), order2d=min(8, int(p)))
            zd, cl, npth = C.c_int(0), C.c_int(1), C.c_int(0)
            pbuf = np.zeros((64, 3))
            rc = L.opem_project_port_impedance(path, k, C.byref(zd), C.byref(cl), C.byref(npth), _dp(pbuf), 64, msg,
                                               512)
            if rc != _lib.OK:
                raise OpemError(rc, f"opem_project_port_impedance: {msg.value.decode()}")
            if npth.value > 0:   # the impedance definition and its current path
                mode.update(zdef={0: "PV", 1: "VI", 2: "PI"}[zd.value], ipath=pbuf[:min(npth.value, 64)].copy(),
                            ipath_closed=bool(cl.value))
        ports.append({"mode": mode})
    prob = {"verts": verts, "tets": tets, "tet_region": reg.astype(np.int64), "bdr_tris": tris,
            "bdr_attr": attr.astype(np.int64), "order": p, "eps_r": mat[:, 0], "tand": mat[:, 1],
            "sigma": mat[:, 2], "mu_r": mat[:, 3], "boundaries": bnd, "ports": ports}
    return prob, fr[:nq]


class Fem3D:
    """One mesh + materials + boundaries resident on the device."""

    def __init__(self, prob, context=None, device=0):
        self.ctx = context if context is not None else Context(device)
        self.ctx._problems.add(self)
        self.prob = prob
        self._ne = len(prob["tets"])
        L = _lib.lib()
        verts = np.ascontiguousarray(prob["verts"], dtype=np.float64)
        tets = np.ascontiguousarray(prob["tets"], dtype=np.int64)
        reg = np.ascontiguousarray(prob["tet_region"], dtype=np.int32)
        tris = np.ascontiguousarray(prob["bdr_tris"], dtype=np.int64)
        attr = np.ascontiguousarray(prob["bdr_attr"], dtype=np.int32)
        self.h = C.c_void_p()
        rc = L.opem_problem_create(self.ctx.h, len(verts), _dp(verts), len(tets), tets.ctypes.data_as(_lib.I64P),
                                   reg.ctypes.data_as(_lib.I32P), len(tris), tris.ctypes.data_as(_lib.I64P),
                                   attr.ctypes.data_as(_lib.I32P), int(prob["order"]), C.byref(self.h))
        _chk(self.ctx.h, rc, "opem_problem_create")
        er = np.ascontiguousarray(prob["eps_r"], dtype=np.float64)
        td = np.ascontiguousarray(prob["tand"], dtype=np.float64)
        sg = np.ascontiguousarray(prob["sigma"], dtype=np.float64)
        mr = np.ascontiguousarray(prob["mu_r"], dtype=np.float64)
        _chk(self.ctx.h, L.opem_problem_set_regions(self.h, len(er), _dp(er), _dp(td), _dp(sg), _dp(mr)), "set_regions")
        for a, spec in prob["boundaries"].items():
            t = _BTYPES[spec["type"]]
            if spec["type"] == "port":
                pr = np.array([float(spec["port"])])
            elif spec["type"] == "impedance":
                pr = np.array([spec["sigma"], spec.get("Rz", 0.0), spec.get("mu_r", 1.0)])
            elif spec["type"] == "radiation":
                pr = np.array([spec.get("wave_impedance", 0.0)])
            else:
                pr = np.zeros(0)
            pr = np.ascontiguousarray(pr, dtype=np.float64)
            _chk(self.ctx.h, L.opem_problem_set_boundary(self.h, int(a), t, _dp(pr) if len(pr) else None, len(pr)),
                 "set_boundary")
        for k, port in enumerate(prob["ports"]):
            d = te_descriptor(port["mode"])
            if port["mode"].get("kind", "TE") == "FEM2D":
                _chk(self.ctx.h, L.opem_problem_set_port_fem2d(self.h, k, _dp(d), int(port["mode"]["nsub"]),
                                                               int(port["mode"].get("order2d", 1))),
                     "set_port_fem2d")
                ip = port["mode"].get("ipath")
                if ip is not None:   # impedance definition with a current path
                    ip = np.ascontiguousarray(ip, dtype=np.float64).reshape(-1, 3)
                    _chk(self.ctx.h, L.opem_problem_set_port_impedance(
                        self.h, k, _ZDEF[port["mode"].get("zdef", "PV")], len(ip), _dp(ip),
                        int(port["mode"].get("ipath_closed", True))), "set_port_impedance")
            else:
                _chk(self.ctx.h, L.opem_problem_set_port_te(self.h, k, _dp(d)), "set_port_te")
        # further modes of ports driven by their own 2D modes: one S-port each, after
        # every port's first mode (the oracle's order)
        nextra = 0
        for k, port in enumerate(prob["ports"]):
            for x in port["mode"].get("extra_modes", ()):
                vp = np.ascontiguousarray(np.concatenate([np.ravel(x["vpath"][0]), np.ravel(x["vpath"][1])]),
                                          dtype=np.float64)
                ip = x.get("ipath")
                ip = None if ip is None else np.ascontiguousarray(ip, dtype=np.float64).reshape(-1, 3)
                _chk(self.ctx.h, L.opem_problem_add_port_mode(
                    self.h, k, int(x["index"]), _dp(vp), _ZDEF[x.get("zdef", "PV")], 0 if ip is None else len(ip),
                    None if ip is None else _dp(ip), int(x.get("ipath_closed", True)), None), "add_port_mode")
                nextra += 1
        self.nports = len(prob["ports"]) + nextra
        self._assembled = False

    @classmethod
    def from_project(cls, proj_path, order=0, context=None, device=0):
        """An OpenParEM3D project (.proj with its gmsh 2.2 mesh, ports file and
        materials databases) -> (Fem3D, frequency plan).  order > 0 replaces
        mesh.order (orders 1-3 are built)."""
        info, freqs = project_info(proj_path, order)
        self = cls.__new__(cls)
        self.ctx = context if context is not None else Context(device)
        self.ctx._problems.add(self)
        self.prob = None
        self.h = C.c_void_p()
        nf = C.c_int()
        fr = np.zeros(max(1, info["frequencies"]))
        rc = _lib.lib().opem_project_load(self.ctx.h, str(proj_path).encode(), int(order), C.byref(self.h),
                                          C.byref(nf), _dp(fr), len(fr))
        _chk(self.ctx.h, rc, "opem_project_load")
        self.nports = info["ports"]
        self._ne = info["tets"]
        self._assembled = False
        return self, fr[:nf.value]

    # fem3D::build_fe_spaces + build_A's frequency-independent part
    def assemble(self):
        _chk(self.ctx.h, _lib.lib().opem_problem_assemble(self.h), "opem_problem_assemble")
        self._assembled = True
        return self

    def info(self):
        a = np.zeros(9, dtype=np.int64)
        _chk(self.ctx.h, _lib.lib().opem_problem_info(self.h, a.ctypes.data_as(_lib.I64P), 9), "info")
        keys = ["ndofs", "nnz", "nports", "npatches", "max_patch", "local_dofs", "device_bytes", "sum_patch",
                "sum_patch_sq"]
        return dict(zip(keys, (int(v) for v in a)))

    def solve(self, freq, opts=None, allow_not_converged=False):
        """One frequency point over every driving set -> (S (N,N) complex, Zo, stats)."""
        N = self.nports
        S = np.zeros(2 * N * N)
        Z = np.zeros(2 * N)
        st = SolveStats()
        o = opts if opts is not None else default_opts()
        rc = _lib.lib().opem_solve_frequency(self.h, float(freq), C.byref(o), _dp(S), _dp(Z), C.byref(st))
        if rc == _lib.ERR_NOT_CONVERGED and allow_not_converged:
            rc = _lib.OK
        _chk(self.ctx.h, rc, "opem_solve_frequency")
        return (S[0::2] + 1j * S[1::2]).reshape(N, N), Z[0::2] + 1j * Z[1::2], st.as_dict()

    def sweep(self, freqs, opts=None):
        freqs = np.ascontiguousarray(freqs, dtype=np.float64)
        N = self.nports
        S = np.zeros(2 * N * N * len(freqs))
        st = (SolveStats * len(freqs))()
        o = opts if opts is not None else default_opts()
        rc = _lib.lib().opem_solve_sweep(self.h, len(freqs), _dp(freqs), C.byref(o), _dp(S), st)
        _chk(self.ctx.h, rc, "opem_solve_sweep")
        return (S[0::2] + 1j * S[1::2]).reshape(len(freqs), N, N), [s.as_dict() for s in st]

    def mesh_errors(self, fraction):
        """ZZ error indicator of the last solve() (opem_mesh_errors) ->
        (errors per element, marked elements largest first, max error)."""
        ne = self._ne
        err = np.zeros(ne)
        cap = max(1, int(ne * fraction))
        marked = np.zeros(cap, dtype=np.int64)
        nm = C.c_int64()
        mx = C.c_double()
        _chk(self.ctx.h, _lib.lib().opem_mesh_errors(self.h, float(fraction), _dp(err), marked.ctypes.data_as(_lib.I64P),
                                                     cap, C.byref(nm), C.byref(mx)), "opem_mesh_errors")
        return err, marked[:nm.value], mx.value

    def fields(self, d):
        n = self.info()["ndofs"]
        e = np.zeros(2 * n)
        h = np.zeros(2 * n)
        _chk(self.ctx.h, _lib.lib().opem_get_fields(self.h, int(d), _dp(e), _dp(h)), "opem_get_fields")
        return e[0::2] + 1j * e[1::2], h[0::2] + 1j * h[1::2]

    OPERATORS = {"K": 0, "M_eps": 1, "M_tand": 2, "M_sig": 3, "M1": 4, "Q_mu": 5}

    def operator(self, name):
        inf = self.info()
        n, nnz = inf["ndofs"], inf["nnz"]
        rp = np.zeros(n + 1, dtype=np.int64)
        cols = np.zeros(nnz, dtype=np.int32)
        vals = np.zeros(nnz)
        _chk(self.ctx.h, _lib.lib().opem_get_operator(self.h, self.OPERATORS[name], rp.ctypes.data_as(_lib.I64P),
                                                      cols.ctypes.data_as(_lib.I32P), _dp(vals)), "get_operator")
        return sp.csr_matrix((vals, cols, rp), shape=(n, n))

    def system_matrix(self, freq, d):
        inf = self.info()
        n, nnz = inf["ndofs"], inf["nnz"]
        rp = np.zeros(n + 1, dtype=np.int64)
        cols = np.zeros(nnz, dtype=np.int32)
        _chk(self.ctx.h, _lib.lib().opem_get_operator(self.h, 0, rp.ctypes.data_as(_lib.I64P),
                                                      cols.ctypes.data_as(_lib.I32P), None), "get_operator")
        v = np.zeros(2 * nnz)
        _chk(self.ctx.h, _lib.lib().opem_get_system_matrix(self.h, float(freq), int(d), _dp(v)), "system_matrix")
        return sp.csr_matrix((v[0::2] + 1j * v[1::2], cols, rp), shape=(n, n))

    def close(self):
        if getattr(self, "h", None):
            _lib.lib().opem_problem_destroy(self.h)
            self.h = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class Server:
    """Serving loop on one GPU (opem_server_*): requests from any thread are
    admitted into ``slots`` concurrent slots by device-memory footprint and
    run overlapped on the device; problems keep their operators resident.

    A submitted Fem3D belongs to the server until its request has been waited
    for; use it (or close it) only afterwards."""

    def __init__(self, device=0, slots=4, hbm_budget_bytes=0):
        self.h = C.c_void_p()
        rc = _lib.lib().opem_server_create(int(device), int(slots), int(hbm_budget_bytes), C.byref(self.h))
        if rc != _lib.OK:
            raise OpemError(rc, "opem_server_create")
        self._pending = {}

    def submit(self, fem, freqs, opts=None):
        freqs = np.ascontiguousarray(np.atleast_1d(freqs), dtype=np.float64)
        o = opts if opts is not None else default_opts()
        rid = C.c_int64()
        rc = _lib.lib().opem_server_submit(self.h, fem.h, len(freqs), _dp(freqs), C.byref(o), C.byref(rid))
        if rc != _lib.OK:
            raise OpemError(rc, "opem_server_submit")
        self._pending[rid.value] = (fem, len(freqs), freqs)
        return rid.value

    def wait(self, rid, timeout=-1.0):
        """-> (S (nfreq, N, N) complex, stats list, {"submitted", "started", "finished"} seconds)."""
        fem, nf, _ = self._pending[rid]
        N = fem.nports
        S = np.zeros(2 * N * N * nf)
        st = (SolveStats * nf)()
        t = np.zeros(3)
        rc = _lib.lib().opem_server_wait(self.h, int(rid), float(timeout), _dp(S), st, _dp(t))
        if rc == _lib.ERR_TIMEOUT:
            raise TimeoutError(f"request {rid} not finished")
        del self._pending[rid]
        if rc not in (_lib.OK, _lib.ERR_NOT_CONVERGED):
            raise OpemError(rc, f"request {rid}")
        times = {"submitted": t[0], "started": t[1], "finished": t[2]}
        return (S[0::2] + 1j * S[1::2]).reshape(nf, N, N), [s.as_dict() for s in st], times

    def cancel(self, rid):
        """Queued: dropped at once; running: stops at its next Krylov step.  Its wait
        then raises OpemError with code ERR_CANCELLED (unless it had finished)."""
        rc = _lib.lib().opem_server_cancel(self.h, int(rid))
        if rc != _lib.OK:
            raise OpemError(rc, f"cancel {rid}")

    def info(self):
        a = np.zeros(6, dtype=np.int64)
        _lib.lib().opem_server_info(self.h, a.ctypes.data_as(_lib.I64P), 6)
        return dict(zip(["queued", "running", "completed", "admitted_bytes", "budget_bytes", "slots"],
                        (int(v) for v in a)))

    def close(self):
        if getattr(self, "h", None):
            _lib.lib().opem_server_destroy(self.h)
            self.h = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def renormalize(S, Zo, zref=50.0):
    """S (nfreq, N, N) or (N, N) with port impedances Zo ((nfreq,) N) -> S referred to
    zref on every port (opem_s_renormalize)."""
    S = np.asarray(S, dtype=np.complex128)
    Zo = np.asarray(Zo, dtype=np.complex128)
    one = S.ndim == 2
    S3 = S[None] if one else S
    Z2 = np.broadcast_to(Zo, (S3.shape[0], S3.shape[1]))
    out = np.empty_like(S3)
    N = S3.shape[1]
    for q in range(S3.shape[0]):
        si = np.ascontiguousarray(S3[q]).view(np.float64).ravel()
        zi = np.ascontiguousarray(Z2[q]).view(np.float64).ravel()
        so = np.zeros(2 * N * N)
        rc = _lib.lib().opem_s_renormalize(N, _dp(si), _dp(zi), float(np.real(zref)), float(np.imag(zref)), _dp(so))
        if rc != _lib.OK:
            raise OpemError(rc, "opem_s_renormalize")
        out[q] = (so[0::2] + 1j * so[1::2]).reshape(N, N)
    return out[0] if one else out


def write_touchstone(path, freqs, S, zref=50.0, fmt="RI", unit="GHz"):
    """Touchstone 1.1 file of renormalised S (nfreq, N, N) (opem_write_touchstone)."""
    freqs = np.ascontiguousarray(freqs, dtype=np.float64)
    S = np.ascontiguousarray(S, dtype=np.complex128)
    N = S.shape[1]
    flat = S.view(np.float64).ravel()
    rc = _lib.lib().opem_write_touchstone(str(path).encode(), len(freqs), _dp(freqs), N, _dp(flat), float(zref),
                                          fmt.encode(), unit.encode())
    if rc != _lib.OK:
        raise OpemError(rc, "opem_write_touchstone")



def mixed_mode(S, pairs, zref=50.0):
    """Mixed-mode S of single-ended S (N, N) renormalised to zref (opem_s_mixed_mode):
    pairs = [(P, N), ...] 1-based S-ports -> (S_mm, Zo)."""
    S = np.ascontiguousarray(S, dtype=np.complex128)
    n = S.shape[0]
    pr = np.ascontiguousarray(np.asarray(pairs, dtype=np.int32).reshape(-1, 2))
    out = np.zeros((n, n), dtype=np.complex128)
    zo = np.zeros(n, dtype=np.complex128)
    rc = _lib.lib().opem_s_mixed_mode(n, _dp(S.view(np.float64).ravel()), len(pr),
                                      pr.ctypes.data_as(C.POINTER(C.c_int)), float(zref),
                                      _dp(out.view(np.float64).ravel()), _dp(zo.view(np.float64).ravel()))
    if rc != _lib.OK:
        raise OpemError(rc, "opem_s_mixed_mode")
    return out, zo


def single_ended(S, Zmode, Tv, Ti, zref=50.0):
    """Single-ended S at zref of modal S (N, N) (opem_s_single_ended): Zmode (N,)
    the modes' impedances, Tv and Ti (N, N) the single-ended -> modal voltage and
    current maps (each port's block on the diagonal, S-port order)."""
    S = np.ascontiguousarray(S, dtype=np.complex128)
    n = S.shape[0]
    zm = np.ascontiguousarray(Zmode, dtype=np.complex128)
    tv = np.ascontiguousarray(Tv, dtype=np.complex128)
    ti = np.ascontiguousarray(Ti, dtype=np.complex128)
    if zm.shape != (n,) or tv.shape != (n, n) or ti.shape != (n, n):
        raise OpemError(_lib.ERR_ARG, "single_ended: shapes")
    out = np.zeros((n, n), dtype=np.complex128)
    rc = _lib.lib().opem_s_single_ended(n, _dp(S.view(np.float64).ravel()), _dp(zm.view(np.float64).ravel()),
                                        _dp(tv.view(np.float64).ravel()), _dp(ti.view(np.float64).ravel()),
                                        float(zref), _dp(out.view(np.float64).ravel()), None)
    if rc != _lib.OK:
        raise OpemError(rc, "opem_s_single_ended")
    return out


def port_line_maps(I, V=None):
    """Line-to-modal maps of one multi-line port (opem_port_line_maps): I and V
    (n, n) the modes' line currents and voltages (row = mode, column = line).
    Returns {"Ti", "Tv", "flipped", "Im", "Vm"}; Im and Vm are the mode currents and
    voltages after the flips (Vm zero without V)."""
    I = np.ascontiguousarray(I, dtype=np.complex128)
    n = I.shape[0]
    if I.shape != (n, n) or n < 1:
        raise OpemError(_lib.ERR_ARG, "port_line_maps: shapes")
    vp = None
    if V is not None:
        V = np.ascontiguousarray(V, dtype=np.complex128)
        if V.shape != (n, n):
            raise OpemError(_lib.ERR_ARG, "port_line_maps: shapes")
        vp = _dp(V.view(np.float64).ravel())
    ti = np.zeros((n, n), dtype=np.complex128)
    tv = np.zeros((n, n), dtype=np.complex128)
    fl = np.zeros(n, dtype=np.int32)
    im = np.zeros(n, dtype=np.complex128)
    vm = np.zeros(n, dtype=np.complex128)
    rc = _lib.lib().opem_port_line_maps(n, _dp(I.view(np.float64).ravel()), vp, _dp(ti.view(np.float64).ravel()),
                                        _dp(tv.view(np.float64).ravel()), fl.ctypes.data_as(C.POINTER(C.c_int)),
                                        _dp(im.view(np.float64).ravel()), _dp(vm.view(np.float64).ravel()))
    if rc != _lib.OK:
        raise OpemError(rc, "opem_port_line_maps")
    return {"Ti": ti, "Tv": tv, "flipped": fl.astype(bool), "Im": im, "Vm": vm}


def write_touchstone2(path, freqs, S, zref=50.0, fmt="RI", unit="GHz", pairs=()):
    """Touchstone 2.0 file (opem_write_touchstone2); pairs mark mixed-mode S-ports."""
    freqs = np.ascontiguousarray(freqs, dtype=np.float64)
    S = np.ascontiguousarray(S, dtype=np.complex128)
    N = S.shape[1]
    pr = np.ascontiguousarray(np.asarray(pairs, dtype=np.int32).reshape(-1, 2))
    rc = _lib.lib().opem_write_touchstone2(str(path).encode(), len(freqs), _dp(freqs), N,
                                           _dp(S.view(np.float64).ravel()), float(zref), fmt.encode(), unit.encode(),
                                           len(pr), pr.ctypes.data_as(C.POINTER(C.c_int)))
    if rc != _lib.OK:
        raise OpemError(rc, "opem_write_touchstone2")


def write_results_csv(path, freqs, S, zref=50.0, fmt="DB", unit="GHz"):
    """The reference's _results.csv layout (opem_write_results_csv); zref <= 0 marks
    S as not renormalised."""
    freqs = np.ascontiguousarray(freqs, dtype=np.float64)
    S = np.ascontiguousarray(S, dtype=np.complex128)
    rc = _lib.lib().opem_write_results_csv(str(path).encode(), len(freqs), _dp(freqs), S.shape[1],
                                           _dp(S.view(np.float64).ravel()), float(zref), fmt.encode(), unit.encode())
    if rc != _lib.OK:
        raise OpemError(rc, "opem_write_results_csv")


def evaluate_test_cases(test_cases, results_csv, out_path):
    """The reference's regression comparator (opem_evaluate_test_cases) ->
    (number of cases, number passed); the evaluation is written to out_path."""
    nc, npass = C.c_int(), C.c_int()
    rc = _lib.lib().opem_evaluate_test_cases(str(test_cases).encode(), str(results_csv).encode(),
                                             str(out_path).encode(), C.byref(nc), C.byref(npass))
    if rc != _lib.OK:
        raise OpemError(rc, "opem_evaluate_test_cases")
    return nc.value, npass.value


def s_relative_change(S_prev, S_cur):
    """Largest column 2-norm of S_cur^-1 (S_prev - S_cur) (opem_s_relative_change)."""
    a = np.ascontiguousarray(S_prev, dtype=np.complex128)
    b = np.ascontiguousarray(S_cur, dtype=np.complex128)
    out = C.c_double()
    rc = _lib.lib().opem_s_relative_change(a.shape[0], _dp(a.view(np.float64).ravel()),
                                           _dp(b.view(np.float64).ravel()), C.byref(out))
    if rc != _lib.OK:
        raise OpemError(rc, "opem_s_relative_change")
    return out.value


def refine_problem(prob, marked):
    """A copy of a problem dict with the marked tetrahedra refined
    (opem_refine_mesh: longest-edge bisection with conforming closure)."""
    verts = np.ascontiguousarray(prob["verts"], dtype=np.float64)
    tets = np.ascontiguousarray(prob["tets"], dtype=np.int64)
    reg = np.ascontiguousarray(prob.get("tet_region", np.zeros(len(tets))), dtype=np.int32)
    tris = np.ascontiguousarray(prob["bdr_tris"], dtype=np.int64)
    attr = np.ascontiguousarray(prob["bdr_attr"], dtype=np.int32)
    mk = np.ascontiguousarray(marked, dtype=np.int64)
    L = _lib.lib()
    cnt = np.zeros(3, dtype=np.int64)
    args = (len(verts), _dp(verts), len(tets), tets.ctypes.data_as(_lib.I64P), reg.ctypes.data_as(_lib.I32P),
            len(tris), tris.ctypes.data_as(_lib.I64P), attr.ctypes.data_as(_lib.I32P), len(mk),
            mk.ctypes.data_as(_lib.I64P), cnt.ctypes.data_as(_lib.I64P))
    rc = L.opem_refine_mesh(*args, None, None, None, None, None)
    if rc != _lib.OK:
        raise OpemError(rc, "opem_refine_mesh")
    nv, nt, nb = (int(c) for c in cnt)
    V = np.zeros((nv, 3)); T = np.zeros((nt, 4), dtype=np.int64); R = np.zeros(nt, dtype=np.int32)
    B = np.zeros((nb, 3), dtype=np.int64); A = np.zeros(nb, dtype=np.int32)
    rc = L.opem_refine_mesh(*args, _dp(V), T.ctypes.data_as(_lib.I64P), R.ctypes.data_as(_lib.I32P),
                            B.ctypes.data_as(_lib.I64P), A.ctypes.data_as(_lib.I32P))
    if rc != _lib.OK:
        raise OpemError(rc, "opem_refine_mesh")
    out = dict(prob)
    out.update(verts=V, tets=T, tet_region=R.astype(np.int64), bdr_tris=B, bdr_attr=A.astype(np.int64))
    return out


def adaptive_solve(prob, step, fraction=0.005, variable="SandH", rel_tol=0.02, abs_tol=1e-6, iter_min=1,
                   iter_max=10, passes=1):
    """The reference's adaptive loop for one frequency point (OpenParEM3D.cpp:442-630,
    is_converged project.c:344-364, isSequentialConverged results.cpp:828-843):
    step(prob) -> (S, max mesh error, marked elements) solves and estimates; the
    change of S between passes (s_relative_change) and/or the max mesh error are
    tested against rel_tol / abs_tol ("S", "SorH", "SandH"), iterations below
    iter_min never converge, the loop stops after `passes` converged passes in a
    row or iter_max passes, and otherwise refines the marked elements
    (refine_problem).  Returns (S, final problem, history of per-pass dicts)."""
    history, S_prev, conv_run = [], None, 0
    for it in range(iter_max):
        S, max_err, marked = step(prob)
        rel = s_relative_change(S_prev, S) if S_prev is not None else -1.0
        ok_rel = 0 <= rel <= rel_tol
        ok_abs = 0 <= max_err <= abs_tol
        conv = {"S": ok_rel, "SorH": ok_rel or ok_abs, "SandH": ok_rel and ok_abs}[variable]
        if it < iter_min - 1:
            conv = False
        conv_run = conv_run + 1 if conv else 0
        history.append({"iteration": it + 1, "tets": len(prob["tets"]), "S": S, "relative_error": rel,
                        "max_mesh_error": max_err, "converged": conv})
        if conv_run >= passes or it == iter_max - 1:
            return S, prob, history
        prob = refine_problem(prob, marked)
        S_prev = S
    return S, prob, history


def device_step(freq, fraction=0.005, opts=None, context=None):
    """A step for adaptive_solve on the device: assemble, opem_solve_frequency,
    opem_mesh_errors."""
    def step(prob):
        F = Fem3D(prob, context=context).assemble()
        S, _, _ = F.solve(freq, opts)
        _, marked, mx = F.mesh_errors(fraction)
        return S, mx, marked
    return step


# the reference's defaults for the adaptive keys (project.c:555-567)
REFINEMENT_DEFAULTS = {"mesh.3D.refinement.fraction": 0.005, "refinement.frequency": "highlow",
                       "refinement.iteration.min": 1, "refinement.iteration.max": 10,
                       "refinement.required.passes": 1, "refinement.relative.tolerance": 0.02,
                       "refinement.absolute.tolerance": 1e-6, "refinement.variable": "SandH"}


def project_refinement(proj_path):
    """The adaptive settings of a project (opem_project_value), the reference's
    defaults where a key is absent, as keyword arguments of adaptive_solve plus
    "frequency" (none | high | low | highlow | all | plan)."""
    buf = C.create_string_buffer(256)
    v = {}
    for k, d in REFINEMENT_DEFAULTS.items():
        rc = _lib.lib().opem_project_value(str(proj_path).encode(), k.encode(), buf, 256)
        v[k] = type(d)(buf.value.decode()) if rc == _lib.OK else d
    return {"fraction": v["mesh.3D.refinement.fraction"], "variable": v["refinement.variable"],
            "rel_tol": v["refinement.relative.tolerance"], "abs_tol": v["refinement.absolute.tolerance"],
            "iter_min": v["refinement.iteration.min"], "iter_max": v["refinement.iteration.max"],
            "passes": v["refinement.required.passes"], "frequency": v["refinement.frequency"]}


def project_value(proj_path, key, default=None):
    """The last value of a .proj key as a string (opem_project_value), or default."""
    buf = C.create_string_buffer(256)
    rc = _lib.lib().opem_project_value(str(proj_path).encode(), key.encode(), buf, 256)
    return buf.value.decode() if rc == _lib.OK else default
