"""Oracle: FP64 per-frequency solve on the host cores by preconditioned GMRES
(test and baseline infrastructure; never called by the product).

``fem.solve_frequency`` factors A(omega) with SuperLU, the reference's own
approach (PCCHOLESKY/PCLU inside KSPGMRES, solveComplexLinearSystem.c:137-168).
Its fill grows too fast for the 681,312-DOF benchmark guide: one point takes
hours on a host CPU.  ``CpuSolver`` solves the same FP64 problem, with the same
Dirichlet procedure (solveComplexLinearSystem.c:114-129), H projection
(fem3D.cpp:192-225) and overlaps / S (port.cpp:3463-3568, :7499-7606), by
GMRES with deflated restarting (Morgan's GMRES-DR; the harmonic Ritz vectors of
each cycle are kept) right-preconditioned by overlapping vertex-patch block
Jacobi, on all host threads: complex CSR products, block inversion and block
apply in oracle/cpu_kernels.c (OpenMP), the Krylov basis updates in numpy
(threaded BLAS), the mass-matrix solve for H by Jacobi-preconditioned CG.
"""
import ctypes as C
import os
import subprocess

import numpy as np

from . import fem

HERE = os.path.dirname(os.path.abspath(__file__))
LIB = os.path.join(HERE, "_build", "libopem_cpu.so")


def build():
    """Compile oracle/cpu_kernels.c into oracle/_build/libopem_cpu.so."""
    os.makedirs(os.path.dirname(LIB), exist_ok=True)
    src = os.path.join(HERE, "cpu_kernels.c")
    if os.path.exists(LIB) and os.path.getmtime(LIB) >= os.path.getmtime(src):
        return LIB
    subprocess.run(["gcc", "-O3", "-march=x86-64-v3", "-fopenmp", "-shared", "-fPIC", src, "-o", LIB, "-lm"],
                   check=True)
    return LIB


_lib = None


def lib():
    global _lib
    if _lib is None:
        build()
        L = C.CDLL(LIB)
        vp = C.c_void_p
        L.opem_cpu_spmv.argtypes = [C.c_int64, vp, vp, vp, vp, vp]
        L.opem_cpu_patch_invert.argtypes = [C.c_int, vp, vp, vp, vp, vp, vp, vp]
        L.opem_cpu_patch_invert.restype = C.c_int
        L.opem_cpu_patch_apply.argtypes = [C.c_int, vp, vp, vp, vp, C.c_int64, vp, vp, vp, vp, vp]
        L.opem_cpu_cg2.argtypes = [C.c_int64, vp, vp, vp, vp, vp, C.c_double, C.c_int, vp, vp]
        L.opem_cpu_cg2.restype = C.c_int
        _lib = L
    return _lib


def _p(a):
    return a.ctypes.data_as(C.c_void_p)


def vertex_patches(topo):
    """Overlapping vertex patches: for each mesh vertex, the DOFs of every edge,
    face and cell that contains it (sorted).  Returns (pptr int64, pdofs int32)."""
    p = topo.p
    nd = fem.ndofs(p)
    tets = topo.tets
    nv = int(tets.max()) + 1
    rows, cols = [], []
    for le, (a, b) in enumerate(fem.EDGES):
        for k in range(nd["edge"]):
            dof = topo.tet_edges[:, le] * nd["edge"] + k
            for vv in (a, b):
                rows.append(tets[:, vv])
                cols.append(dof)
    base_f = topo.nE * nd["edge"]
    for lf, f in enumerate(fem.FACES):
        for k in range(nd["face"]):
            dof = base_f + topo.tet_faces[:, lf] * nd["face"] + k
            for vv in f:
                rows.append(tets[:, vv])
                cols.append(dof)
    base_i = base_f + topo.nF * nd["face"]
    for k in range(nd["interior"]):
        dof = base_i + np.arange(len(tets)) * nd["interior"] + k
        for vv in range(4):
            rows.append(tets[:, vv])
            cols.append(dof)
    key = np.unique(np.concatenate(rows).astype(np.int64) * topo.n + np.concatenate(cols))
    vert = key // topo.n
    dofs = (key % topo.n).astype(np.int32)
    pptr = np.zeros(nv + 1, dtype=np.int64)
    np.add.at(pptr, vert + 1, 1)
    return np.cumsum(pptr), dofs


class BlockJacobi:
    """Additive vertex-patch block Jacobi: M^{-1} x = sum_v R_v^T (R_v A R_v^T)^{-1} R_v x."""

    def __init__(self, A, pptr, pdofs):
        L = lib()
        self.n = A.shape[0]
        self.pptr, self.pdofs = pptr, pdofs
        s = np.diff(pptr)
        self.boff = np.concatenate([[0], np.cumsum(s.astype(np.int64) ** 2)[:-1]]).astype(np.int64)
        self.blocks = np.empty(int((s.astype(np.int64) ** 2).sum()), dtype=np.complex128)
        A = A.tocsr()
        A.sort_indices()
        rp = A.indptr.astype(np.int64)
        ci = A.indices.astype(np.int32)
        vals = np.ascontiguousarray(A.data, dtype=np.complex128)
        self.bad = L.opem_cpu_patch_invert(len(s), _p(pptr), _p(pdofs), _p(self.boff), _p(rp), _p(ci), _p(vals),
                                           _p(self.blocks))
        order = np.argsort(pdofs, kind="stable")
        self.d2p_idx = order.astype(np.int64)
        cnt = np.bincount(pdofs, minlength=self.n)
        self.d2p_ptr = np.concatenate([[0], np.cumsum(cnt)]).astype(np.int64)
        self.t = np.empty(len(pdofs), dtype=np.complex128)

    def __call__(self, x):
        x = np.ascontiguousarray(x, dtype=np.complex128)
        y = np.empty(self.n, dtype=np.complex128)
        lib().opem_cpu_patch_apply(len(self.pptr) - 1, _p(self.pptr), _p(self.pdofs), _p(self.boff),
                                   _p(self.blocks), self.n, _p(self.d2p_ptr), _p(self.d2p_idx), _p(x), _p(self.t),
                                   _p(y))
        return y


class Csr:
    def __init__(self, A):
        A = A.tocsr()
        self.n = A.shape[0]
        self.rp = A.indptr.astype(np.int64)
        self.ci = A.indices.astype(np.int32)
        self.vals = np.ascontiguousarray(A.data, dtype=np.complex128)

    def __call__(self, x):
        x = np.ascontiguousarray(x, dtype=np.complex128)
        y = np.empty(self.n, dtype=np.complex128)
        lib().opem_cpu_spmv(self.n, _p(self.rp), _p(self.ci), _p(self.vals), _p(x), _p(y))
        return y


def gmres_dr(matvec, prec, b, m=100, k=30, rtol=1e-10, maxits=10000):
    """Right-preconditioned GMRES with deflated restarting (Morgan, SIAM J. Sci.
    Comput. 24 (2002)): solves A M^{-1} u = b, returns x = M^{-1} u and the
    number of Arnoldi steps.  Classical Gram-Schmidt with one
    reorthogonalisation; after each cycle the k harmonic Ritz vectors of
    smallest magnitude and the residual are kept as the next cycle's basis."""
    n = len(b)
    bn = np.linalg.norm(b)
    x = np.zeros(n, dtype=np.complex128)
    if bn == 0:
        return x, 0
    V = np.zeros((n, m + 1), dtype=np.complex128, order="F")
    H = np.zeros((m + 1, m), dtype=np.complex128)
    c = np.zeros(m + 1, dtype=np.complex128)
    V[:, 0] = b / bn
    c[0] = bn
    j0, its = 0, 0
    while True:
        jend = j0
        done = False
        for j in range(j0, m):
            w = matvec(prec(V[:, j]))
            Vj = V[:, :j + 1]
            h = Vj.conj().T @ w
            w -= Vj @ h
            h2 = Vj.conj().T @ w
            w -= Vj @ h2
            h += h2
            hn = np.linalg.norm(w)
            H[:j + 1, j] = h
            H[j + 1, j] = hn
            V[:, j + 1] = w / hn if hn > 0 else 0
            its += 1
            jend = j + 1
            y = np.linalg.lstsq(H[:jend + 1, :jend], c[:jend + 1], rcond=None)[0]
            res = np.linalg.norm(c[:jend + 1] - H[:jend + 1, :jend] @ y)
            if res <= rtol * bn or its >= maxits or hn == 0:
                done = True
                break
        y = np.linalg.lstsq(H[:jend + 1, :jend], c[:jend + 1], rcond=None)[0]
        x += prec(V[:, :jend] @ y)
        if done:
            return x, its
        # deflated restart: harmonic Ritz vectors of H_m
        s = c - H @ y
        Hm = H[:m, :m]
        em = np.zeros(m, dtype=np.complex128)
        em[-1] = 1
        f = np.linalg.solve(Hm.conj().T, em)
        theta, G = np.linalg.eig(Hm + abs(H[m, m - 1]) ** 2 * np.outer(f, em))
        P = G[:, np.argsort(np.abs(theta))[:k]]
        Pk = np.zeros((m + 1, k + 1), dtype=np.complex128)
        Pk[:m, :k] = P
        Pk[:, k] = s
        Q, _ = np.linalg.qr(Pk)
        V[:, :k + 1] = V @ Q
        Hn = Q.conj().T @ H @ Q[:m, :k]
        H[:] = 0
        H[:k + 1, :k] = Hn
        c[:] = 0
        c[:k + 1] = Q.conj().T @ s
        j0 = k


class CpuSolver:
    """The oracle problem of ``fem.Operators`` solved frequency by frequency on
    the host cores (see the module docstring); ``solve_frequency`` returns what
    ``fem.solve_frequency`` returns plus the Krylov step counts."""

    def __init__(self, ops, restart=100, deflate=30, rtol=1e-10, h_rtol=1e-12):
        self.ops = ops
        self.m, self.k, self.rtol, self.h_rtol = restart, deflate, rtol, h_rtol
        self.pptr, self.pdofs = vertex_patches(ops.topo)
        P = ops.M1.tocsr()
        P.sort_indices()
        self.P_rp = P.indptr.astype(np.int64)
        self.P_ci = P.indices.astype(np.int32)
        self.P_v = np.ascontiguousarray(P.data, dtype=np.float64)

    def _mass_solve(self, q):
        n = len(q)
        re = np.ascontiguousarray(q.real)
        im = np.ascontiguousarray(q.imag)
        xr = np.empty(n)
        xi = np.empty(n)
        it = lib().opem_cpu_cg2(n, _p(self.P_rp), _p(self.P_ci), _p(self.P_v), _p(re), _p(im), self.h_rtol, 20000,
                                _p(xr), _p(xi))
        return xr + 1j * xi, it

    def solve_frequency(self, freq, reciprocal=True):
        ops, topo = self.ops, self.ops.topo
        w = 2 * np.pi * freq
        N = len(ops.ports)
        mm = [fem.port_mode(ops, k, freq) for k in range(N)]
        Et = [ops.port_trace(k, mm[k]["Et"]) for k in range(N)]
        Ht = [ops.port_trace(k, mm[k]["Ht"]) for k in range(N)]
        Cp = np.zeros((N, N), dtype=np.complex128)
        Cm = np.zeros((N, N), dtype=np.complex128)
        its, h_its = [], []
        for d in range(N):
            A = fem.assemble_A(ops, freq, d)
            A = fem.eliminate(A, ops.pec_dofs)
            x0 = np.zeros(topo.n, dtype=np.complex128)
            pd = ops.ports[d]["dofs"]
            x0[pd] = Et[d][pd]
            b = -(A @ x0)
            b[pd] = x0[pd]
            A = fem.eliminate(A, pd)
            M = BlockJacobi(A, self.pptr, self.pdofs)
            e, it = gmres_dr(Csr(A), M, b, self.m, self.k, self.rtol)
            its.append(it)
            qe = (ops.Q_mu @ e) / (w * fem.MU0)
            hs, hit = self._mass_solve(qe)
            h_its.append(hit)
            h = 1j * hs
            for k in range(N):
                Bm = ops.ports[k]["Bm1"]
                e0 = np.vdot(Et[k], Bm @ e)
                e2 = np.vdot(Et[k], Bm @ Et[k])
                h0 = np.vdot(Ht[k], Bm @ h)
                h2 = np.vdot(Ht[k], Bm @ Ht[k])
                Cp[d, k] = 0.5 * (e0 / e2 + h0 / h2)
                Cm[d, k] = 0.5 * (e0 / e2 - h0 / h2)
        S = fem.s_matrix(Cp, Cm, [q["V"] for q in mm], [q["Z"] for q in mm])
        if reciprocal:
            S = 0.5 * (S + S.T)
        return {"S": S, "Cp": Cp, "Cm": Cm, "iterations": its, "h_iterations": h_its}
