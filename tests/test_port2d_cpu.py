"""The library's host 2D port-mode solver (opem_port_mode_2d) against the oracle
(oracle/port2d.py) on the same meshes, and against closed forms."""
import ctypes as C

import numpy as np

from oracle import port2d
from openparem_b200 import _lib

A, B = 22.86e-3, 10.16e-3


def _solve(pts, tris, freq, eps):
    L = _lib.lib()
    xy = np.ascontiguousarray(pts, dtype=np.float64).ravel()
    t = np.ascontiguousarray(tris, dtype=np.int64).ravel()
    er = np.ascontiguousarray(np.broadcast_to(np.asarray(eps, dtype=np.complex128), (len(tris),))).view(np.float64).ravel()
    beta = np.zeros(2)
    ne = C.c_int64()
    rc = L.opem_port_mode_2d(len(pts), xy.ctypes.data_as(_lib.DP), len(tris), t.ctypes.data_as(_lib.I64P),
                             er.ctypes.data_as(_lib.DP), None, freq, beta.ctypes.data_as(_lib.DP), C.byref(ne),
                             None, None, None)
    assert rc == _lib.OK
    edges = np.zeros(2 * ne.value, dtype=np.int64)
    et = np.zeros(2 * ne.value)
    ez = np.zeros(2 * len(pts))
    rc = L.opem_port_mode_2d(len(pts), xy.ctypes.data_as(_lib.DP), len(tris), t.ctypes.data_as(_lib.I64P),
                             er.ctypes.data_as(_lib.DP), None, freq, beta.ctypes.data_as(_lib.DP), C.byref(ne),
                             edges.ctypes.data_as(_lib.I64P), et.ctypes.data_as(_lib.DP), ez.ctypes.data_as(_lib.DP))
    assert rc == _lib.OK
    return beta[0] + 1j * beta[1], edges.reshape(-1, 2), et[0::2] + 1j * et[1::2], ez[0::2] + 1j * ez[1::2]


def test_matches_oracle_on_loaded_guide():
    w, f = 2e-3, 8.3e9
    pts, tris = port2d.rect_mesh(A, B, 46, 23, x_breaks=(-w / 2, w / 2))
    cx = pts[tris].mean(axis=1)[:, 0]
    eps = np.where(np.abs(cx) < w / 2, 2.2, 1.0006)
    b1, edges, et, ez = _solve(pts, tris, f, eps)
    b0, et0, ez0, edges0 = port2d.solve_mode(pts, tris, f, eps)
    assert abs(b1 - b0) / abs(b0) < 1e-10
    assert np.array_equal(edges, edges0)
    s0 = 1.0 / et0[np.argmax(np.abs(et0))]
    assert np.abs(et - et0 * s0).max() < 1e-8
    # e_z of this TE-like mode is ~1e-5 of the field's natural scale (e_t / h), so its
    # relative agreement is limited by the eigenvectors' accuracy
    assert np.abs(ez - ez0 * s0).max() < 1e-2 * np.abs(ez0 * s0).max()


def test_empty_guide_and_lossy_fill():
    f = 10e9
    k0 = 2 * np.pi * f / 299792458.0
    pts, tris = port2d.rect_mesh(A, B, 64, 32)
    b, _, _, _ = _solve(pts, tris, f, 1.0)
    exact = np.sqrt(k0 ** 2 - (np.pi / A) ** 2)
    assert abs(b - exact) / exact < 5e-5
    # lossy homogeneous fill: beta = sqrt(k0^2 eps_c - kc^2) with the same discretisation error
    eps_c = 2.0 - 0.02j
    bl, _, _, _ = _solve(pts, tris, f, eps_c)
    exact_l = np.sqrt(k0 ** 2 * eps_c - (np.pi / A) ** 2)
    assert abs(bl - exact_l) / abs(exact_l) < 5e-5 and bl.imag < 0   # exp(-j beta z) decays
