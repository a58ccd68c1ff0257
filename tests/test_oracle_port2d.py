"""The 2D port-mode oracle (oracle/port2d.py) against closed forms and against
the reference's own recorded result for its slab-loaded WR90 guide.

The reference's regression project WR90/straight-loaded (mesh straight-loaded.msh:
a 22.86 x 10.16 mm guide, 0.1 m long, with a full-height teflon slab eps_r 2.2 for
|x| < 1 mm, air eps_r 1.0006; one point at 8.3 GHz) gets its port modes from
OpenParEM2D; the guide is uniform and matched, so arg S21 = -beta L (mod 360).
The expected and found values come from tests/golden/wr90_expected.json.
"""
import json
import os

import numpy as np

from oracle import port2d

HERE = os.path.dirname(os.path.abspath(__file__))
A, B = 22.86e-3, 10.16e-3


def _loaded_case():
    d = json.load(open(os.path.join(HERE, "golden", "wr90_expected.json")))
    return d["cases"]["./WR90/straight-loaded/straight-loaded.proj"]["straight-loaded_1_3_result"]


def _wrap(deg):
    return (deg + 180.0) % 360.0 - 180.0


def test_empty_guide_te10_converges():
    f = 10e9
    k0 = 2 * np.pi * f / 299792458.0
    exact = np.sqrt(k0 ** 2 - (np.pi / A) ** 2)
    errs = []
    for n in (8, 16, 32):
        pts, tris = port2d.rect_mesh(A, B, 2 * n, n)
        beta, et, ez, _ = port2d.solve_mode(pts, tris, f, 1.0)
        errs.append(abs(beta - exact) / exact)
        assert np.abs(ez).max() < 1e-9 * np.abs(et).max()   # TE: no longitudinal field
    assert errs[-1] < 2e-5
    assert 3.5 < errs[0] / errs[1] < 4.5 and 3.5 < errs[1] / errs[2] < 4.5   # second order


def test_slab_dispersion_matches_reference_regression():
    case = _loaded_case()
    beta = port2d.slab_beta(A, 2e-3, 2.2, case["frequency"], eps_air=1.0006)
    phase = _wrap(np.degrees(-beta * 0.1))
    assert abs(phase - case["expected"]) < 1e-6
    assert abs(phase - case["found"]) <= 1e-5 * abs(case["expected"])   # the reference's own tolerance


def test_fem_mode_of_the_loaded_guide():
    case = _loaded_case()
    f, w = case["frequency"], 2e-3
    exact = port2d.slab_beta(A, w, 2.2, f, eps_air=1.0006)
    betas = []
    for n in (46, 92):
        pts, tris = port2d.rect_mesh(A, B, n, n // 2, x_breaks=(-w / 2, w / 2))
        cx = pts[tris].mean(axis=1)[:, 0]
        eps = np.where(np.abs(cx) < w / 2, 2.2, 1.0006)
        betas.append(port2d.solve_mode(pts, tris, f, eps)[0].real)
    assert abs(betas[1] - exact) / exact < 5e-5
    rich = (4 * betas[1] - betas[0]) / 3          # second-order Richardson extrapolation
    assert abs(rich - exact) / exact < 1e-6
    assert abs(_wrap(np.degrees(-rich * 0.1)) - case["expected"]) <= 1e-5 * abs(case["expected"])
