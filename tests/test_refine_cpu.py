"""Conforming refinement of marked tetrahedra (opem_refine_mesh) and the
reference's adaptive loop (fem3d.adaptive_solve) on the CPU, with the oracle
as the solver and error indicator."""
import os
from collections import Counter

import numpy as np
import pytest

from openparem_b200 import meshgen
from openparem_b200.fem3d import refine_problem, s_relative_change, adaptive_solve
from oracle import fem
from oracle.estimate import mesh_errors

HERE = os.path.dirname(os.path.abspath(__file__))
FACE = ([0, 1, 2], [0, 1, 3], [0, 2, 3], [1, 2, 3])


def _vol(V, T):
    P = V[T]
    return np.abs(np.linalg.det(np.stack([P[:, 1] - P[:, 0], P[:, 2] - P[:, 0], P[:, 3] - P[:, 0]], 2))) / 6


def _check_conforming(p):
    T = np.asarray(p["tets"])
    fc = Counter(tuple(sorted(t[f])) for t in T for f in FACE)
    assert set(fc.values()) <= {1, 2}
    outer = {k for k, c in fc.items() if c == 1}
    assert outer == set(map(tuple, np.sort(p["bdr_tris"], axis=1)))


def test_refinement_is_conforming_and_keeps_regions():
    from test_oracle_golden import loaded_problem
    prob = loaded_problem(1)
    rng = np.random.default_rng(0)
    marked = rng.choice(len(prob["tets"]), 25, replace=False)
    p2 = refine_problem(prob, marked)
    assert len(p2["tets"]) >= len(prob["tets"]) + 25
    _check_conforming(p2)
    for r in (0, 1):   # each material keeps its volume
        v0 = _vol(prob["verts"], prob["tets"][prob["tet_region"] == r]).sum()
        v1 = _vol(p2["verts"], p2["tets"][p2["tet_region"] == r]).sum()
        assert abs(v1 - v0) <= 1e-12 * v0
    assert _vol(p2["verts"], p2["tets"]).min() > 0
    # boundary attributes carry over: the port planes keep their area
    for a in np.unique(prob["bdr_attr"]):
        def area(p):
            t = np.asarray(p["bdr_tris"])[np.asarray(p["bdr_attr"]) == a]
            P = np.asarray(p["verts"])[t]
            return 0.5 * np.linalg.norm(np.cross(P[:, 1] - P[:, 0], P[:, 2] - P[:, 0]), axis=1).sum()
        assert abs(area(p2) - area(prob)) <= 1e-12 * area(prob)
    # refining everything twice stays conforming; no marks leaves the mesh alone
    p3 = refine_problem(refine_problem(prob, np.arange(len(prob["tets"]))), np.arange(10))
    _check_conforming(p3)
    p0 = refine_problem(prob, [])
    assert len(p0["tets"]) == len(prob["tets"])


def test_relative_change_matches_reference_formula():
    rng = np.random.default_rng(4)
    for n in (1, 2, 3):
        A = rng.normal(size=(n, n)) + 1j * rng.normal(size=(n, n))
        B = A + 1e-3 * (rng.normal(size=(n, n)) + 1j * rng.normal(size=(n, n)))
        E = np.linalg.inv(B) @ (A - B)
        assert abs(s_relative_change(A, B) - np.linalg.norm(E, axis=0).max()) < 1e-14


def test_adaptive_loop_with_oracle_step():
    """WR90 straight, ND2: the loop refines the marked elements, the change of S
    between passes falls, and the phase of S21 moves toward the exact -beta L."""
    prob = meshgen.waveguide_problem(meshgen.WR_A, meshgen.WR_B, 50e-3, 6, 3, 15, 2)
    f = 10e9

    def step(p):
        ops = fem.Operators(p)
        r = fem.solve_frequency(ops, f, return_fields=True)
        err, marked, mx = mesh_errors(ops, [h for _, h in r["fields"]], 0.1)
        return r["S"], mx, marked

    S, pf, hist = adaptive_solve(prob, step, fraction=0.1, variable="S", rel_tol=1e-12, iter_max=3)
    assert [h["iteration"] for h in hist] == [1, 2, 3] and not any(h["converged"] for h in hist)
    assert hist[0]["relative_error"] == -1 and hist[1]["relative_error"] > 0
    assert hist[2]["tets"] > hist[1]["tets"] > hist[0]["tets"]
    _check_conforming(pf)
    k0 = 2 * np.pi * f / 299792458.0
    exact = np.angle(np.exp(-1j * np.sqrt(k0 ** 2 - (np.pi / meshgen.WR_A) ** 2) * 50e-3), deg=True)
    e0 = abs(np.angle(hist[0]["S"][1, 0], deg=True) - exact)
    e2 = abs(np.angle(hist[2]["S"][1, 0], deg=True) - exact)
    assert e2 < e0
    # a loose tolerance stops at the second pass; iter_min holds it back
    _, _, h2 = adaptive_solve(prob, step, fraction=0.1, variable="S", rel_tol=1.0, iter_max=5)
    assert len(h2) == 2 and h2[-1]["converged"]
    _, _, h3 = adaptive_solve(prob, step, fraction=0.1, variable="S", rel_tol=1.0, iter_min=3, iter_max=5)
    assert len(h3) == 3 and not h3[1]["converged"] and h3[2]["converged"]


def test_refine_rejects_bad_input():
    from openparem_b200.fem3d import OpemError
    from openparem_b200 import _lib
    prob = meshgen.waveguide_problem(meshgen.WR_A, meshgen.WR_B, 50e-3, 2, 1, 2, 1)
    with pytest.raises(OpemError) as e:
        refine_problem(prob, [len(prob["tets"])])          # no such tetrahedron
    assert e.value.code == _lib.ERR_ARG
    bad = dict(prob, bdr_tris=np.array([[0, 1, 10 ** 6]]), bdr_attr=np.array([1]))
    with pytest.raises(OpemError):
        refine_problem(bad, [0])                            # vertex out of range
