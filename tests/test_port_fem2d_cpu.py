"""Ports driven by their own 2D mode (CPU: oracle and the library's host side).

The reference drives every port with the mode its 2D solver finds on the port
faces (port.cpp:5081-5176, :5302-5453, :3234-3341).  opem_problem_set_port_fem2d
does the same in-process: the port faces split nsub x nsub, the fundamental
Lee-Sun-Cendes mode (opem_port_mode_2d), H_t = n x (gamma e_t + grad e_z)/(j w mu),
V along the voltage path and Z = V V*/(2 Pz*).  Here:
  * the library's mode (opem_port_mode_faces) equals the oracle's
    (oracle/portmode.py) on the slab-loaded WR90 ports, with first- and
    second-order 2D elements: gamma and Z to 1e-10,
    E_t and H_t at points of the port faces to 1e-10 (up to the mode's
    arbitrary complex scale, which S does not depend on);
  * on the empty guide the oracle's S with 2D-mode ports converges to the S
    with the analytic TE10 at second order in the split;
  * through the project reader (which picks second-order 2D modes on a split of
    the port faces near 1024 triangles for ports whose faces see more than one
    material) the oracle at the reference's ND6 on its slab-loaded WR90 project
    comes within 1.2e-6 deg of the reference's found arg S21 and 5e-10 dB of
    its |S21| (the test allows 5e-6 deg and 1e-8 dB).
"""
import os

import numpy as np
import pytest

from oracle import fem
from oracle.materials import relative_eps
from oracle.nd_basis import FACES
from oracle.portmode import Fem2DMode
from openparem_b200.fem3d import port_mode_faces, project_problem
from project_files import reference_project

HERE = os.path.dirname(os.path.abspath(__file__))


def loaded(order):
    from test_oracle_golden import loaded_problem
    return loaded_problem(order)


@pytest.mark.parametrize("order,nsub", [(1, 6), (2, 4)])
def test_library_mode_equals_oracle(order, nsub):
    prob = loaded(1)
    ops = fem.Operators(prob)
    topo = ops.topo
    f = 8.3e9
    rng = np.random.default_rng(3)
    for k in range(2):
        mode = dict(prob["ports"][k]["mode"], kind="FEM2D", nsub=nsub, order2d=order)
        faces = ops.ports[k]["faces"]
        om = Fem2DMode(prob, topo, faces, mode, f)
        fv = np.array([topo.tets[topo.face_owner[x]][list(FACES[topo.face_lface[x]])] for x in faces])
        reg = np.asarray(prob["tet_region"])[topo.face_owner[faces]]
        eps = relative_eps(f, prob["eps_r"][reg], prob["tand"][reg], prob["sigma"][reg])
        pf = rng.integers(0, len(faces), 300)
        a = rng.random((300, 2))
        a = np.where(a.sum(1, keepdims=True) > 1, 1 - a[:, ::-1], a)
        met, E, Hy = port_mode_faces(prob["verts"], fv, eps, mode, nsub, f, pf, a, order=order)
        V = np.asarray(prob["verts"])
        X = V[fv[pf, 0]] + a[:, 0:1] * (V[fv[pf, 1]] - V[fv[pf, 0]]) + a[:, 1:2] * (V[fv[pf, 2]] - V[fv[pf, 0]])
        Eo = np.concatenate([om.metrics()["Et"].at_face(pf[i], a[i:i + 1], X[i:i + 1]) for i in range(len(pf))])
        Ho = np.concatenate([om.metrics()["Ht"].at_face(pf[i], a[i:i + 1], X[i:i + 1]) for i in range(len(pf))])
        y = om.gamma / (1j * 2 * np.pi * f * 4e-7 * np.pi * om.mu_port)
        c = np.vdot(E.ravel(), Eo.ravel()) / np.vdot(E.ravel(), E.ravel())   # the modes' relative scale
        assert abs(met["gamma"] - om.gamma) <= 1e-10 * abs(om.gamma)
        assert abs(met["Z"] - om.Z) <= 1e-10 * abs(om.Z)
        assert abs(c * met["V"] - om.V) <= 1e-10 * abs(om.V)
        assert np.abs(Eo - c * E).max() <= 1e-10 * np.abs(Eo).max()
        assert np.abs(Ho - c * y * Hy).max() <= 1e-10 * np.abs(Ho).max()
        # the loaded guide's mode is slower than the empty guide's TE10
        assert om.gamma.imag > np.sqrt((2 * np.pi * f / 299792458.0) ** 2 * 1.0006 - (np.pi / 22.86e-3) ** 2)


def test_empty_guide_converges_to_analytic_te10():
    from test_oracle_golden import wr90_problem
    prob = wr90_problem(2)
    ref = fem.solve_frequency(fem.Operators(prob), 9e9)["S"]
    errs = []
    for nsub in (2, 4, 8):
        p2 = dict(prob)
        p2["ports"] = [{"mode": dict(p["mode"], kind="FEM2D", nsub=nsub)} for p in prob["ports"]]
        S = fem.solve_frequency(fem.Operators(p2), 9e9)["S"]
        errs.append(np.abs(S - ref).max())
    assert errs[2] < 1e-3
    assert errs[1] / errs[2] > 3.0      # second order in the split


def test_reader_loaded_project_nd6_near_reference(tmp_path):
    """The reader drives the reference's slab-loaded project's ports by order-6
    modes on the unsplit port faces, the reference's own 2D problem; the oracle
    then reproduces the reference's found arg S21 to 2e-7 deg and |S21| to 1e-10
    dB (with second-order modes on faces split 10 x 10: 1.2e-6 deg)."""
    proj, rec = reference_project(str(tmp_path), "straight-loaded")
    prob, fr = project_problem(proj)
    assert [p["mode"]["kind"] for p in prob["ports"]] == ["FEM2D", "FEM2D"]
    assert all(p["mode"]["nsub"] == 1 and p["mode"]["order2d"] == 6 for p in prob["ports"])
    assert np.allclose(fr, [8.3e9])
    S = fem.solve_frequency(fem.Operators(prob), 8.3e9)["S"]
    import json
    with open(os.path.join(HERE, "golden", "wr90_expected.json")) as f:
        cases = json.load(f)["cases"]["./WR90/straight-loaded/straight-loaded.proj"]
    found = [v["found"] for v in cases.values() if v["variable"] == "argS(deg)" and v["portOut"] == 2
             and v["portIn"] == 1][0]
    found_db = [v["found"] for v in cases.values() if v["variable"] == "magS(dB)" and v["portOut"] == 2
                and v["portIn"] == 1][0]
    assert abs(np.angle(S[1, 0], deg=True) - found) < 2e-7
    assert abs(20 * np.log10(abs(S[1, 0])) - found_db) < 1e-10
    assert 20 * np.log10(abs(S[0, 0])) < -100


@pytest.mark.parametrize("order,nsub", [(3, 1), (4, 1), (6, 1), (3, 2)])
def test_library_order_p_mode_equals_oracle(order, nsub):
    """Order-p port modes (the reference's 2D spaces at mesh.order p): the
    library's gamma, Z, V and fields equal the oracle's restatement
    (oracle/port2d_pp.py) on the slab-loaded guide's ports."""
    prob = loaded(1)
    ops = fem.Operators(prob)
    topo = ops.topo
    f = 8.3e9
    rng = np.random.default_rng(5)
    for k in range(2):
        mode = dict(prob["ports"][k]["mode"], kind="FEM2D", nsub=nsub, order2d=order)
        faces = ops.ports[k]["faces"]
        om = Fem2DMode(prob, topo, faces, mode, f)
        fv = np.array([topo.tets[topo.face_owner[x]][list(FACES[topo.face_lface[x]])] for x in faces])
        reg = np.asarray(prob["tet_region"])[topo.face_owner[faces]]
        eps = relative_eps(f, prob["eps_r"][reg], prob["tand"][reg], prob["sigma"][reg])
        pf = rng.integers(0, len(faces), 150)
        a = rng.random((150, 2))
        a = np.where(a.sum(1, keepdims=True) > 1, 1 - a[:, ::-1], a)
        met, E, Hy = port_mode_faces(prob["verts"], fv, eps, mode, nsub, f, pf, a, order=order)
        V = np.asarray(prob["verts"])
        X = V[fv[pf, 0]] + a[:, 0:1] * (V[fv[pf, 1]] - V[fv[pf, 0]]) + a[:, 1:2] * (V[fv[pf, 2]] - V[fv[pf, 0]])
        Eo = np.concatenate([om.metrics()["Et"].at_face(pf[i], a[i:i + 1], X[i:i + 1]) for i in range(len(pf))])
        Ho = np.concatenate([om.metrics()["Ht"].at_face(pf[i], a[i:i + 1], X[i:i + 1]) for i in range(len(pf))])
        y = om.gamma / (1j * 2 * np.pi * f * 4e-7 * np.pi * om.mu_port)
        c = np.vdot(E.ravel(), Eo.ravel()) / np.vdot(E.ravel(), E.ravel())
        assert abs(met["gamma"] - om.gamma) <= 1e-10 * abs(om.gamma)
        assert abs(met["Z"] - om.Z) <= 1e-10 * abs(om.Z)
        assert abs(c * met["V"] - om.V) <= 1e-10 * abs(om.V)
        assert np.abs(Eo - c * E).max() <= 1e-10 * np.abs(Eo).max()
        assert np.abs(Ho - c * y * Hy).max() <= 1e-10 * np.abs(Ho).max()


def test_order_p_modes_converge_to_analytic():
    """The order-p 2D solve (oracle/port2d_pp.py) reproduces the order-1 and
    order-2 solvers' spaces exactly and converges with p: TE10 of an empty guide
    and the slab-loaded guide's dispersion relation."""
    from oracle.port2d import rect_mesh, solve_mode, solve_mode_p2, slab_beta
    from oracle.port2d_pp import solve_mode_pp
    a, b = 22.86e-3, 10.16e-3
    pts, tris = rect_mesh(a, b, 8, 4)
    f = 10e9
    assert abs(solve_mode_pp(pts, tris, f, 1.0, p=1)[0] - solve_mode(pts, tris, f, 1.0)[0]) < 1e-12 * 160
    assert abs(solve_mode_pp(pts, tris, f, 1.0, p=2)[0] - solve_mode_p2(pts, tris, f, 1.0)[0]) < 1e-12 * 160
    exact = np.sqrt((2 * np.pi * f / 299792458.0) ** 2 - (np.pi / a) ** 2)
    errs = [abs(solve_mode_pp(pts, tris, f, 1.0, p=p)[0] - exact) / exact for p in (2, 3, 4)]
    assert errs[0] < 1e-5 and errs[1] < 1e-8 and errs[2] < 1e-10
    w = 4e-3
    pts2, tris2 = rect_mesh(a, b, 8, 4, x_breaks=(-w / 2, w / 2))
    cen = pts2[tris2].mean(1)
    eps = np.where(np.abs(cen[:, 0]) < w / 2, 2.2, 1.0)
    ex2 = slab_beta(a, w, 2.2, f)
    assert abs(solve_mode_pp(pts2, tris2, f, eps, p=6)[0] - ex2) / ex2 < 1e-11


def test_higher_modes_library_equals_oracle_and_analytic():
    """Modes beyond the fundamental (subspace iteration in the library, shifted
    Arnoldi in the oracle): on an empty WR90 cross-section at 16 GHz the three
    leading modes TE10, TE20 and TE01 come out in decreasing beta with the
    analytic propagation constants (order-4 elements on the unsplit port faces:
    2e-8 and better), and the library's gamma and Z equal the oracle's."""
    from openparem_b200 import meshgen
    from openparem_b200.fem3d import port_mode_faces_z
    from project_files import faces_at_z
    a, b = meshgen.WR_A, meshgen.WR_B
    prob = meshgen.waveguide_problem(a, b, 20e-3, 6, 3, 4, 1)
    ops = fem.Operators(prob)
    topo = ops.topo
    faces = ops.ports[0]["faces"]
    fv = np.array([topo.tets[topo.face_owner[x]][list(FACES[topo.face_lface[x]])] for x in faces])
    f = 16e9
    k0 = 2 * np.pi * f / 299792458.0
    kc = sorted([np.pi / a, 2 * np.pi / a, np.pi / b])
    base = dict(prob["ports"][0]["mode"], kind="FEM2D", nsub=1, order2d=4)
    eps = np.ones(len(fv), dtype=complex)
    for mi in range(3):
        lib = port_mode_faces_z(prob["verts"], fv, eps, base, 1, f, order=4, mode_index=mi)
        om = Fem2DMode(prob, topo, faces, dict(base, mode_index=mi), f)
        exact = np.sqrt(k0 ** 2 - kc[mi] ** 2)
        assert abs(lib["gamma"].imag - exact) <= 3e-8 * exact, (mi, lib["gamma"], exact)
        assert abs(lib["gamma"] - om.gamma) <= 1e-9 * abs(om.gamma)
        assert abs(lib["Z"] - om.Z) <= 1e-7 * abs(om.Z) + 1e-9
