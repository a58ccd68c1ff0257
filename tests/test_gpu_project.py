"""GPU: a problem read from OpenParEM3D project files (gmsh 2.2 mesh, ports file,
materials database, .proj) solves to the same S as the same guide built in
memory (|dS| <= 1e-10, solver rtol 1e-12)."""
import numpy as np
import pytest

from openparem_b200 import meshgen, Fem3D, default_opts
from openparem_b200.fem3d import Context
from project_files import write_guide_project

pytestmark = pytest.mark.gpu


def test_project_matches_in_memory_problem(tmp_path):
    ctx = Context(0)
    proj = write_guide_project(str(tmp_path), order=1)
    F, freqs = Fem3D.from_project(proj, context=ctx)
    assert np.allclose(freqs, [9e9, 10e9, 10.5e9, 11e9])
    F.assemble()
    G = Fem3D(meshgen.waveguide_problem(meshgen.WR_A, meshgen.WR_B, 50e-3, 6, 3, 15, 1), context=ctx).assemble()
    o = default_opts(rtol=1e-12, restart=200)
    for f in (9e9, 10.5e9):
        S1, _, st1 = F.solve(f, o)
        S2, _, _ = G.solve(f, o)
        assert st1["converged"] == 1
        assert np.abs(S1 - S2).max() <= 1e-10, f
    # an order override reads the same files at ND2
    F2, _ = Fem3D.from_project(proj, order=2, context=ctx)
    S3, _, st3 = F2.assemble().solve(10e9, o)
    assert st3["converged"] == 1 and np.abs(S3).max() <= 1 + 1e-9


@pytest.mark.parametrize("name", ["straight-rotated-xyz", "shorted", "opened"])
def test_reference_projects_match_oracle(tmp_path, name):
    """The reference's rotated, shorted and opened WR90 projects, read by the
    C++ reader, solve on the device (ND2) to the oracle's S on the problem the
    same reader produced (|dS| <= 1e-8, solver rtol 1e-12)."""
    from oracle import fem
    from openparem_b200.fem3d import project_problem
    from project_files import reference_project
    proj, _ = reference_project(str(tmp_path), name)
    F, _ = Fem3D.from_project(proj, order=2, context=Context(0))
    F.assemble()
    prob, _ = project_problem(proj, order=2)
    ops = fem.Operators(prob)
    o = default_opts(rtol=1e-12, restart=200, maxits=6000, h_rtol=1e-13)
    for f in (9e9, 11e9):
        S, _, st = F.solve(f, o)
        assert st["converged"] == 1
        ref = fem.solve_frequency(ops, f)["S"]
        assert np.abs(S - ref).max() <= 1e-8, (name, f, S, ref)


def test_loaded_project_2d_mode_ports_match_oracle(tmp_path):
    """The reference's slab-loaded WR90 project: its ports see air and teflon, so
    the reader drives them by their own 2D modes (solved per frequency on the
    port faces with 2D elements of the problem's order).  ND2 on the device, plain FP64 and the batched
    mixed sweep, against the oracle on the problem the same reader produced
    (|dS| <= 1e-8 plain with solver rtol 1e-12; <= 1e-6 mixed)."""
    from oracle import fem
    from openparem_b200 import _lib
    from openparem_b200.fem3d import project_problem
    from project_files import reference_project
    proj, _ = reference_project(str(tmp_path), "straight-loaded")
    F, _ = Fem3D.from_project(proj, order=2, context=Context(0))
    F.assemble()
    prob, _ = project_problem(proj, order=2)
    assert [p["mode"]["kind"] for p in prob["ports"]] == ["FEM2D", "FEM2D"]
    ops = fem.Operators(prob)
    o = default_opts(rtol=1e-12, restart=200, maxits=6000, h_rtol=1e-13)
    fr = [8.3e9, 9.5e9]
    refs = [fem.solve_frequency(ops, f)["S"] for f in fr]
    for f, ref in zip(fr, refs):
        S, _, st = F.solve(f, o)
        assert st["converged"] == 1
        assert np.abs(S - ref).max() <= 1e-8, (f, S, ref)
    Sm, stm = F.sweep(fr, default_opts(precision=_lib.PREC_MIXED, rtol=1e-10))
    for i in range(len(fr)):
        assert np.abs(Sm[i] - refs[i]).max() <= 1e-6


def test_default_copper_walls_project_matches_oracle(tmp_path):
    """The reference's straight-lossy project: materials.default.boundary copper
    makes every wall no port claims a copper surface impedance.  ND2 on the
    device against the oracle on the problem the same reader produced
    (|dS| <= 1e-8, solver rtol 1e-12)."""
    from oracle import fem
    from openparem_b200.fem3d import project_problem
    from project_files import reference_project
    proj, _ = reference_project(str(tmp_path), "straight-lossy")
    F, fr = Fem3D.from_project(proj, order=2, context=Context(0))
    F.assemble()
    prob, _ = project_problem(proj, order=2)
    assert prob["boundaries"][1]["type"] == "impedance"
    S, _, st = F.solve(fr[0], default_opts(rtol=1e-12, restart=200, maxits=6000, h_rtol=1e-13))
    assert st["converged"] == 1
    ref = fem.solve_frequency(fem.Operators(prob), fr[0])["S"]
    assert np.abs(S - ref).max() <= 1e-8


def test_polygon_port_project_matches_oracle(tmp_path):
    """A guide of L-shaped cross-section whose port paths are six-point
    outlines: the reader drives both ports by their own 2D modes.  ND1 on the
    device, plain FP64 and the batched mixed sweep, against the oracle on the
    problem the same reader produced (|dS| <= 1e-8 plain with solver rtol
    1e-12; <= 1e-6 mixed); the straight guide passes the wave (|S21| > 0.99)."""
    from oracle import fem
    from openparem_b200 import _lib
    from openparem_b200.fem3d import project_problem
    from project_files import write_lguide_project
    proj = write_lguide_project(str(tmp_path))
    F, fr = Fem3D.from_project(proj, context=Context(0))
    F.assemble()
    prob, _ = project_problem(proj)
    ref = fem.solve_frequency(fem.Operators(prob), fr[0])["S"]
    S, _, st = F.solve(fr[0], default_opts(rtol=1e-12, restart=200, maxits=6000, h_rtol=1e-13))
    assert st["converged"] == 1
    assert np.abs(S - ref).max() <= 1e-8, (S, ref)
    assert abs(S[1, 0]) > 0.99
    Sm, _ = F.sweep([fr[0]], default_opts(precision=_lib.PREC_MIXED, rtol=1e-10))
    assert np.abs(Sm[0] - ref).max() <= 1e-6


def test_coax_project_impedance_definitions(tmp_path):
    """A rectangular coaxial line read from projects whose ports use the PI, VI
    and PV impedance definitions (current paths about the inner conductor): the
    device solve's port impedance equals the host 2D mode's under the same
    definition (the same faces unsplit, second-order 2D elements), the three
    definitions agree to 5 % on this TEM line (with H_t projected onto the edge
    space and Pz by the order-(p-1) nodal rule, as the reference forms them, PI
    and VI sit 3.0 % and 1.5 % from PV on these 4 mm cells, 0.33 % and 0.16 % on
    1 mm cells), and the line passes the wave (|S21| > 0.99)."""
    import os
    from openparem_b200.fem3d import port_mode_faces_z
    from project_files import write_coax_project, coax_mesh, faces_at_z
    verts, tets = coax_mesh()
    fv = faces_at_z(verts, tets, 0.0)
    mode = {"kind": "FEM2D", "origin": [-12e-3, -8e-3, 0.0], "u": [1, 0, 0], "v": [0, 1, 0], "normal": [0, 0, -1],
            "a": 24e-3, "b": 16e-3, "m": 1, "n": 0, "vpath": ([4e-3, 0.0, 0.0], [12e-3, 0.0, 0.0])}
    loop = np.array([[-8e-3, -6e-3, 0.0], [8e-3, -6e-3, 0.0], [8e-3, 6e-3, 0.0], [-8e-3, 6e-3, 0.0]])
    ctx = Context(0)
    zo = {}
    for zdef in ("PI", "VI", "PV"):
        d = tmp_path / zdef
        os.makedirs(d)
        F, fr = Fem3D.from_project(write_coax_project(str(d), zdef), order=2, context=ctx)
        F.assemble()
        S, Zo, st = F.solve(fr[0], default_opts(rtol=1e-10, restart=200, maxits=6000))
        assert st["converged"] == 1 and abs(S[1, 0]) > 0.99, (zdef, S)
        host = port_mode_faces_z(verts, fv, np.ones(len(fv), dtype=complex), mode, 1, fr[0], zdef, loop)["Z"]
        assert abs(Zo[0] / host - 1) < 1e-8, (zdef, Zo, host)
        zo[zdef] = Zo[0]
    assert abs(zo["PI"] / zo["PV"] - 1) < 5e-2 and abs(zo["VI"] / zo["PV"] - 1) < 5e-2
