"""CPU tests of the port impedance definitions (opem_port_mode_faces_z, host
only): on a rectangular coaxial line the fundamental mode is TEM, for which
the three definitions of OpenParEM2D's Mode::calculateImpedance
(fem2D.cpp:1803-1824) agree: V / I = V V* / (2 Pz*) = 2 Pz / (I I*)."""
import numpy as np
import pytest

from openparem_b200.fem3d import port_mode_faces_z, OpemError
from project_files import coax_mesh, faces_at_z

C0 = 299792458.0


def _coax_port():
    verts, tets = coax_mesh()
    fv = faces_at_z(verts, tets, 0.0)
    mode = {"kind": "FEM2D", "origin": [-12e-3, -8e-3, 0.0], "u": [1, 0, 0], "v": [0, 1, 0], "normal": [0, 0, -1],
            "a": 24e-3, "b": 16e-3, "m": 1, "n": 0,
            "vpath": ([4e-3, 0.0, 0.0], [12e-3, 0.0, 0.0])}              # inner conductor -> outer wall
    # a closed loop about the inner conductor, halfway to the outer wall
    loop = np.array([[-8e-3, -6e-3, 0.0], [8e-3, -6e-3, 0.0], [8e-3, 6e-3, 0.0], [-8e-3, 6e-3, 0.0]])
    return verts, fv, mode, loop


def test_coax_definitions_agree():
    verts, fv, mode, loop = _coax_port()
    assert len(fv) == 2 * (6 * 4 - 4)
    eps = np.ones(len(fv), dtype=complex)
    f = 3e9
    z = {d: port_mode_faces_z(verts, fv, eps, mode, 4, f, d, loop) for d in ("PV", "VI", "PI")}
    beta = z["PV"]["gamma"].imag
    assert abs(beta / (2 * np.pi * f / C0) - 1) < 1e-6           # TEM: beta = k0
    zpv, zvi, zpi = z["PV"]["Z"], z["VI"]["Z"], z["PI"]["Z"]
    assert zpv.real > 0 and abs(zpv.imag) < 1e-6 * abs(zpv)
    assert abs(abs(zvi) / zpv.real - 1) < 2e-3 and abs(zpi.real / zpv.real - 1) < 4e-3
    # the same mode in every definition; the current does not depend on the loop's size
    assert np.allclose([z[d]["gamma"] for d in z], z["PV"]["gamma"], rtol=1e-12)
    small = loop * np.array([0.75, 0.85, 1.0])
    i2 = port_mode_faces_z(verts, fv, eps, mode, 4, f, "PI", small)["I"]
    assert abs(abs(i2) / abs(z["PI"]["I"]) - 1) < 3e-3


def test_current_path_required():
    verts, fv, mode, loop = _coax_port()
    eps = np.ones(len(fv), dtype=complex)
    with pytest.raises(OpemError):
        port_mode_faces_z(verts, fv, eps, mode, 2, 3e9, "PI", None)


def test_project_impedance_definitions(tmp_path):
    """The reader takes impedance_definition and the current IntegrationPath; a
    port that uses its current is driven by its own 2D mode; VI or PI without a
    current path is an error."""
    from openparem_b200.fem3d import project_info, project_problem
    from project_files import write_coax_project
    import os
    d1 = tmp_path / "pi"
    os.makedirs(d1)
    info, _ = project_info(write_coax_project(str(d1), "PI"))
    assert info["ports"] == 2 and info["port_faces"] == 2 * 2 * (6 * 4 - 4)
    prob, _ = project_problem(str(d1 / "coax.proj"))
    assert [p["mode"]["kind"] for p in prob["ports"]] == ["FEM2D", "FEM2D"]
    # PV: the inner conductor is a hole in the rectangle's faces, so still the 2D mode
    d0 = tmp_path / "pv"
    os.makedirs(d0)
    prob, _ = project_problem(write_coax_project(str(d0), "PV"))
    assert [p["mode"]["kind"] for p in prob["ports"]] == ["FEM2D", "FEM2D"]
    d2 = tmp_path / "nocurrent"
    os.makedirs(d2)
    with pytest.raises(OpemError) as e:
        project_info(write_coax_project(str(d2), "PI", with_current=False))
    assert "current path" in str(e.value)


def test_multi_conductor_ports_rejected(tmp_path):
    """A port with two Line blocks (two modes, as the reference's differential
    pairs) needs the multi-mode 2D solve: the reader says so instead of reading
    one mode."""
    from openparem_b200.fem3d import project_info
    from project_files import write_project, coax_mesh
    verts, tets = coax_mesh()
    spec = {"paths": [{"name": "p1", "points": [(-12e-3, -8e-3, 0.0), (12e-3, -8e-3, 0.0), (12e-3, 8e-3, 0.0),
                                                 (-12e-3, 8e-3, 0.0)], "closed": True},
                      {"name": "v1", "points": [(4e-3, 0.0, 0.0), (12e-3, 0.0, 0.0)], "closed": False}],
            "boundaries": [],
            "ports": [{"name": "1", "paths": ["+p1"], "impedance_definition": "PV", "impedance_calculation": "line",
                       "lines": [{"Sport": 1, "integration": [{"type": "voltage", "paths": ["+v1"]}]},
                                 {"Sport": 2, "integration": [{"type": "voltage", "paths": ["-v1"]}]}]}]}
    proj = write_project(str(tmp_path), "pair", verts, tets, 1, {1: "air"}, spec,
                         {"air": {"er": 1.0, "mur": 1.0, "tand": 0.0, "Rz": 0.0}}, 1, [3e9])
    with pytest.raises(OpemError) as e:
        project_info(proj)
    assert "multi-conductor" in str(e.value)


def test_library_equals_oracle_definitions(tmp_path):
    """The library's current and impedance under each definition equal the
    oracle's restatement (oracle/portmode.py) on the coaxial project's port, as
    read by the project reader (its current path included)."""
    from oracle import fem
    from oracle.materials import relative_eps
    from oracle.nd_basis import FACES
    from oracle.portmode import Fem2DMode
    from openparem_b200.fem3d import project_problem
    from project_files import write_coax_project
    prob, fr = project_problem(write_coax_project(str(tmp_path), "PI"))
    mode = prob["ports"][0]["mode"]
    assert mode["zdef"] == "PI" and mode["ipath"].shape == (4, 3) and mode["ipath_closed"]
    ops = fem.Operators(prob)
    topo, faces = ops.topo, ops.ports[0]["faces"]
    fv = np.array([topo.tets[topo.face_owner[x]][list(FACES[topo.face_lface[x]])] for x in faces])
    reg = np.asarray(prob["tet_region"])[topo.face_owner[faces]]
    f = fr[0]
    eps = relative_eps(f, prob["eps_r"][reg], prob["tand"][reg], prob["sigma"][reg])
    for zdef in ("PV", "VI", "PI"):
        m = dict(mode, zdef=zdef)
        om = Fem2DMode(prob, topo, faces, m, f)
        lib = port_mode_faces_z(prob["verts"], fv, eps, m, m["nsub"], f, zdef, m["ipath"], order=m["order2d"])
        assert abs(lib["Z"] - om.Z) <= 1e-10 * abs(om.Z), (zdef, lib["Z"], om.Z)
        # V and I scale with the mode's normalisation; their ratio does not
        assert abs(lib["V"] / lib["I"] - om.V / om.I) <= 1e-10 * abs(om.V / om.I)
