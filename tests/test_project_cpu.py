"""CPU tests of the OpenParEM3D project reader (opem_project_info: host only)."""
import os

import numpy as np
import pytest

from openparem_b200.fem3d import project_info, OpemError
from project_files import write_guide_project


def test_synthetic_guide_project(tmp_path):
    proj = write_guide_project(str(tmp_path), copper_wall=True)
    info, fr = project_info(proj)
    assert info["tets"] == 1620 and info["regions"] == 1 and info["ports"] == 2 and info["order"] == 1
    assert info["port_faces"] == 2 * 6 * 3 * 2
    assert info["boundary_faces"] == 3 * 15 * 2               # the x = a/2 wall, copper
    assert info["pec_faces"] == info["exterior_faces"] - info["port_faces"] - info["boundary_faces"]
    assert np.allclose(fr, [9e9, 10e9, 10.5e9, 11e9])
    info3, _ = project_info(proj, order=3)
    assert info3["order"] == 3


def test_project_errors(tmp_path):
    proj = write_guide_project(str(tmp_path))
    os.remove(os.path.join(str(tmp_path), "materials.txt"))
    with pytest.raises(OpemError) as e:
        project_info(proj)
    assert "material" in str(e.value)
    with pytest.raises(OpemError):
        project_info(os.path.join(str(tmp_path), "missing.proj"))


# The reference's OpenParEM source tree, when one is mounted: its location comes
# from OPEM_REFERENCE_ROOT (unset: the test is skipped).
_ROOT = os.environ.get("OPEM_REFERENCE_ROOT", "")
REF = os.path.join(_ROOT, "regression/OpenParEM3D/WR90/straight/straight.proj") if _ROOT else ""


@pytest.mark.skipif(not REF or not os.path.exists(REF), reason="the reference tree is not mounted here")
def test_reference_wr90_straight_project():
    """The reference's own regression project reads: 282 tets, two TE10 ports,
    its three frequency points, mesh order 6."""
    info, fr = project_info(REF)
    assert info["tets"] == 282 and info["ports"] == 2 and info["order"] == 6
    assert info["port_faces"] > 0 and info["pec_faces"] > 0
    assert np.allclose(fr, [9e9, 9.999999999e9, 11e9])


def test_project_refinement_settings(tmp_path):
    from openparem_b200.fem3d import project_refinement
    proj = write_guide_project(str(tmp_path))
    r = project_refinement(proj)
    assert r == {"fraction": 0.005, "variable": "SandH", "rel_tol": 0.02, "abs_tol": 1e-6, "iter_min": 1,
                 "iter_max": 10, "passes": 1, "frequency": "highlow"}
    with open(proj, "a") as f:
        f.write("refinement.variable            S   // on S only\nrefinement.iteration.max       30\n"
                "refinement.relative.tolerance  0.001\nmesh.3D.refinement.fraction    0.05\n")
    r = project_refinement(proj)
    assert (r["variable"], r["iter_max"], r["rel_tol"], r["fraction"]) == ("S", 30, 0.001, 0.05)


def test_project_value_missing(tmp_path):
    from openparem_b200.fem3d import project_value
    proj = write_guide_project(str(tmp_path))
    assert project_value(proj, "mesh.order") == "1"
    assert project_value(proj, "no.such.key", "x") == "x"
    assert project_value(os.path.join(str(tmp_path), "none.proj"), "mesh.order") is None


def test_frequency_plans(tmp_path):
    """linear, linear.refine, log and point entries expand as the reference's
    FrequencyPlan does (repeated step / repeated factor up to stop (1 + 1e-12))."""
    proj = write_guide_project(str(tmp_path))
    with open(proj, "a") as f:
        f.write("frequency.plan.log             1e9,1e10,4\n"
                "frequency.plan.linear.refine   20e9,22e9,1e9   // refined\n")
    _, fr = project_info(proj)
    logs = [1e9 * 10 ** (k / 4) for k in range(5)]
    expect = sorted(set([9e9, 10e9, 10.5e9, 11e9, 20e9, 21e9, 22e9]) | set(logs))
    assert len(fr) == len(expect) and np.allclose(fr, expect, rtol=1e-12)


def test_frequency_plan_duplicates_and_integer_points_per_decade(tmp_path):
    """Points whose relative difference is below 1e-14 are one point, points
    1e-13 apart stay two (FrequencyPlan::eliminateDuplicates); a log plan's
    points per decade must be an integer, as the reference's project parser
    requires."""
    proj = write_guide_project(str(tmp_path))
    with open(proj, "a") as f:
        f.write("frequency.plan.point           12e9\n"
                f"frequency.plan.point           {12e9 * (1 + 2e-16)!r}\n"
                f"frequency.plan.point           {13e9 * (1 + 1e-13)!r}\n"
                "frequency.plan.point           13e9\n")
    _, fr = project_info(proj)
    assert np.sum(np.abs(np.asarray(fr) - 12e9) < 1e3) == 1
    assert np.sum(np.abs(np.asarray(fr) - 13e9) < 1e3) == 2
    d2 = tmp_path / "b"
    d2.mkdir()
    proj2 = write_guide_project(str(d2))
    with open(proj2, "a") as f:
        f.write("frequency.plan.log             1e9,1e10,2.5\n")
    with pytest.raises(Exception):
        project_info(proj2)


def test_polygon_port_paths(tmp_path):
    """Port paths that are not rectangles (the six-point outline of an L-shaped
    guide) are read: their faces are the port's, and the port is driven by the
    fundamental mode of its own faces, with an outward normal."""
    from openparem_b200.fem3d import project_problem
    from project_files import write_lguide_project
    proj = write_lguide_project(str(tmp_path))
    info, fr = project_info(proj)
    assert info["tets"] == 1080 and info["ports"] == 2
    assert info["port_faces"] == 2 * 18 * 2                 # 3/4 of the 6 x 4 cross-section, two triangles a quad
    assert info["pec_faces"] == info["exterior_faces"] - info["port_faces"]
    prob, _ = project_problem(proj)
    modes = [p["mode"] for p in prob["ports"]]
    assert [m["kind"] for m in modes] == ["FEM2D", "FEM2D"] and all(m["nsub"] > 0 for m in modes)
    assert np.allclose(modes[0]["normal"], [0, 0, -1]) and np.allclose(modes[1]["normal"], [0, 0, 1])
    assert np.allclose([modes[0]["a"], modes[0]["b"]], [24e-3, 16e-3])   # the outline's bounding box
    assert np.allclose(modes[1]["vpath"][0], [-6e-3, -8e-3, 40e-3])


@pytest.mark.skipif(not _ROOT or not os.path.isdir(os.path.join(_ROOT, "regression", "OpenParEM3D")),
                    reason="the reference tree is not mounted here")
def test_reference_regression_projects_read():
    """Every regression project of the reference reads (80 of 88, gmsh and MFEM
    mesh formats), except those the reader declines with a reason:
    multi-conductor ports (several Line / Mode blocks, or integration paths
    summed from several paths) and a mesh file the tree does not hold."""
    import glob
    from openparem_b200.fem3d import project_info
    paths = sorted(glob.glob(os.path.join(_ROOT, "regression", "OpenParEM3D", "*", "*", "*.proj")))
    ok, declined = 0, 0
    for p in paths:
        try:
            info, _ = project_info(p)
            assert info["tets"] > 0 and info["ports"] >= 1
            ok += 1
        except OpemError as e:
            msg = str(e)
            assert ("multi-conductor" in msg or "summed from several paths" in msg or "no tetrahedra" in msg
                    or "cannot read mesh" in msg), (p, msg)
            declined += 1
    assert ok >= 80 and ok + declined == len(paths)


def test_mfem_format_mesh_reads_as_gmsh(tmp_path):
    """A project whose mesh is in MFEM's format (with the reference's regions
    file materials_for_<mesh>) reads to the same problem as the same mesh in
    gmsh 2.2: vertices, tetrahedra, regions and materials, boundary
    classification and ports."""
    from openparem_b200 import meshgen
    from openparem_b200.fem3d import project_problem
    from project_files import write_mfem_mesh
    proj = write_guide_project(str(tmp_path))
    pg, fg = project_problem(proj)
    verts, tets = meshgen.box_kuhn(meshgen.WR_A, meshgen.WR_B, 50e-3, 6, 3, 15)
    d2 = tmp_path / "mfem"
    os.makedirs(d2)
    for fn in os.listdir(tmp_path):
        if fn.endswith((".proj", ".txt")):
            with open(tmp_path / fn) as a, open(d2 / fn, "w") as b:
                b.write(a.read())
    write_mfem_mesh(str(d2 / "guide.msh"), verts, tets, 1, {1: "air"})
    pm, fm = project_problem(str(d2 / "guide.proj"))
    for k in ("verts", "tets", "tet_region", "bdr_tris", "bdr_attr", "eps_r", "mu_r"):
        assert np.array_equal(np.asarray(pg[k]), np.asarray(pm[k])), k
    assert np.allclose(fg, fm) and len(pm["ports"]) == 2
    os.remove(d2 / "materials_for_guide.msh")
    with pytest.raises(OpemError) as e:
        project_problem(str(d2 / "guide.proj"))
    assert "regions file" in str(e.value)
