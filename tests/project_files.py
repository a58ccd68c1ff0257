"""Writers of small OpenParEM3D-format project files (gmsh 2.2 mesh, ports file,
materials database, .proj) for the project-reader tests."""
import os

import numpy as np

from openparem_b200 import meshgen


def write_gmsh22(path, verts, tets, tag=1, name="air", names=None):
    """tag: one physical volume tag, or one per tetrahedron (then names maps
    tag -> physical name)."""
    tags = np.broadcast_to(np.asarray(tag, dtype=np.int64), (len(tets),))
    names = names if names is not None else {int(tag): name}
    with open(path, "w") as f:
        f.write("$MeshFormat\n2.2 0 8\n$EndMeshFormat\n")
        f.write(f"$PhysicalNames\n{len(names)}\n")
        for t, nm in sorted(names.items()):
            f.write(f'3 {int(t)} "{nm}"\n')
        f.write("$EndPhysicalNames\n")
        f.write(f"$Nodes\n{len(verts)}\n")
        for i, v in enumerate(verts):
            f.write(f"{i + 1} {float(v[0]):.17g} {float(v[1]):.17g} {float(v[2]):.17g}\n")
        f.write("$EndNodes\n")
        f.write(f"$Elements\n{len(tets)}\n")
        for e, t in enumerate(tets):
            f.write(f"{e + 1} 4 2 {tags[e]} 1 {t[0] + 1} {t[1] + 1} {t[2] + 1} {t[3] + 1}\n")
        f.write("$EndElements\n")


def write_ports_file(path, spec):
    """A ports file from plain data: spec = {"paths": [{name, points, closed}],
    "boundaries": [{name, type, material, paths}], "ports": [{name, paths,
    impedance_definition, impedance_calculation, lines: [{Sport, integration:
    [{type, paths}]}]}]}."""
    out = ["#OpenParEMports 1.0", ""]
    for pth in spec["paths"]:
        out.append("Path")
        out.append(f"   name={pth['name']}")
        for x in pth["points"]:
            out.append(f"   point=({x[0]!r},{x[1]!r},{x[2]!r})")
        out.append(f"   closed={'true' if pth['closed'] else 'false'}")
        out += ["EndPath", ""]
    for b in spec["boundaries"]:
        out += ["Boundary", f"   name={b['name']}", f"   type={b['type']}"]
        if b.get("material"):
            out.append(f"   material={b['material']}")
        out += [f"   path={q}" for q in b["paths"]]
        out += ["EndBoundary", ""]
    for p in spec["ports"]:
        out += ["Port", f"   name={p['name']}"]
        out += [f"   path={q}" for q in p["paths"]]
        for k in ("impedance_definition", "impedance_calculation"):
            if p.get(k):
                out.append(f"   {k}={p[k]}")
        for ln in p["lines"]:
            blk = ln.get("block", "Line")
            out += [f"   {blk}", f"      Sport={ln['Sport']}"]
            for ip in ln["integration"]:
                out += ["      IntegrationPath", f"         type={ip['type']}"]
                out += [f"         path={q}" for q in ip["paths"]]
                out.append("      EndIntegrationPath")
            out.append(f"   End{blk}")
        out += ["EndPort", ""]
    with open(path, "w") as f:
        f.write("\n".join(out) + "\n")


def write_materials(path, mats):
    """A materials database with one temperature=any / frequency=any entry per material."""
    with open(path, "w") as f:
        f.write("#OpenParEMmaterials 1.0\n\n")
        for name, m in mats.items():
            body = "\n".join(f"         {k}={v!r}" for k, v in m.items())
            f.write(f"Material\n   name={name}\n   Temperature\n      temperature=any\n      Frequency\n"
                    f"         frequency=any\n{body}\n      EndFrequency\n   EndTemperature\n"
                    f"   Source\n   EndSource\nEndMaterial\n\n")


def write_project(d, stem, verts, tets, phys, names, ports_spec, materials, order, freqs, default_boundary="PEC",
                  freq_linear=(), reference_impedance=0.0):
    """A complete project in directory d (stem.proj, stem.msh, stem_ports.txt,
    materials.txt); returns the .proj path."""
    write_gmsh22(os.path.join(d, stem + ".msh"), verts, tets, tag=phys, names=names)
    write_ports_file(os.path.join(d, stem + "_ports.txt"), ports_spec)
    write_materials(os.path.join(d, "materials.txt"), materials)
    proj = os.path.join(d, stem + ".proj")
    with open(proj, "w") as f:
        f.write("#OpenParEM3Dproject 1.0\n\n")
        f.write(f"mesh.file                      {stem}.msh\nmesh.order                     {order}\n")
        f.write(f"port.definition.file           {stem}_ports.txt\n")
        f.write("materials.global.path          ./\nmaterials.global.name          materials.txt\n")
        f.write("materials.local.path           ./\nmaterials.local.name           //local_materials.txt\n")
        if default_boundary != "PEC":
            f.write(f"materials.default.boundary     {default_boundary}\n")
        for fr in freqs:
            f.write(f"frequency.plan.point           {fr!r}\n")
        for lin in freq_linear:
            f.write(f"frequency.plan.linear          {lin}\n")
        f.write(f"reference.impedance            {reference_impedance!r}\n")
        f.write("solution.3D.tolerance          1e-14\n")
    return proj


def reference_project(d, name):
    """One of the reference's WR90 regression projects (tests/golden/wr90_projects.*)
    written out in directory d; returns (.proj path, its fixture record)."""
    import json
    here = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
    with open(os.path.join(here, "wr90_projects.json")) as f:
        rec = json.load(f)["projects"][name]
    z = np.load(os.path.join(here, "wr90_projects.npz"))
    k = rec["npz_key"]
    names = {int(t): v for t, v in rec["physical_names"].items()}
    proj = write_project(d, rec["stem"], z[k + "_verts"], z[k + "_tets"], z[k + "_phys"], names,
                         rec["ports_file"], rec["materials"], rec["order"], rec["freqs"],
                         rec.get("default_boundary", "PEC"), rec.get("freq_linear", ()),
                         rec.get("reference_impedance", 0.0))
    return proj, rec


def _rect(name, a, b, z):
    return (f"Path\n   name={name}\n   point=({-a / 2!r},{-b / 2!r},{z!r})\n   point=({a / 2!r},{-b / 2!r},{z!r})\n"
            f"   point=({a / 2!r},{b / 2!r},{z!r})\n   point=({-a / 2!r},{b / 2!r},{z!r})\n   closed=true\nEndPath\n\n")


def _line(name, p0, p1):
    return (f"Path\n   name={name}\n   point=({p0[0]!r},{p0[1]!r},{p0[2]!r})\n   point=({p1[0]!r},{p1[1]!r},{p1[2]!r})\n"
            f"   closed=false\nEndPath\n\n")


def _port(name, path, sport, vpath):
    return (f"Port\n   name={name}\n   path=+{path}\n   impedance_definition=PV\n   impedance_calculation=line\n"
            f"   Line\n      Sport={sport}\n      IntegrationPath\n         type=voltage\n         path=+{vpath}\n"
            f"      EndIntegrationPath\n   EndLine\nEndPort\n\n")


def write_guide_project(d, nx=6, ny=3, nz=15, L=50e-3, order=1, copper_wall=False):
    """The 6x3x15-hex air-filled WR90 box as a project in directory d; returns the .proj path."""
    a, b = meshgen.WR_A, meshgen.WR_B
    verts, tets = meshgen.box_kuhn(a, b, L, nx, ny, nz)
    write_gmsh22(os.path.join(d, "guide.msh"), verts, tets)
    ports = "#OpenParEMports 1.0\n\n"
    ports += _rect("p_in", a, b, 0.0) + _line("v_in", (0.0, -b / 2, 0.0), (0.0, b / 2, 0.0))
    ports += _rect("p_out", a, b, L) + _line("v_out", (0.0, -b / 2, L), (0.0, b / 2, L))
    ports += _port("input", "p_in", 1, "v_in") + _port("output", "p_out", 2, "v_out")
    if copper_wall:
        x = a / 2
        ports += (f"Path\n   name=side\n   point=({x!r},{-b / 2!r},0.0)\n   point=({x!r},{b / 2!r},0.0)\n"
                  f"   point=({x!r},{b / 2!r},{L!r})\n   point=({x!r},{-b / 2!r},{L!r})\n   closed=true\nEndPath\n\n")
        ports += "Boundary\n   name=Cu\n   type=surface_impedance\n   material=copper\n   path=+side\nEndBoundary\n"
    with open(os.path.join(d, "guide_ports.txt"), "w") as f:
        f.write(ports)
    with open(os.path.join(d, "materials.txt"), "w") as f:
        f.write("#OpenParEMmaterials 1.0\n\n")
        for name, body in (("air", "er=1.0\n         mur=1\n         tand=0\n         Rz=0"),
                           ("copper", "er=1\n         mur=1\n         conductivity=5.8e7\n         Rz=0")):
            f.write(f"Material\n   name={name}\n   Temperature\n      temperature=any\n      Frequency\n"
                    f"         frequency=any\n         {body}\n      EndFrequency\n   EndTemperature\n"
                    f"   Source\n   EndSource\nEndMaterial\n\n")
    proj = os.path.join(d, "guide.proj")
    with open(proj, "w") as f:
        f.write("#OpenParEM3Dproject 1.0\n\n")
        f.write(f"mesh.file                      guide.msh\nmesh.order                     {order}\n")
        f.write("port.definition.file           guide_ports.txt\n")
        f.write("materials.global.path          ./\nmaterials.global.name          materials.txt\n")
        f.write("materials.local.path           ./\nmaterials.local.name           //local_materials.txt\n")
        f.write("frequency.plan.linear          9e9,11e9,1e9\nfrequency.plan.point           10.5e9\n")
        f.write("frequency.plan.point           10e9\nsolution.3D.tolerance          1e-10\n")
    return proj


def write_lguide_project(d, nx=6, ny=4, nz=10, L=40e-3, order=1, freqs=(8e9, 8.5e9)):
    """An air-filled guide of L-shaped cross-section (the a x b = 24 x 16 mm box
    without its x > 0, y > 0 quadrant, whole Kuhn hexes removed), length L, as a
    project in directory d: the port paths are the six-point L outline at z = 0
    and z = L, the voltage paths cross the tall arm at x = -a/4.  Returns the
    .proj path."""
    a, b = 24e-3, 16e-3
    verts, tets = meshgen.box_kuhn(a, b, L, nx, ny, nz)
    cen = verts[tets].mean(axis=1)
    tets = tets[~((cen[:, 0] > 0) & (cen[:, 1] > 0))]
    used = np.unique(tets)
    remap = -np.ones(len(verts), dtype=np.int64)
    remap[used] = np.arange(len(used))
    verts, tets = verts[used], remap[tets]
    outline = [(-a / 2, -b / 2), (a / 2, -b / 2), (a / 2, 0.0), (0.0, 0.0), (0.0, b / 2), (-a / 2, b / 2)]
    spec = {"paths": [], "boundaries": [], "ports": []}
    for k, z in ((1, 0.0), (2, L)):
        spec["paths"].append({"name": f"port{k}", "points": [(x, y, z) for x, y in outline], "closed": True})
        spec["paths"].append({"name": f"V{k}", "points": [(-a / 4, -b / 2, z), (-a / 4, b / 2, z)], "closed": False})
        spec["ports"].append({"name": str(k), "paths": [f"+port{k}"], "impedance_definition": "PV",
                              "impedance_calculation": "line",
                              "lines": [{"Sport": k, "integration": [{"type": "voltage", "paths": [f"+V{k}"]}]}]})
    return write_project(d, "lguide", verts, tets, 1, {1: "air"}, spec,
                         {"air": {"er": 1.0, "mur": 1.0, "tand": 0.0, "Rz": 0.0}}, order, list(freqs))


def coax_mesh(nx=6, ny=4, nz=6, L=24e-3):
    """An air-filled rectangular coaxial line: the 24 x 16 mm box without the
    8 x 8 mm inner conductor about its axis (whole Kuhn hexes removed), length L
    along z.  Returns (verts, tets)."""
    a, b = 24e-3, 16e-3
    verts, tets = meshgen.box_kuhn(a, b, L, nx, ny, nz)
    cen = verts[tets].mean(axis=1)
    tets = tets[~((np.abs(cen[:, 0]) < 4e-3) & (np.abs(cen[:, 1]) < 4e-3))]
    used = np.unique(tets)
    remap = -np.ones(len(verts), dtype=np.int64)
    remap[used] = np.arange(len(used))
    return verts[used], remap[tets]


def faces_at_z(verts, tets, z):
    """The exterior faces of a tetrahedral mesh whose three vertices lie on the
    plane z (vertex triples in the owning tetrahedron's local order)."""
    from collections import Counter
    loc = ((0, 1, 2), (0, 1, 3), (0, 2, 3), (1, 2, 3))
    cnt = Counter(tuple(sorted(t[list(l)])) for t in tets for l in loc)
    out = []
    for t in tets:
        for l in loc:
            f = t[list(l)]
            if cnt[tuple(sorted(f))] == 1 and np.all(np.abs(verts[f, 2] - z) < 1e-12):
                out.append(f)
    return np.array(out, dtype=np.int64)


def write_coax_project(d, zdef="PI", with_current=True, freqs=(3e9,)):
    """The rectangular coaxial line of coax_mesh as a project in directory d:
    ports on the 24 x 16 mm outline at z = 0 and z = L (the inner conductor a hole
    in their faces), voltage paths from the inner conductor to the outer wall
    along +x, current paths a loop about the inner conductor, clockwise seen from
    outside each port (so the port's current has the sign of its voltage, as the
    reference's own port files orient them); impedance_definition zdef.  Returns
    the .proj path."""
    L = 24e-3
    verts, tets = coax_mesh(L=L)
    outline = [(-12e-3, -8e-3), (12e-3, -8e-3), (12e-3, 8e-3), (-12e-3, 8e-3)]
    loop = [(-8e-3, -6e-3), (8e-3, -6e-3), (8e-3, 6e-3), (-8e-3, 6e-3)]
    spec = {"paths": [], "boundaries": [], "ports": []}
    for k, z in ((1, 0.0), (2, L)):
        spec["paths"].append({"name": f"port{k}", "points": [(x, y, z) for x, y in outline], "closed": True})
        spec["paths"].append({"name": f"V{k}", "points": [(4e-3, 0.0, z), (12e-3, 0.0, z)], "closed": False})
        lp = loop if k == 1 else loop[::-1]   # outward normals -z and +z
        spec["paths"].append({"name": f"I{k}", "points": [(x, y, z) for x, y in lp], "closed": True})
        integ = [{"type": "voltage", "paths": [f"+V{k}"]}]
        if with_current:
            integ.append({"type": "current", "paths": [f"+I{k}"]})
        spec["ports"].append({"name": str(k), "paths": [f"+port{k}"], "impedance_definition": zdef,
                              "impedance_calculation": "line", "lines": [{"Sport": k, "integration": integ}]})
    return write_project(d, "coax", verts, tets, 1, {1: "air"}, spec,
                         {"air": {"er": 1.0, "mur": 1.0, "tand": 0.0, "Rz": 0.0}}, 1, list(freqs))


def write_mfem_mesh(path, verts, tets, attr, names):
    """A mesh in MFEM's ASCII format (v1.0) with the reference's regions file
    materials_for_<name> beside it: attr (per tetrahedron, 1-based) and names
    {attribute: material}; the boundary section lists no faces (the reader
    marks the boundary from the ports file)."""
    attr = np.broadcast_to(np.asarray(attr, dtype=np.int64), (len(tets),))
    with open(path, "w") as f:
        f.write("MFEM mesh v1.0\n\n#\n# written for the reader tests\n#\n\ndimension\n3\n\n")
        f.write(f"elements\n{len(tets)}\n")
        for a, t in zip(attr, tets):
            f.write(f"{int(a)} 4 {t[0]} {t[1]} {t[2]} {t[3]}\n")
        f.write("\nboundary\n0\n\n")
        f.write(f"vertices\n{len(verts)}\n3\n")
        for v in verts:
            f.write(f"{float(v[0]):.17g} {float(v[1]):.17g} {float(v[2]):.17g}\n")
    d, base = os.path.split(path)
    with open(os.path.join(d, "materials_for_" + base), "w") as f:
        f.write("OpenParEM Regions v1.0\n")
        for a, nm in sorted(names.items()):
            f.write(f"{int(a) - 1} {nm}\n")
