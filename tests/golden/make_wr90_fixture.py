"""Generate the WR90 golden fixtures from the OpenParEM source tree.

Reads, from the reference tree given on the command line (default: the
directory named by the OPEM_REFERENCE_ROOT environment variable):
  regression/OpenParEM3D/WR90/straight/straight.msh      (gmsh 2.2 mesh, 282 tets)
  regression/OpenParEM3D/WR90/straight-loaded/straight-loaded.msh
  regression/OpenParEM3D/regression_results.csv.current  (the reference's own
                                                          recorded found values)
and writes
  tests/golden/wr90_straight_mesh.npz   vertex coordinates (m) and tetrahedra
  tests/golden/wr90_loaded_mesh.npz     the same for straight-loaded.msh (physical
                                        volume 1 = air, 2 = teflon)
  tests/golden/wr90_expected.json       found S-parameter values per case (straight,
                                        straight-lossy, straight-loaded, and the
                                        projects below)
and, for the project-reader pins, from
  regression/OpenParEM3D/WR90/{straight-flipped,straight-rotated-xyz,shorted,opened,
                              straight-loaded}
  tests/golden/wr90_projects.npz        their meshes (vertices, tetrahedra, physical tags)
  tests/golden/wr90_projects.json       their ports files (paths, boundaries, ports)
                                        as data, mesh order, frequency points and
                                        the database entries of their materials
  tests/golden/wr90_regression.json     for the comparator: the test cases of the
                                        straight, straight-lossy, straight-loaded,
                                        shorted and opened projects (*_test_cases.csv
                                        rows) and the reference's evaluation of them
                                        (the first block of each in
                                        regression_results.csv.current, in order)

Run once in a container that has the reference tree; the outputs are
committed so the tests never need the reference at run time.
"""
import json
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))


def read_gmsh22(path):
    with open(path) as f:
        lines = [ln.strip() for ln in f]
    i = lines.index("$Nodes")
    nn = int(lines[i + 1])
    ids, xyz = [], []
    for ln in lines[i + 2:i + 2 + nn]:
        t = ln.split()
        ids.append(int(t[0])); xyz.append([float(v) for v in t[1:4]])
    idmap = {v: k for k, v in enumerate(ids)}
    i = lines.index("$Elements")
    ne = int(lines[i + 1])
    tets, phys = [], []
    for ln in lines[i + 2:i + 2 + ne]:
        t = [int(v) for v in ln.split()]
        etype, ntags = t[1], t[2]
        if etype == 4:
            nodes = t[3 + ntags:3 + ntags + 4]
            tets.append([idmap[v] for v in nodes])
            phys.append(t[3])
    return np.array(xyz), np.array(tets, dtype=np.int64), np.array(phys, dtype=np.int64)


def read_results(path):
    """Parse regression_results.csv.current into {project: {test name: row}}."""
    out, cur = {}, None
    with open(path) as f:
        for ln in f:
            ln = ln.strip()
            if ln.startswith("#./"):
                cur = ln[1:].split()[0]
                out.setdefault(cur, {})
                continue
            if not ln or ln.startswith("#") or cur is None:
                continue
            t = ln.split(",")
            name, status, freq, pout, pin, var, fn = t[:7]
            if fn == "equal":
                expected, found = float(t[7]), float(t[8])
            else:
                expected, found = None, float(t[7])
            out[cur][name] = {"frequency": float(freq), "portOut": int(pout), "portIn": int(pin),
                              "variable": var, "function": fn, "expected": expected, "found": found}
    return out


def read_physical_names(path):
    with open(path) as f:
        lines = [ln.strip() for ln in f]
    if "$PhysicalNames" not in lines:
        return {}
    i = lines.index("$PhysicalNames")
    out = {}
    for ln in lines[i + 2:i + 2 + int(lines[i + 1])]:
        dim, tag, name = ln.split(maxsplit=2)
        if dim == "3":
            out[int(tag)] = name.strip('"')
    return out


def _point(v):
    return [float(t) for t in v.strip().strip("()").split(",")]


def read_ports_file(path):
    """The Path, Boundary and Port blocks of an OpenParEM ports file as plain data
    (File blocks and comments dropped)."""
    spec = {"paths": [], "boundaries": [], "ports": []}
    block, port_line, ipath = None, None, None
    with open(path) as f:
        for raw in f:
            ln = raw.split("//")[0].strip()
            if not ln or ln.startswith("#"):
                continue
            if ln in ("Path", "Boundary", "Port", "File"):
                block = {"kind": ln, "paths": [], "points": [], "lines": []}
                continue
            if ln in ("EndPath", "EndBoundary", "EndPort", "EndFile"):
                k = block["kind"]
                if k == "Path":
                    spec["paths"].append({"name": block["name"], "points": block["points"],
                                          "closed": block.get("closed", "false") == "true"})
                elif k == "Boundary":
                    spec["boundaries"].append({"name": block["name"], "type": block["type"],
                                               "material": block.get("material"), "paths": block["paths"]})
                elif k == "Port":
                    spec["ports"].append({"name": block["name"], "paths": block["paths"],
                                          "impedance_definition": block.get("impedance_definition"),
                                          "impedance_calculation": block.get("impedance_calculation"),
                                          "lines": block["lines"]})
                block = None
                continue
            if block is None or block["kind"] == "File":
                continue
            if ln in ("Line", "Mode"):
                port_line = {"Sport": None, "integration": [], "block": ln}
                continue
            if ln in ("EndLine", "EndMode"):
                block["lines"].append(port_line)
                port_line = None
                continue
            if ln == "IntegrationPath":
                ipath = {"type": None, "paths": []}
                continue
            if ln == "EndIntegrationPath":
                port_line["integration"].append(ipath)
                ipath = None
                continue
            key, val = (t.strip() for t in ln.split("=", 1))
            if ipath is not None:
                if key == "path":
                    ipath["paths"].append(val)
                else:
                    ipath[key] = val
            elif port_line is not None:
                port_line[key] = int(val) if key == "Sport" else val
            elif key == "point":
                block["points"].append(_point(val))
            elif key == "path":
                block["paths"].append(val)
            else:
                block[key] = val
    return spec


def read_proj(path):
    out = {"freqs": []}
    with open(path) as f:
        for ln in f:
            t = ln.split("//")[0].split()
            if len(t) < 2:
                continue
            if t[0] == "mesh.order":
                out["order"] = int(t[1])
            elif t[0] == "frequency.plan.point":
                out["freqs"].append(float(t[1]))
            elif t[0] == "frequency.plan.linear":
                out.setdefault("freq_linear", []).append(t[1])
            elif t[0] == "reference.impedance":
                out["reference.impedance"] = float(t[1])
            elif t[0] in ("mesh.file", "port.definition.file", "materials.global.path", "materials.global.name",
                          "materials.local.path", "materials.local.name", "materials.default.boundary"):
                out[t[0]] = t[1]
    return out


def read_material(paths, name):
    """er, mur, tand, conductivity, Rz of one material of the first materials
    database (of paths: the local one, then the global one) that has it (the
    temperature=any / frequency=any entry)."""
    for path in paths:
        if not os.path.exists(path):
            continue
        with open(path) as f:
            lines = [ln.strip() for ln in f]
        if f"name={name}" in lines:
            break
    i = lines.index(f"name={name}")
    out = {}
    for ln in lines[i + 1:]:
        if ln == "EndMaterial":
            break
        if "=" in ln:
            k, v = ln.split("=", 1)
            if k in ("er", "mur", "tand", "conductivity", "Rz"):
                out[k] = float(v.split("//")[0])   # a trailing // comment is not part of the value
    return out


def read_test_cases(path):
    """Rows (field lists) of a *_test_cases.csv (comments dropped)."""
    rows = []
    with open(path) as f:
        for ln in f:
            ln = ln.strip()
            if not ln or ln.startswith("#"):
                continue
            rows.append(ln.split("//")[0].split(","))
    return rows


def read_first_block(path, project):
    """The rows (field lists, trailing empty field dropped) of the first block of
    a project in regression_results.csv.current."""
    rows, inside = [], False
    with open(path) as f:
        for ln in f:
            ln = ln.rstrip("\n")
            if ln.startswith("#./"):
                if inside:
                    break
                inside = ln[1:].split()[0] == project
                continue
            if inside and ln and not ln.startswith("#"):
                t = ln.split(",")
                rows.append(t[:-1] if t[-1] == "" else t)
    return rows


REGRESSION = {"straight": "straight", "straight-lossy": "straight", "straight-loaded": "straight-loaded",
              "shorted": "shorted", "opened": "opened"}


# further regression projects with rectangular ports, outside WR90/: fixture name -> (directory, stem)
OTHER = {"partially-filled-lossless": ("partially_filled_rect_waveguide/partially_filled_rect_waveguide_lossless",
                                       "part"),
         "partially-filled-lossy": ("partially_filled_rect_waveguide/partially_filled_rect_waveguide_lossy", "part"),
         "tee": ("WR90/tee", "tee"),
         "t-junction": ("WR75/T-Junction", "T-Junction"),
         "permeability-straight": ("permeability/rectangular_waveguide", "straight"),
         "permeability-partially-filled": ("permeability/partially_filled_rect_waveguide", "part"),
         # a microstrip line over a GaAs substrate crossing a dielectric bridge: the
         # strip is a hole in the port faces (conductor inside the cross-section)
         "bridge-3p78": ("microstrip/bridge", "bridge_3p78")}

PROJECTS = {"straight-flipped": "straight-flipped", "straight-rotated-xyz": "straight-rotated",
            "shorted": "shorted", "opened": "opened", "straight-loaded": "straight-loaded",
            "straight-lossy": "straight", "straight-loaded-lossy": "straight-loaded",
            "straight-rotated-x": "straight-rotated", "straight-rotated-y": "straight-rotated",
            "straight-asymmetric": "straight-asymmetric"}


def main(ref):
    wr = os.path.join(ref, "regression", "OpenParEM3D", "WR90")
    xyz, tets, phys = read_gmsh22(os.path.join(wr, "straight", "straight.msh"))
    np.savez_compressed(os.path.join(HERE, "wr90_straight_mesh.npz"), verts=xyz, tets=tets, phys=phys)
    xyz, tets, phys = read_gmsh22(os.path.join(wr, "straight-loaded", "straight-loaded.msh"))
    np.savez_compressed(os.path.join(HERE, "wr90_loaded_mesh.npz"), verts=xyz, tets=tets, phys=phys)
    res = read_results(os.path.join(ref, "regression", "OpenParEM3D", "regression_results.csv.current"))
    keep = {}
    for proj in ("./WR90/straight/straight.proj", "./WR90/straight-lossy/straight.proj",
                 "./WR90/straight-loaded/straight-loaded.proj"):
        keep[proj] = res[proj]
    arrays, projects = {}, {}
    todo = [(d, f"WR90/{d}", stem) for d, stem in PROJECTS.items()] + [(d, r, s) for d, (r, s) in OTHER.items()]
    for d, rel, stem in todo:
        pd = os.path.join(ref, "regression", "OpenParEM3D", rel)
        pj = read_proj(os.path.join(pd, stem + ".proj"))
        xyz, tets, phys = read_gmsh22(os.path.join(pd, pj["mesh.file"]))
        key = d.replace("-", "_")
        arrays[key + "_verts"], arrays[key + "_tets"], arrays[key + "_phys"] = xyz, tets, phys
        names = read_physical_names(os.path.join(pd, pj["mesh.file"]))
        mdb = [os.path.join(pd, pj.get("materials.local.path", "./"), pj.get("materials.local.name", "-")),
               os.path.join(pd, pj.get("materials.global.path", "./"), pj.get("materials.global.name", "-"))]
        dflt = pj.get("materials.default.boundary", "PEC")
        ports_file = read_ports_file(os.path.join(pd, pj["port.definition.file"]))
        bmats = {b["material"] for b in ports_file["boundaries"] if b.get("material")}
        mats = sorted(set(names.values()) | ({dflt} if dflt != "PEC" else set()) | bmats)
        projects[d] = {"stem": stem, "npz_key": key, "order": pj["order"], "freqs": pj["freqs"],
                       "physical_names": {str(k): v for k, v in names.items()},
                       "default_boundary": dflt, "freq_linear": pj.get("freq_linear", []),
                       "reference_impedance": pj.get("reference.impedance", 0.0),
                       "results_key": f"./{rel}/{stem}.proj",
                       "materials": {v: read_material(mdb, v) for v in mats},
                       "ports_file": ports_file}
        if f"./{rel}/{stem}.proj" in res:   # (the permeability guide has test cases but no recorded run)
            keep[f"./{rel}/{stem}.proj"] = res[f"./{rel}/{stem}.proj"]
    np.savez_compressed(os.path.join(HERE, "wr90_projects.npz"), **arrays)
    reg = {}
    rpath = os.path.join(ref, "regression", "OpenParEM3D", "regression_results.csv.current")
    for d, stem in REGRESSION.items():
        reg[d] = {"test_cases": read_test_cases(os.path.join(wr, d, stem + "_test_cases.csv")),
                  "evaluation": read_first_block(rpath, f"./WR90/{d}/{stem}.proj")}
    reg["permeability-straight"] = {
        "test_cases": read_test_cases(os.path.join(ref, "regression", "OpenParEM3D", "permeability",
                                                   "rectangular_waveguide", "straight_test_cases.csv")),
        "evaluation": []}
    reg["permeability-partially-filled"] = {
        "test_cases": read_test_cases(os.path.join(ref, "regression", "OpenParEM3D", "permeability",
                                                   "partially_filled_rect_waveguide", "part_test_cases.csv")),
        "evaluation": []}
    reg["bridge-3p78"] = {
        "test_cases": read_test_cases(os.path.join(ref, "regression", "OpenParEM3D", "microstrip", "bridge",
                                                   "bridge_3p78_test_cases.csv")),
        "evaluation": []}
    with open(os.path.join(HERE, "wr90_regression.json"), "w") as f:
        json.dump({"source": "regression/OpenParEM3D", "projects": reg}, f, indent=0)
    with open(os.path.join(HERE, "wr90_projects.json"), "w") as f:
        json.dump({"source": "regression/OpenParEM3D/WR90", "projects": projects}, f, indent=1, sort_keys=True)
    meta = {
        "source": "regression/OpenParEM3D/regression_results.csv.current",
        "mesh": "regression/OpenParEM3D/WR90/straight/straight.msh",
        "order": 6,
        "ports": {"1": "z=0.1 plane (name input)", "2": "z=0 plane (name output)"},
        "copper_sigma": 5.813e7,
        "cases": keep,
    }
    with open(os.path.join(HERE, "wr90_expected.json"), "w") as f:
        json.dump(meta, f, indent=1, sort_keys=True)
    print("wrote", len(tets), "tets and", sum(len(v) for v in keep.values()), "results")


if __name__ == "__main__":
    root = sys.argv[1] if len(sys.argv) > 1 else os.environ.get("OPEM_REFERENCE_ROOT", "")
    if not root:
        sys.exit("usage: make_wr90_fixture.py REFERENCE_ROOT (or set OPEM_REFERENCE_ROOT)")
    main(root)
