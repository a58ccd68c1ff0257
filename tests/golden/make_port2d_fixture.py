"""Extract the reference's OpenParEM2D regression cases that run without mesh
refinement (their 2D meshes, materials, modes-file voltage paths, frequency
plans and exact test cases) into tests/golden/port2d_cases.json.

Run from a checkout of the reference (the directory named by the first argument
or by the OPEM_REFERENCE_ROOT environment variable):
    python tests/golden/make_port2d_fixture.py REFERENCE_ROOT
The cases are data of the reference's regression suite
(regression/OpenParEM2D/*/..._exact_test_cases.csv: alpha in dB/m, beta / k0 and
Z of each mode against closed-form values, with the reference's tolerances).
"""
import json
import os
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, HERE)
from make_wr90_fixture import read_material, read_test_cases   # noqa: E402

# case name -> (project directory under regression/OpenParEM2D, project file)
CASES = {
    "WR90_order_6": ("WR90_rectangular_waveguide/WR90/WR90_order_6_norefinement", "WR90.proj"),
    "PartFilled_order_4": ("partially_filled_rect_waveguide/PartFilled_order_4_norefinement", "PartFilled.proj"),
    "PartFilled_order_5": ("partially_filled_rect_waveguide/PartFilled_order_5_norefinement", "PartFilled.proj"),
    "PartFilled_order_6": ("partially_filled_rect_waveguide/PartFilled_order_6_norefinement", "PartFilled.proj"),
    # meshes refined uniformly (mesh.uniform_refinement.count) before the solve
    "WR90_order_3_refined3": ("WR90_rectangular_waveguide/WR90/WR90_order_3_no_refinement_no_mesh_reuse", "WR90.proj"),
    "PartFilled_order_3_refined1": ("partially_filled_rect_waveguide/PartFilled_order_3_norefinement",
                                    "PartFilled.proj"),
    "PartFilled_order_4_refined1_wide": ("partially_filled_rect_waveguide/PartFilled_order_4_norefinement_widebandwidth",
                                         "PartFilled.proj"),
}


def read_proj2d(path):
    kv = {}
    with open(path) as f:
        for ln in f:
            ln = ln.split("//")[0].strip()
            if not ln or ln.startswith("#"):
                continue
            t = ln.split(None, 1)
            kv[t[0]] = t[1].strip() if len(t) > 1 else ""
    return kv


def read_mesh2d(path):
    """gmsh 2.2 triangles: nodes (x, y), triangles (0-based), physical tag per
    triangle, physical names."""
    with open(path) as f:
        lines = [ln.strip() for ln in f]
    names = {}
    if "$PhysicalNames" in lines:
        i = lines.index("$PhysicalNames")
        for ln in lines[i + 2:i + 2 + int(lines[i + 1])]:
            t = ln.split(None, 2)
            names[int(t[1])] = t[2].strip('"')
    i = lines.index("$Nodes")
    nn = int(lines[i + 1])
    ids, xy = [], []
    for ln in lines[i + 2:i + 2 + nn]:
        t = ln.split()
        ids.append(int(t[0]))
        xy.append([float(t[1]), float(t[2])])
    idmap = {v: k for k, v in enumerate(ids)}
    i = lines.index("$Elements")
    tris, phys = [], []
    for ln in lines[i + 2:i + 2 + int(lines[i + 1])]:
        t = [int(v) for v in ln.split()]
        if t[1] == 2:
            tris.append([idmap[v] for v in t[3 + t[2]:6 + t[2]]])
            phys.append(t[3])
    return xy, tris, phys, names


def read_modes(path):
    """Voltage paths of the modes file: {mode number: [p0, p1]} (2D points)."""
    paths, modes = {}, {}
    block, name, pts, mode = None, None, [], {}
    with open(path) as f:
        for ln in f:
            ln = ln.split("//")[0].strip()
            if ln in ("Path", "Mode", "File", "Boundary"):
                block, name, pts, mode = ln, None, [], {}
            elif ln == "EndPath":
                paths[name] = pts
            elif ln == "EndMode":
                if mode.get("type") == "voltage":
                    modes[int(mode["mode"])] = paths[mode["path"].lstrip("+")]
            elif "=" in ln:
                k, v = [s.strip() for s in ln.split("=", 1)]
                if block == "Path" and k == "name":
                    name = v
                elif block == "Path" and k == "point":
                    pts.append([float(s) for s in v.strip("()").split(",")])
                elif block == "Mode":
                    mode[k] = v
    return modes


def main(ref):
    root = os.path.join(ref, "regression", "OpenParEM2D")
    out = {}
    for case, (rel, pf) in CASES.items():
        d = os.path.join(root, rel)
        kv = read_proj2d(os.path.join(d, pf))
        assert kv.get("refinement.frequency") == "none"
        xy, tris, phys, names = read_mesh2d(os.path.join(d, kv["mesh.file"]))
        mdb = [os.path.join(d, kv.get("materials.local.path", "./"), kv.get("materials.local.name") or "-"),
               os.path.join(d, kv.get("materials.global.path", "./"), kv.get("materials.global.name") or "-")]
        mats = {names[p]: read_material(mdb, names[p]) for p in sorted(set(phys))}
        f0, f1, df = (float(v) for v in kv["frequency.plan.linear"].split(","))
        freqs = [f0 + i * df for i in range(int(round((f1 - f0) / df)) + 1)]
        mf = kv.get("mode.definition.file", "")
        vpaths = read_modes(os.path.join(d, mf)) if mf else {}
        tc = [f for f in os.listdir(d) if f.endswith("_exact_test_cases.csv")][0]
        cases = [r for r in read_test_cases(os.path.join(d, tc)) if "_result_" in r[0]]
        out[case] = {"project": f"regression/OpenParEM2D/{rel}/{pf}", "order": int(kv["mesh.order"]),
                     "uniform_refinement": int(kv.get("mesh.uniform_refinement.count", "0") or 0),
                     "modes": int(kv["solution.modes"]), "impedance": kv.get("solution.impedance.definition", "none"),
                     "freqs": freqs, "xy": xy, "tris": tris, "material": [names[p] for p in phys],
                     "materials": mats, "vpaths": {str(k): v for k, v in vpaths.items()}, "cases": cases}
    with open(os.path.join(HERE, "port2d_cases.json"), "w") as f:
        json.dump({"source": "regression/OpenParEM2D", "cases": out}, f, indent=0)
    print("wrote", {k: (len(v["tris"]), len(v["cases"])) for k, v in out.items()})


if __name__ == "__main__":
    root = sys.argv[1] if len(sys.argv) > 1 else os.environ.get("OPEM_REFERENCE_ROOT", "")
    if not root:
        sys.exit("usage: make_port2d_fixture.py REFERENCE_ROOT (or set OPEM_REFERENCE_ROOT)")
    main(root)
