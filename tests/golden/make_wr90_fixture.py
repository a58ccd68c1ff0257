"""Generate the WR90 golden fixtures from the OpenParEM source tree.

Reads, from the reference tree given on the command line (default
/root/reference):
  regression/OpenParEM3D/WR90/straight/straight.msh      (gmsh 2.2 mesh, 282 tets)
  regression/OpenParEM3D/WR90/straight-loaded/straight-loaded.msh
  regression/OpenParEM3D/regression_results.csv.current  (the reference's own
                                                          recorded found values)
and writes
  tests/golden/wr90_straight_mesh.npz   vertex coordinates (m) and tetrahedra
  tests/golden/wr90_loaded_mesh.npz     the same for straight-loaded.msh (physical
                                        volume 1 = air, 2 = teflon)
  tests/golden/wr90_expected.json       found S-parameter values per case (straight,
                                        straight-lossy, straight-loaded)

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
    main(sys.argv[1] if len(sys.argv) > 1 else "/root/reference")
