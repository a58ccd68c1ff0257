"""Writers of small OpenParEM3D-format project files (gmsh 2.2 mesh, ports file,
materials database, .proj) for the project-reader tests."""
import os

import numpy as np

from openparem_b200 import meshgen


def write_gmsh22(path, verts, tets, tag=1, name="air"):
    with open(path, "w") as f:
        f.write("$MeshFormat\n2.2 0 8\n$EndMeshFormat\n")
        f.write(f'$PhysicalNames\n1\n3 {tag} "{name}"\n$EndPhysicalNames\n')
        f.write(f"$Nodes\n{len(verts)}\n")
        for i, v in enumerate(verts):
            f.write(f"{i + 1} {float(v[0]):.17g} {float(v[1]):.17g} {float(v[2]):.17g}\n")
        f.write("$EndNodes\n")
        f.write(f"$Elements\n{len(tets)}\n")
        for e, t in enumerate(tets):
            f.write(f"{e + 1} 4 2 {tag} 1 {t[0] + 1} {t[1] + 1} {t[2] + 1} {t[3] + 1}\n")
        f.write("$EndElements\n")


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
