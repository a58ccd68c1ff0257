"""Structured waveguide meshes and problem descriptions.

Builds the inputs the solve stage takes (the data OpenParEM3D has after
``mfem::Mesh(msh)``, ``BoundaryDatabase::assignAttributes`` and
``markMeshBoundaries``, src/OpenParEM3D/OpenParEM3D.cpp:284-327): vertex
coordinates, tetrahedra with region attributes, boundary triangles with
boundary attributes, region materials, boundary types and port modes.

Hexahedra are split into 6 tetrahedra along the (0,0,0)-(1,1,1) diagonal
(Kuhn/Freudenthal split), which is conforming between neighbouring hexes.
"""
import itertools
import numpy as np

C0 = 299792458.0


def box_kuhn(a, b, L, nx, ny, nz, z0=0.0):
    xs = np.linspace(-a / 2, a / 2, nx + 1)
    ys = np.linspace(-b / 2, b / 2, ny + 1)
    zs = z0 + np.linspace(0.0, L, nz + 1)
    X, Y, Z = np.meshgrid(xs, ys, zs, indexing="ij")
    verts = np.stack([X.transpose(2, 1, 0).ravel(), Y.transpose(2, 1, 0).ravel(),
                      Z.transpose(2, 1, 0).ravel()], axis=1)

    def vid(i, j, k):
        return i + (nx + 1) * (j + (ny + 1) * k)

    I, J, K = np.meshgrid(np.arange(nx), np.arange(ny), np.arange(nz), indexing="ij")
    I = I.transpose(2, 1, 0).ravel(); J = J.transpose(2, 1, 0).ravel(); K = K.transpose(2, 1, 0).ravel()
    tets = []
    for perm in itertools.permutations(range(3)):
        path = [np.zeros(3, dtype=int)]
        for ax in perm:
            nxt = path[-1].copy(); nxt[ax] = 1; path.append(nxt)
        tets.append(np.stack([vid(I + d[0], J + d[1], K + d[2]) for d in path], axis=1))
    tets = np.stack(tets, axis=1).reshape(-1, 4)
    return verts, tets.astype(np.int64)


def boundary_faces(tets):
    f = np.concatenate([tets[:, [0, 1, 2]], tets[:, [0, 1, 3]], tets[:, [0, 2, 3]], tets[:, [1, 2, 3]]])
    fs = np.sort(f, axis=1)
    u, inv, cnt = np.unique(fs, axis=0, return_inverse=True, return_counts=True)
    return u[cnt == 1]


def te10_mode(a, b, z, outward, ycenter_path=True):
    """TE10 on the rectangle [-a/2,a/2]x[-b/2,b/2] in the plane z.  Voltage path
    from the bottom wall to the top wall at x=0 (as v1/v2 in the reference's
    WR90 port files)."""
    return {"kind": "TE", "m": 1, "n": 0, "a": a, "b": b,
            "origin": [-a / 2, -b / 2, z], "u": [1.0, 0, 0], "v": [0, 1.0, 0],
            "normal": [0, 0, float(outward)],
            "vpath": ([0.0, -b / 2, z], [0.0, b / 2, z])}


def waveguide_problem(a, b, L, nx, ny, nz, order, *, eps_r=1.0, tand=0.0, slab=None,
                      wall="pec", wall_sigma=5.8e7, wall_Rz=0.0, per_element_eps=None,
                      ports=("zmin", "zmax"), radiation_cap=0.0, cap_nz=0):
    """Rectangular guide along z, PEC (or surface-impedance) walls.

    slab = (z_lo, z_hi, eps_r, tand) puts a dielectric region between two z planes.
    per_element_eps : optional (ne,) array, one region per tetrahedron.
    radiation_cap > 0 appends an air section of that length whose far face is a
    first-order radiation boundary (then only the zmin port is used).
    """
    Ltot = L + radiation_cap
    nzt = nz + cap_nz
    if radiation_cap > 0:
        # non-uniform z grid: nz cells over L, cap_nz cells over the cap
        verts, tets = box_kuhn(a, b, 1.0, nx, ny, nzt)
        zs = np.concatenate([np.linspace(0, L, nz + 1), L + np.linspace(0, radiation_cap, cap_nz + 1)[1:]])
        kz = np.rint(verts[:, 2] * nzt).astype(int)
        verts[:, 2] = zs[kz]
    else:
        verts, tets = box_kuhn(a, b, L, nx, ny, nz)
    ne = len(tets)
    cz = verts[tets].mean(axis=1)[:, 2]
    if per_element_eps is not None:
        region = np.arange(ne, dtype=np.int64)
        er = np.asarray(per_element_eps, dtype=np.float64)
        td = np.full(ne, tand)
        sg = np.zeros(ne)
        mr = np.ones(ne)
    else:
        region = np.zeros(ne, dtype=np.int64)
        er = [eps_r]; td = [tand]; sg = [0.0]; mr = [1.0]
        if slab is not None:
            z_lo, z_hi, e2, t2 = slab
            region[(cz > z_lo) & (cz < z_hi)] = 1
            er = [eps_r, e2]; td = [tand, t2]; sg = [0.0, 0.0]; mr = [1.0, 1.0]
        er = np.array(er); td = np.array(td); sg = np.array(sg); mr = np.array(mr)
    tris = boundary_faces(tets)
    tz = verts[tris][:, :, 2]
    tol = 1e-9 * max(Ltot, 1e-3)
    on_zmin = np.all(np.abs(tz - 0.0) < tol, axis=1)
    on_zmax = np.all(np.abs(tz - Ltot) < tol, axis=1)
    attr = np.ones(len(tris), dtype=np.int64)          # 1 = walls
    boundaries = {}
    port_list = []
    if wall == "pec":
        boundaries[1] = {"type": "pec"}
    else:
        boundaries[1] = {"type": "impedance", "sigma": wall_sigma, "Rz": wall_Rz, "mu_r": 1.0}
    nxt = 2
    if "zmin" in ports:
        attr[on_zmin] = nxt
        boundaries[nxt] = {"type": "port", "port": len(port_list)}
        port_list.append({"mode": te10_mode(a, b, 0.0, -1)})
        nxt += 1
    elif not radiation_cap:
        attr[on_zmin] = 1
    if radiation_cap > 0:
        attr[on_zmax] = nxt
        boundaries[nxt] = {"type": "radiation", "wave_impedance": float(np.sqrt(4e-7 * np.pi / 8.8541878176e-12))}
        nxt += 1
    elif "zmax" in ports:
        attr[on_zmax] = nxt
        boundaries[nxt] = {"type": "port", "port": len(port_list)}
        port_list.append({"mode": te10_mode(a, b, Ltot, +1)})
        nxt += 1
    return {
        "verts": verts, "tets": tets, "tet_region": region,
        "bdr_tris": tris, "bdr_attr": attr, "order": int(order),
        "eps_r": er, "tand": td, "sigma": sg, "mu_r": mr,
        "boundaries": boundaries, "ports": port_list,
    }


# ---- the benchmark configurations ----------------------------------------
WR_A, WR_B = 22.86e-3, 10.16e-3


def config1():
    """Air-filled 22.86x10.16x50 mm guide, 6x3x15 hex -> 1620 tets, ND1, 10 GHz."""
    return waveguide_problem(WR_A, WR_B, 50e-3, 6, 3, 15, 1), np.array([10e9])


def config2(nfreq=51):
    """Same box, slab eps_r=4.4 tan_d=0.02 for z in [20,30] mm, 24x12x60 hex
    (103,680 tets), ND2, 51 points 8-12 GHz."""
    prob = waveguide_problem(WR_A, WR_B, 50e-3, 24, 12, 60, 2, slab=(20e-3, 30e-3, 4.4, 0.02))
    return prob, np.linspace(8e9, 12e9, nfreq)


def config3(nfreq=101, seed=0):
    """40x20x100 hex (480k tets), ND2, copper walls sigma=5.8e7 with 0.5 um
    roughness, per-element eps_r ~ lognormal(ln 3, 0.1), 101 points 8-12 GHz.
    The 0.5 um RMS roughness is passed as the reference's Rz parameter."""
    rng = np.random.default_rng(seed)
    ne = 40 * 20 * 100 * 6
    eps = rng.lognormal(np.log(3.0), 0.1, size=ne)
    prob = waveguide_problem(WR_A, WR_B, 50e-3, 40, 20, 100, 2, wall="impedance",
                             wall_sigma=5.8e7, wall_Rz=0.5e-6, per_element_eps=eps)
    return prob, np.linspace(8e9, 12e9, nfreq)


def config4(seed=0, count=64):
    """64 uneven waveguide sections: length U(10, 60) mm, 3 hex per cm in z over a
    6x3 WR90 cross-section, ND1 or ND2 (coin flip), one frequency U(8, 12) GHz
    each, a 5 mm air cap at z_max closed by a first-order radiation boundary
    (the section's only port is at z = 0).  -> list of (problem, freqs)."""
    rng = np.random.default_rng(seed)
    out = []
    for _ in range(count):
        L = rng.uniform(10e-3, 60e-3)
        nz = max(1, int(round(3 * L * 100)))
        order = int(rng.integers(1, 3))
        f = rng.uniform(8e9, 12e9)
        prob = waveguide_problem(WR_A, WR_B, L, 6, 3, nz, order, ports=("zmin",), radiation_cap=5e-3, cap_nz=2)
        out.append((prob, np.array([f])))
    return out


# DOF per hexahedron (Kuhn split) for ND1 / ND2 / ND3 on large structured grids
DOF_PER_HEX = {1: 7.43, 2: 39.4, 3: 114.0}


def config5(seed=0, count=24, rate=200.0, max_dofs=2_000_000):
    """Serving stream: Poisson arrivals at `rate` req/s; each request is a guide of
    width a ~ U(20, 24) mm (TE10 the only mode above cutoff in the air sections over
    8-12 GHz), height a/2, length U(10, 60) mm, ND order 1-3, a dielectric block
    eps_r ~ U(1, 10) with tan_d = 0.01 over the middle half of its length, 1-4
    frequencies in 8-12 GHz, meshed for a DOF count drawn log-uniformly from 20k to
    max_dofs.  The block's small loss damps the higher modes trapped in it (they do
    not couple to the TE10 ports, so without loss their resonances make the system
    singular).  -> list of (arrival time s, problem, freqs)."""
    rng = np.random.default_rng(seed)
    t = 0.0
    out = []
    for _ in range(count):
        t += rng.exponential(1.0 / rate)
        a = rng.uniform(20e-3, 24e-3)
        b = a / 2
        L = rng.uniform(10e-3, 60e-3)
        order = int(rng.integers(1, 4))
        er = rng.uniform(1.0, 10.0)
        nf = int(rng.integers(1, 5))
        freqs = np.sort(rng.uniform(8e9, 12e9, nf))
        target = np.exp(rng.uniform(np.log(2e4), np.log(max_dofs)))
        nhex = target / DOF_PER_HEX[order]
        h = (a * b * L / nhex) ** (1.0 / 3.0)
        nx, ny, nz = (max(2, int(round(d / h))) for d in (a, b, L))
        prob = waveguide_problem(a, b, L, nx, ny, nz, order, slab=(0.25 * L, 0.75 * L, er, 0.01))
        out.append((t, prob, freqs))
    return out


def small_case(order=1, nx=3, ny=2, nz=4, L=20e-3, **kw):
    return waveguide_problem(WR_A, WR_B, L, nx, ny, nz, order, **kw)
