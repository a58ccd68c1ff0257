"""Benchmark: frequency-point solves/s of the per-frequency FEM solve stage.

Workload (one GPU): the 24x12x60-hex (103,680 tets) WR90-size guide with the
eps_r=4.4 / tan_d=0.02 slab, Nedelec order 2 (681,312 DOF, 28.97M nnz), both
wave ports, frequencies from the 51-point 8-12 GHz sweep.  One step = one
frequency point = both driving sets (E solve, H projection, overlaps, S).

Arms
  (default)          this repo's CUDA path through the C ABI
  --impl reference   the FP64 CPU restatement of the reference algorithm
                     (oracle/: assembly, sparse direct LU as the reference's
                     Cholesky/LU-preconditioned KSP, H projection, overlaps, S)
                     on a bounded sample, see cpu_sample()

Inputs are synthetic (seeded structured mesh).  Operator arrays are ~1 GB,
larger than the 126 MB L2, so no explicit L2 flush is done between steps.
"""
import argparse
import json
import os
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "freq-point solves/sec at |dS|<=1e-6 vs FP64, mixed vs plain; p50/p99 latency"
UNIT = "freq-points/s"
C2_NDOF = 681312
REF_ND2_EXPONENT = 1.53   # reference's own ND2 timings: 103,146 -> 656,168 DOF, 18.45 -> 315.4 s


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=4)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--mode", default="plain", choices=["plain", "mixed"])
    ap.add_argument("--restart", type=int, default=100)
    ap.add_argument("--deflate", type=int, default=30)
    ap.add_argument("--mesh", default="24,12,60",
                    help="hex grid nx,ny,nz of the same box/slab/ND2 problem (profiling runs use a smaller one)")
    ap.add_argument("--rtol", type=float, default=1e-10)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    return ap.parse_args()


# ---------------------------------------------------------------------------
# CPU restatement (oracle) on a bounded sample
# ---------------------------------------------------------------------------
def _cpu_point(args):
    nx, ny, nz, f = args
    from openparem_b200 import meshgen
    from oracle import fem
    prob = meshgen.waveguide_problem(meshgen.WR_A, meshgen.WR_B, 50e-3, nx, ny, nz, 2,
                                     slab=(20e-3, 30e-3, 4.4, 0.02))
    t0 = time.perf_counter()
    ops = fem.Operators(prob)
    r = fem.solve_frequency(ops, f)
    dt = time.perf_counter() - t0
    return dt, ops.topo.n, r["S"]


def cpu_sample(npoints=None, cores=None):
    """Oracle per-frequency solves (assembly + LU + H + overlaps + S) of the same
    box / slab / ND2 problem on a 6x3x15-hex mesh (11,838 DOF), one point per
    process in a spawn pool.  The per-point time is scaled to the 681,312-DOF
    workload with the reference's own ND2 growth exponent (1.53, from its
    published 103k -> 656k DOF timings)."""
    import multiprocessing as mp
    cores = cores or min(8, os.cpu_count() or 1)
    npoints = npoints or cores
    freqs = np.linspace(8e9, 12e9, 51)[:npoints]
    ctx = mp.get_context("spawn")
    t0 = time.perf_counter()
    with ctx.Pool(cores) as pool:
        res = pool.map(_cpu_point, [(6, 3, 15, f) for f in freqs])
    wall = time.perf_counter() - t0
    per_point = float(np.mean([r[0] for r in res]))
    n_s = res[0][1]
    scaled = per_point * (C2_NDOF / n_s) ** REF_ND2_EXPONENT
    value = cores / scaled            # freq-points/s with `cores` points in flight
    return {"value": value, "unit": UNIT, "cores": cores, "kind": "port",
            "sample": (f"oracle (FP64 numpy/scipy, SuperLU direct solve) on {npoints} points of the 8-12 GHz sweep, "
                       f"6x3x15-hex ND2 mesh ({n_s} DOF), {per_point:.2f} s/point/core measured, "
                       f"scaled to {C2_NDOF} DOF by (n ratio)^{REF_ND2_EXPONENT}; wall {wall:.1f} s"),
            "sample_value": len(freqs) / wall}


# ---------------------------------------------------------------------------
# clocks sampler
# ---------------------------------------------------------------------------
class Clocks:
    def __init__(self, gpu):
        self.gpu = gpu
        self.samples = []
        self.proc = None

    def __enter__(self):
        q = ("clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.hw_slowdown,"
             "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
             "clocks_event_reasons.sw_power_cap")
        try:
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.gpu), f"--query-gpu={q}",
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except FileNotFoundError:
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            parts = [p.strip() for p in line.split(",")]
            if len(parts) >= 7:
                self.samples.append(parts)

    def __exit__(self, *a):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()

    def summary(self):
        if not self.samples:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}
        sm = [float(s[0]) for s in self.samples if s[0].replace(".", "").isdigit()]
        mx = [float(s[1]) for s in self.samples if s[1].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[i] for s in self.samples for i in range(4) if s[3 + i].lower().startswith("active")})
        return {"sm_mhz": float(np.median(sm)) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": reasons, "samples": len(self.samples)}


def peaks():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            d = json.load(f)
        return float(d["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


# ---------------------------------------------------------------------------
def run_reference(args, rank, world):
    if rank != 0:
        return
    steps = []
    for _ in range(args.warmup):
        pass
    for _ in range(args.steps):
        steps.append(cpu_sample())
    v = float(np.median([s["value"] for s in steps]))
    cb = dict(steps[-1])
    cb["value"] = v
    line = {"impl": "reference", "metric": METRIC, "value": v, "unit": UNIT, "n_gpus": args.gpus,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1000.0 / v if v else None,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "c128",
            "data": "synthetic", "config": config_dict(args), "cpu_baseline": cb,
            "e2e": {"value": v, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


def config_dict(args):
    return {"workload": "WR90 guide 24x12x60 hex (103,680 tets), eps_r 4.4/tan_d 0.02 slab, ND2 "
                        "(681,312 DOF), 2 wave ports, 51-point 8-12 GHz sweep",
            "order": 2, "ndof": C2_NDOF, "nnz": 28969152, "driving_sets_per_step": 2, "mode": args.mode,
            "mesh": args.mesh, "gmres_restart": args.restart, "gmres_deflate": args.deflate, "rtol": args.rtol,
            "krylov": "GMRES-DR (deflated restarting)", "precond": "vertex-patch block Jacobi",
            "l2": "operator arrays ~1 GB > 126 MB L2, no flush", "parallelism": f"replicas x{args.gpus}"}


def run_ours(args, rank, world, local_rank):
    import torch
    import torch.distributed as dist
    from openparem_b200 import meshgen, Fem3D, default_opts, _lib
    from openparem_b200.fem3d import Context
    import ctypes as C
    dev = local_rank
    torch.cuda.set_device(dev)
    nx, ny, nz = (int(v) for v in args.mesh.split(","))
    if (nx, ny, nz) == (24, 12, 60):
        prob, freqs = meshgen.config2()
    else:
        prob = meshgen.waveguide_problem(meshgen.WR_A, meshgen.WR_B, 50e-3, nx, ny, nz, 2,
                                         slab=(20e-3, 30e-3, 4.4, 0.02))
        freqs = np.linspace(8e9, 12e9, 51)
    ctx = Context(dev)
    F = Fem3D(prob, context=ctx).assemble()
    info = F.info()
    opts = default_opts(rtol=args.rtol, restart=args.restart, deflate=args.deflate, maxits=20000)
    # rank r takes frequencies r, r+world, ...
    my_freqs = freqs[rank::world]

    def step(i):
        f = my_freqs[i % len(my_freqs)]
        S, Z, st = F.solve(f, opts, allow_not_converged=True)
        return S, st

    for i in range(args.warmup):
        step(i)
    if world > 1:
        dist.barrier()
    torch.cuda.synchronize()
    l0 = C.c_int64()
    _lib.lib().opem_context_launches(ctx.h, C.byref(l0))
    dev_s = []
    wall_s = []
    its = []
    conv = []
    with Clocks(dev) as clk:
        for i in range(args.steps):
            t0 = time.perf_counter()
            S, st = step(args.warmup + i)
            wall_s.append(time.perf_counter() - t0)
            dev_s.append(st["seconds"])
            its.append(st["iterations"])
            conv.append(st["converged"])
    torch.cuda.synchronize()
    if world > 1:
        dist.barrier()
    l1 = C.c_int64()
    _lib.lib().opem_context_launches(ctx.h, C.byref(l1))
    t_dev = sum(dev_s)
    t_wall = sum(wall_s)
    tmax = torch.tensor([t_dev, t_wall], dtype=torch.float64, device=f"cuda:{dev}")
    if world > 1:
        dist.all_reduce(tmax, op=dist.ReduceOp.MAX)
    t_dev, t_wall = float(tmax[0]), float(tmax[1])
    # kernel roofline (CUDA events inside the library, same stream as the solve)
    prof = np.zeros(12)
    rc = _lib.lib().opem_profile_kernels(F.h, float(freqs[len(freqs) // 2]), 20,
                                        prof.ctypes.data_as(_lib.DP), 12)
    if rank != 0:
        return
    peak, peak_kind = peaks()
    names = ["spmv_c64", "patch_apply1", "multidot64", "cgs_update64"]
    kern = {names[k]: {"ms": prof[3 * k], "bytes": prof[3 * k + 1],
                       "GBps": prof[3 * k + 1] / (prof[3 * k] * 1e-3) / 1e9 if prof[3 * k] > 0 else None}
            for k in range(4)} if rc == 0 else {"error": rc}
    dom = "patch_apply1"
    ach = kern[dom]["GBps"] if rc == 0 else None
    units = args.steps * world
    value = units / t_dev
    e2e = units / t_wall
    n = info["ndofs"]
    line = {"metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": 1000.0 * t_dev / args.steps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "c128" if args.mode == "plain" else "c64/c128",
            "data": "synthetic", "config": config_dict(args),
            "e2e": {"value": e2e, "unit": UNIT, "h2d_bytes_per_step": 8 + 48,
                    "d2h_bytes_per_step": 2 * 16 * 4 + 2 * 2 * n * 16,
                    "note": "ctypes opem_solve_frequency call per step; returns S, Zo and E/H DOF vectors of both driving sets to host"},
            "gpu_launches": int(l1.value - l0.value),
            "roofline": {"bound": "hbm", "kernel": dom, "achieved": ach, "peak": peak, "unit": "GB/s",
                         "frac": (ach / peak) if ach else None, "traffic": None, "peak_kind": peak_kind,
                         "kernels": kern},
            "solver": {"iterations_per_step": its, "converged": conv, "patches": info["npatches"],
                       "max_patch": info["max_patch"]},
            "clocks": clk.summary()}
    if not args.no_cpu_baseline:
        line["cpu_baseline"] = cpu_sample()
    print(json.dumps(line), flush=True)


def main():
    args = parse()
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local_rank = int(os.environ.get("LOCAL_RANK", "0"))
    if args.impl == "reference":
        run_reference(args, rank, world)
        return
    if world > 1:
        import torch.distributed as dist
        from datetime import timedelta
        dist.init_process_group("nccl", timeout=timedelta(seconds=600))
    try:
        run_ours(args, rank, world, local_rank)
    finally:
        if world > 1:
            import torch.distributed as dist
            dist.destroy_process_group()


if __name__ == "__main__":
    main()
