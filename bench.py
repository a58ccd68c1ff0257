"""Benchmark: frequency-point solves/s of the per-frequency FEM solve stage.

Workload (one GPU): the 24x12x60-hex (103,680 tets) WR90-size guide with the
eps_r=4.4 / tan_d=0.02 slab, Nedelec order 2 (681,312 DOF, 28.97M nnz), both
wave ports, frequencies from the 51-point 8-12 GHz sweep.  One step = one
frequency point = both driving sets (E solve, H projection, overlaps, S).

Arms
  (default)          this repo's CUDA path through the C ABI
  --impl reference   the oracle's FP64 CPU solve of the same 681,312-DOF point
                     on every host thread (oracle/cpu_solve.py: assembly,
                     Dirichlet procedure, preconditioned GMRES-DR, H projection),
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
# ncu dram__bytes_read+write / algorithmic bytes of the FP64 block apply, measured on the
# 16x8x40-hex ND2 case (traffic grows with the patches, so the ratio carries to 24x12x60)
TRAFFIC_RATIO_PATCH = 726.0 / 727.1
# the same for the batched block apply (tensor-core kernel, 26 systems), 16x8x40-hex ND2 case
TRAFFIC_RATIO_PATCH_BATCH = (396.159488 + 83.910656) / 561.419724
# nominal FP32 FMA rate: 148 SMs x 128 lanes x 2 flops x 1.965 GHz
FP32_PEAK_TFLOPS = 148 * 128 * 2 * 1.965e9 / 1e12
BATCH_KERNELS = ["patch_apply1_batch", "spmv_batch_f32", "spmv_batch_f64op_f32vec", "spmv_batch_f64",
                 "patch_apply2_batch", "patch_apply1_batch_fma", "patch_apply1_batch_tensor"]
FP64_KERNELS = ["spmv_c64", "patch_apply1", "multidot64", "cgs_update64"]


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=3)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--mode", default="both", choices=["plain", "mixed", "both"])
    ap.add_argument("--batch", type=int, default=13, help="frequency points per mixed-precision batch")
    ap.add_argument("--poly", type=int, default=16, help="GMRES-polynomial preconditioner degree of the batched path")
    ap.add_argument("--restart", type=int, default=100)
    ap.add_argument("--deflate", type=int, default=30)
    ap.add_argument("--config", type=int, default=2, choices=[2, 3],
                    help="2: the 24x12x60 slab guide, 51 points (headline); 3: the 40x20x100 copper-walled guide with "
                         "per-element eps_r, 101 points")
    ap.add_argument("--plain-points", type=int, default=0,
                    help="points of the sweep the FP64 comparison arm solves (0: all)")
    ap.add_argument("--mesh", default="24,12,60",
                    help="hex grid nx,ny,nz of the same box/slab/ND2 problem (profiling runs use a smaller one)")
    ap.add_argument("--rtol", type=float, default=1e-10)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--serve", choices=["c4", "c5"], default=None,
                    help="serving-loop workloads instead of the sweep: c4 = 64 uneven sections submitted at "
                         "once, c5 = Poisson stream of 20k-2M DOF requests (one GPU, not the headline line)")
    ap.add_argument("--serve-requests", type=int, default=24, help="requests of the c5 stream")
    ap.add_argument("--slots", type=int, default=4, help="concurrent requests of the serving loop")
    ap.add_argument("--kernels", action="store_true",
                    help="only time the hot kernels in isolation (--steps launches each) and print them")
    return ap.parse_args()


# ---------------------------------------------------------------------------
# CPU restatement (oracle) of the same 681,312-DOF point on a bounded sample
# ---------------------------------------------------------------------------
# Krylov steps of the oracle's FP64 CPU solve (GMRES-DR(100, 30), vertex-patch
# block Jacobi, rtol 1e-10) for the full config-2 point at 10 GHz, per driving
# set, measured by running that solve to convergence (805 s on 8 host cores).
CPU_STEPS_10GHZ = (649, 647)
CPU_SAMPLE_STEPS = 100   # one restart cycle of GMRES-DR(100, 30)


def cpu_sample(ops=None, nsteps=CPU_SAMPLE_STEPS):
    """A bounded sample of the config-2 workload (the 681,312-DOF guide, ND2,
    slab) on every host thread with the oracle's FP64 CPU solve
    (oracle/cpu_solve.py): for the 10 GHz point and driving set 1, the system
    assembly with the Dirichlet procedure, the vertex-patch block inversion,
    `nsteps` GMRES-DR steps (one restart cycle) and the H mass-matrix solve are
    timed.  A point is both driving sets' set-up and H solves plus the measured
    CPU_STEPS_10GHZ Krylov steps at the sampled cost per step; the result is in
    freq-points/s.  The reference's own path (sparse direct factorisation) is
    the oracle's SuperLU solve, which cannot factor this size in bench time."""
    from openparem_b200 import meshgen
    from oracle import fem, cpu_solve
    t0 = time.perf_counter()
    if ops is None:
        prob, _ = meshgen.config2()
        ops = fem.Operators(prob)
    t_ops = time.perf_counter() - t0
    cs = cpu_solve.CpuSolver(ops)
    f, d = 10e9, 0
    t1 = time.perf_counter()
    A = fem.assemble_A(ops, f, d)
    A = fem.eliminate(A, ops.pec_dofs)
    mm = fem.port_mode(ops, d, f)
    Et = ops.port_trace(d, mm["Et"])
    pd = ops.ports[d]["dofs"]
    x0 = np.zeros(ops.topo.n, dtype=np.complex128)
    x0[pd] = Et[pd]
    b = -(A @ x0)
    b[pd] = x0[pd]
    A = fem.eliminate(A, pd)
    t2 = time.perf_counter()
    M = cpu_solve.BlockJacobi(A, cs.pptr, cs.pdofs)
    t3 = time.perf_counter()
    e, its = cpu_solve.gmres_dr(cpu_solve.Csr(A), M, b, cs.m, cs.k, cs.rtol, maxits=nsteps)
    t4 = time.perf_counter()
    qe = (ops.Q_mu @ e) / (2 * np.pi * f * fem.MU0)
    cs._mass_solve(qe)
    t5 = time.perf_counter()
    t_asm, t_inv, t_step, t_h = t2 - t1, t3 - t2, (t4 - t3) / max(1, its), t5 - t4
    per_point = 2 * (t_asm + t_inv + t_h) + sum(CPU_STEPS_10GHZ) * t_step
    cores = os.cpu_count() or 1
    return {"value": 1.0 / per_point, "unit": UNIT, "cores": cores, "kind": "port",
            "sample": (f"oracle FP64 CPU solve (GMRES-DR(100,30) + vertex-patch block Jacobi, OpenMP kernels, "
                       f"{cores} threads) of the 681,312-DOF config-2 point at 10 GHz: driving set 1 timed "
                       f"(assembly {t_asm:.1f} s, block inversion {t_inv:.1f} s, {its} Krylov steps at "
                       f"{t_step * 1e3:.0f} ms, H solve {t_h:.1f} s); a point = 2 x set-up + "
                       f"{sum(CPU_STEPS_10GHZ)} measured Krylov steps = {per_point:.0f} s; operators {t_ops:.1f} s "
                       f"once per sweep"),
            "seconds_per_point": per_point, "krylov_step_ms": t_step * 1e3, "sample_seconds": t5 - t0}


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
def run_reference(args, rank, world, budget_s=200.0):
    """The reference arm: the oracle's FP64 CPU solve of the config-2 point on
    the host cores (rank 0 only; other ranks exit without work).  Each step is
    one bounded sample (cpu_sample, about a minute); steps run until `--steps`
    or the time budget, whichever comes first (at least one), and the line
    reports both."""
    if rank != 0:
        return
    from openparem_b200 import meshgen
    from oracle import fem
    t0 = time.perf_counter()
    prob, _ = meshgen.config2()
    ops = fem.Operators(prob)   # frequency-independent operators: once, untimed (warm-up)
    t_setup = time.perf_counter() - t0
    steps, walls = [], []
    t_start = time.perf_counter()
    while len(steps) < max(1, args.steps):
        w0 = time.perf_counter()
        steps.append(cpu_sample(ops))
        walls.append(time.perf_counter() - w0)
        if time.perf_counter() - t_start + walls[-1] > budget_s:
            break
    v = float(np.median([s_["value"] for s_ in steps]))
    cb = dict(steps[-1])
    cb["value"] = v
    line = {"impl": "reference", "metric": METRIC, "value": v, "unit": UNIT, "n_gpus": args.gpus,
            "steps": len(steps), "steps_requested": args.steps, "warmup": args.warmup,
            "warmup_note": f"operator assembly once before the timed samples ({t_setup:.1f} s); no sample is repeated "
                           "as warm-up (CPU code, no compilation)",
            "ms_per_step": 1000.0 * float(np.mean(walls)), "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "c128", "data": "synthetic", "config": config_dict(args),
            "cpu_baseline": cb,
            "e2e": {"value": v, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


def config_dict(args):
    if getattr(args, "config", 2) == 3:
        wl, nd, nz = ("WR90 guide 40x20x100 hex (480,000 tets), copper walls sigma 5.8e7 with 0.5 um roughness, "
                      "per-element eps_r ~ lognormal(ln 3, 0.1), ND2 (3,108,320 DOF), 2 wave ports, 101-point "
                      "8-12 GHz sweep", 3108320, 133589440)
    else:
        wl, nd, nz = ("WR90 guide 24x12x60 hex (103,680 tets), eps_r 4.4/tan_d 0.02 slab, ND2 "
                      "(681,312 DOF), 2 wave ports, 51-point 8-12 GHz sweep", C2_NDOF, 28969152)
    return {"workload": wl,
            "order": 2, "ndof": nd, "nnz": nz, "mode": args.mode, "plain_points": args.plain_points or "all",
            "step": (f"mixed: one batch of {args.batch} frequency points x 2 driving sets; plain: one point"
                     if args.mode != "plain" else "one frequency point (2 driving sets)"),
            "mesh": args.mesh, "gmres_restart": args.restart, "gmres_deflate": args.deflate, "rtol": args.rtol,
            "krylov": "GMRES-DR (deflated restarting); batched path: flexible GMRES-DR",
            "precond": "vertex-patch block Jacobi (FP64 plain; FP32 blocks + GMRES polynomial in the batched path)",
            "poly_degree": args.poly,
            "l2": "operator arrays ~1 GB > 126 MB L2, no flush", "parallelism": f"replicas x{args.gpus}"}


def kernel_profile(F, freq, nsys, reps, _lib):
    """CUDA-event times of the hot kernels in isolation (library stream): the
    batched path's kernels for nsys systems and the FP64 path's kernels."""
    out = {}
    b = np.zeros(21)
    rc = _lib.lib().opem_profile_batch_kernels(F.h, freq, nsys, reps, b.ctypes.data_as(_lib.DP), 21)
    f = np.zeros(12)
    rc2 = _lib.lib().opem_profile_kernels(F.h, freq, reps, f.ctypes.data_as(_lib.DP), 12)
    for names, arr, code in ((BATCH_KERNELS, b, rc), (FP64_KERNELS, f, rc2)):
        for k, nm in enumerate(names):
            if code != 0:
                out[nm] = {"error": code}
                continue
            ms, by = float(arr[3 * k]), float(arr[3 * k + 1])
            out[nm] = {"ms": ms, "bytes": by, "GBps": by / (ms * 1e-3) / 1e9 if ms > 0 else None}
    return out


def run_ours(args, rank, world, local_rank):
    import torch
    import torch.distributed as dist
    from openparem_b200 import meshgen, Fem3D, default_opts, _lib
    from openparem_b200.fem3d import Context, _dp
    import ctypes as C
    dev = local_rank
    torch.cuda.set_device(dev)
    nx, ny, nz = (int(v) for v in args.mesh.split(","))
    if args.config == 3:
        prob, freqs = meshgen.config3()
    elif (nx, ny, nz) == (24, 12, 60):
        prob, freqs = meshgen.config2()
    else:
        prob = meshgen.waveguide_problem(meshgen.WR_A, meshgen.WR_B, 50e-3, nx, ny, nz, 2,
                                         slab=(20e-3, 30e-3, 4.4, 0.02))
        freqs = np.linspace(8e9, 12e9, 51)
    ctx = Context(dev)
    F = Fem3D(prob, context=ctx).assemble()
    info = F.info()
    N = F.nports
    if args.kernels:
        if rank == 0:
            kern = kernel_profile(F, float(freqs[len(freqs) // 2]), min(32, args.batch * max(1, N)),
                                  max(1, args.steps), _lib)
            print(json.dumps({"mesh": args.mesh, "ndofs": info["ndofs"], "nnz": info["nnz"],
                              "systems": min(32, args.batch * max(1, N)), "kernels": kern}), flush=True)
        return
    plain_o = default_opts(rtol=args.rtol, restart=args.restart, deflate=args.deflate, maxits=5000)
    mixed_o = default_opts(rtol=args.rtol, restart=args.restart, deflate=args.deflate, maxits=3000,
                           precision=_lib.PREC_MIXED, poly_degree=args.poly)
    from openparem_b200.replicas import partition, max_over_ranks
    my_freqs = partition(freqs, rank, world)
    nb = args.batch

    nbatch = max(1, (len(my_freqs) + nb - 1) // nb)

    def batch_freqs(i):
        # contiguous slices of the sweep (a batch shares one block-Jacobi set per driving set)
        k = i % nbatch
        return np.ascontiguousarray(my_freqs[k * nb:(k + 1) * nb])

    def mixed_step(i):
        fr = batch_freqs(i)
        S = np.zeros(2 * N * N * len(fr))
        st = (_lib.SolveStats * len(fr))()
        t0 = time.perf_counter()
        rc = _lib.lib().opem_solve_sweep(F.h, len(fr), _dp(fr), C.byref(mixed_o), _dp(S), st)
        wall = time.perf_counter() - t0
        if rc not in (_lib.OK, _lib.ERR_NOT_CONVERGED):
            raise RuntimeError(f"opem_solve_sweep failed: {rc}")
        S = (S[0::2] + 1j * S[1::2]).reshape(len(fr), N, N)
        return fr, S, [s.as_dict() for s in st], wall

    def plain_step(f):
        t0 = time.perf_counter()
        S, Z, st = F.solve(f, plain_o, allow_not_converged=True)
        return S, st, time.perf_counter() - t0

    modes = ["mixed", "plain"] if args.mode == "both" else [args.mode]
    res = {}
    l0 = C.c_int64()
    l1 = C.c_int64()
    clk_summary = None
    def note(msg):
        if rank == 0:
            print(f"[bench] {msg}", file=sys.stderr, flush=True)

    note(f"assembled n={info['ndofs']} nnz={info['nnz']} patches={info['npatches']}")
    for mode in modes:
        if mode == modes[0]:
            steps, warm = args.steps, args.warmup
        else:
            # the FP64 comparison arm solves every point of this rank's sweep (or
            # --plain-points of them, spread over it), so |dS| mixed vs FP64 is
            # stated for those results
            steps, warm = len(my_freqs), 1
            if args.plain_points and args.plain_points < len(my_freqs):
                steps = args.plain_points
        for i in range(warm):
            note(f"{mode} warmup {i}")
            if mode == "mixed":
                mixed_step(i)
            else:
                plain_step(my_freqs[i % len(my_freqs)])
        if world > 1:
            dist.barrier()
        torch.cuda.synchronize()
        _lib.lib().opem_context_launches(ctx.h, C.byref(l0))
        dev_s, wall_s, lat, its, conv, outer, Sd = [], [], [], [], [], [], {}
        with Clocks(dev) as clk:
            for i in range(steps):
                note(f"{mode} step {i}")
                if mode == "mixed":
                    fr, S, st, wall = mixed_step(warm + i)
                    dev_s.append(sum(x["seconds"] for x in st))
                    wall_s.append(wall)
                    lat += [sum(x["seconds"] for x in st)] * len(fr)
                    its.append(st[0]["iterations"])
                    outer.append(st[0]["outer"])
                    conv += [x["converged"] for x in st]
                    for f, Sf in zip(fr, S):
                        Sd[float(f)] = Sf
                else:
                    if "mixed" in res:
                        stride = max(1, len(my_freqs) // steps)
                        f = float(my_freqs[(i * stride) % len(my_freqs)])
                    else:
                        f = my_freqs[(warm + i) % len(my_freqs)]
                    S, st, wall = plain_step(f)
                    dev_s.append(st["seconds"])
                    wall_s.append(wall)
                    lat.append(st["seconds"])
                    its.append(st["iterations"])
                    conv.append(st["converged"])
                    Sd[float(f)] = S
        torch.cuda.synchronize()
        if world > 1:
            dist.barrier()
        _lib.lib().opem_context_launches(ctx.h, C.byref(l1))
        units = sum(len(batch_freqs(warm + i)) for i in range(steps)) if mode == "mixed" else steps
        t = max_over_ranks([sum(dev_s), sum(wall_s)], dist if world > 1 else None, device=f"cuda:{dev}")
        res[mode] = {"units": units * world, "t_dev": float(t[0]), "t_wall": float(t[1]), "steps": steps,
                     "launches": int(l1.value - l0.value), "lat": lat, "its": its, "outer": outer, "conv": conv,
                     "S": Sd, "freqs": sorted(Sd.keys()), "clocks": clk.summary()}
        if mode == modes[0]:
            clk_summary = clk.summary()
        if mode == "mixed" and "plain" in modes:
            # batches the warm-up and timed steps did not reach (untimed), so every
            # point of the sweep has a mixed result to compare with FP64
            for i in range(nbatch):
                if any(float(f) not in res["mixed"]["S"] for f in batch_freqs(i)):
                    note(f"mixed coverage batch {i}")
                    fr, S, st, _ = mixed_step(i)
                    for f, Sf in zip(fr, S):
                        res["mixed"]["S"][float(f)] = Sf
                    res["mixed"]["conv"] += [x["converged"] for x in st]
    # the batched path applies the blocks of patches away from the ports to the
    # systems of both driving sets at once: profile that launch (2 x batch systems)
    nsys_apply = min(32, args.batch * max(1, N))
    kern = kernel_profile(F, float(freqs[len(freqs) // 2]), nsys_apply, 20, _lib)
    if rank != 0:
        return
    peak, peak_kind = peaks()
    if modes[0] == "mixed":
        # the batched path's dominant kernel: FP32 block apply for one driving set of `batch` systems
        dom, dom_label, ratio = ("patch_apply1_batch", f"batched block apply (FP32 blocks x {nsys_apply} systems)",
                                 TRAFFIC_RATIO_PATCH_BATCH)
        traffic_src = ("ncu dram__bytes_read+write of the same kernel on the 16x8x40-hex ND2 case, "
                       "scaled by algorithmic bytes")
    else:
        dom, dom_label, ratio = "patch_apply1", "patch_apply1_kernel (FP64 path)", TRAFFIC_RATIO_PATCH
        traffic_src = ("ncu dram__bytes_read+write of the same kernel on the 16x8x40-hex ND2 case, "
                       "scaled by algorithmic bytes")
    ach = kern[dom].get("GBps")
    fp32 = None
    if dom == "patch_apply1_batch" and kern[dom].get("ms"):
        sum_s2 = float(info["sum_patch_sq"]) if "sum_patch_sq" in info else None
        if sum_s2:
            fl = sum_s2 * nsys_apply * 8.0
            tf = fl / (kern[dom]["ms"] * 1e-3) / 1e12
            fp32 = {"flops_per_launch": fl, "tflops": tf, "peak_tflops_nominal": FP32_PEAK_TFLOPS,
                    "frac": tf / FP32_PEAK_TFLOPS}
    head = res[modes[0]]
    value = head["units"] / head["t_dev"]
    e2e = head["units"] / head["t_wall"]
    n = info["ndofs"]
    if modes[0] == "mixed":
        nfp = args.batch
        h2d = 8 * nfp + 64
        d2h = 16 * N * N * nfp + 48 * nfp
        e2e_note = "ctypes opem_solve_sweep call per step (13 points x 2 driving sets, host S buffer)"
    else:
        h2d = 8 + 64
        d2h = 2 * 16 * 4 + 2 * 2 * n * 16
        e2e_note = "ctypes opem_solve_frequency call per step; returns S, Zo and E/H DOF vectors of both driving sets"
    lat = np.array(head["lat"]) * 1e3
    line = {"metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": 1000.0 * head["t_dev"] / head["steps"], "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None,
            "dtype": "c128 Krylov+SpMV, c64 block-Jacobi+polynomial" if modes[0] == "mixed" else "c128",
            "data": "synthetic", "config": config_dict(args),
            "e2e": {"value": e2e, "unit": UNIT, "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": d2h, "note": e2e_note},
            "gpu_launches": head["launches"],
            "latency_ms": {"p50": float(np.percentile(lat, 50)), "p99": float(np.percentile(lat, 99)),
                           "what": "device time until a frequency point's S is available (its whole batch in mixed mode)"},
            "roofline": {"bound": "hbm", "kernel": dom_label, "achieved": ach, "peak": peak, "unit": "GB/s",
                         "frac": (ach / peak) if ach else None,
                         "traffic": (kern[dom]["bytes"] * ratio) if kern[dom].get("bytes") else None,
                         "traffic_source": traffic_src, "peak_kind": peak_kind, "fp32_fma": fp32, "kernels": kern},
            "solver": {"iterations_per_step": head["its"], "outer_steps": head["outer"],
                       "converged": head["conv"], "patches": info["npatches"], "max_patch": info["max_patch"]},
            "clocks": clk_summary}
    if "mixed" in res and "plain" in res:
        pv = res["plain"]["units"] / res["plain"]["t_dev"]
        common = [f for f in res["plain"]["freqs"] if f in res["mixed"]["S"]]
        dS = max(float(np.abs(res["mixed"]["S"][f] - res["plain"]["S"][f]).max()) for f in common) if common else None
        line["plain_fp64"] = {"value": pv, "unit": UNIT, "ms_per_point": 1000.0 / pv,
                              "iterations_per_point": res["plain"]["its"], "steps": res["plain"]["steps"],
                              "launches": res["plain"]["launches"]}
        line["mixed_vs_plain"] = value / pv
        per = [float(np.abs(res["mixed"]["S"][f] - res["plain"]["S"][f]).max()) for f in common]
        line["dS_mixed_vs_fp64"] = {"max": dS, "points": len(common), "tolerance": 1e-6,
                                    "within_tolerance": int(sum(d <= 1e-6 for d in per)),
                                    "median": float(np.median(per)) if per else None,
                                    "mixed_converged": int(sum(c == 1 for c in res["mixed"]["conv"])),
                                    "plain_converged": int(sum(c == 1 for c in res["plain"]["conv"]))}
    if not args.no_cpu_baseline:
        note("cpu baseline")
        try:
            line["cpu_baseline"] = cpu_sample()
        except Exception as e:   # reported, never silently replaced
            line["cpu_baseline"] = {"error": repr(e)}
    print(json.dumps(line), flush=True)


def run_serve(args, local_rank):
    """Serving-loop workloads through opem_server_* (the batched solver per request):
    freq-points/s over the whole stream (first submission to last completion),
    per-request latency p50/p99, and |dS| of a subset against FP64 solves of the
    same requests."""
    import torch
    from openparem_b200 import meshgen, Fem3D, Server, default_opts, _lib
    from openparem_b200.fem3d import Context
    dev = local_rank
    torch.cuda.set_device(dev)
    if args.serve == "c4":
        reqs = [(0.0, p, f) for p, f in meshgen.config4()]
        workload = "64 uneven WR90 sections, L ~ U(10,60) mm, 3 hex/cm, ND1/ND2, 5 mm radiation cap, 1 freq each"
    else:
        reqs = meshgen.config5(count=args.serve_requests)
        workload = (f"{len(reqs)} requests, Poisson 200 req/s, guides a ~ U(20,24) mm, L ~ U(10,60) mm, ND1-3, "
                    "eps_r block U(1,10) tan_d 0.01, 1-4 freqs, 20k-2M DOF log-uniform")
    ctx = Context(dev)
    fems = [Fem3D(p, context=ctx) for _, p, _ in reqs]   # assembled by their first request
    opts = default_opts(rtol=args.rtol, restart=args.restart, deflate=args.deflate, maxits=3000,
                        precision=_lib.PREC_MIXED, poly_degree=args.poly)
    srv = Server(dev, slots=args.slots)
    t0 = time.perf_counter()
    ids = []
    for (ta, _, f), F in zip(reqs, fems):
        dt = t0 + ta - time.perf_counter()
        if dt > 0:
            time.sleep(dt)
        ids.append(srv.submit(F, f, opts))
    res = [srv.wait(i) for i in ids]
    t_first = min(r[2]["submitted"] for r in res)
    t_last = max(r[2]["finished"] for r in res)
    points = sum(len(f) for _, _, f in reqs)
    lat = np.array([r[2]["finished"] - r[2]["submitted"] for r in res]) * 1e3
    conv = all(s["converged"] == 1 for r in res for s in r[1])
    # |dS| against FP64 solves of the smallest requests (after the timed stream)
    order = np.argsort([F.info()["ndofs"] for F in fems])[:6]
    plain = default_opts(rtol=1e-12, restart=200, maxits=6000)
    ids2 = [srv.submit(fems[k], reqs[k][2], plain) for k in order]
    dS = max(float(np.abs(srv.wait(i)[0] - res[k][0]).max()) for i, k in zip(ids2, order))
    info = srv.info()
    srv.close()
    dofs = [F.info()["ndofs"] for F in fems]
    line = {"mode": "serve", "workload": args.serve, "metric": METRIC, "value": points / (t_last - t_first),
            "unit": UNIT, "n_gpus": 1, "requests": len(reqs), "points": points, "slots": args.slots,
            "seconds": t_last - t_first, "latency_ms": {"p50": float(np.percentile(lat, 50)),
                                                         "p99": float(np.percentile(lat, 99)),
                                                         "what": "request submitted -> S available"},
            "converged": conv, "dS_vs_fp64": {"max": dS, "requests": len(order), "tolerance": 1e-6},
            "dofs": {"min": int(min(dofs)), "max": int(max(dofs)), "total": int(sum(dofs))},
            "config": {"workload": workload, "poly_degree": args.poly, "rtol": args.rtol,
                       "budget_bytes": info["budget_bytes"]},
            "data": "synthetic", "dtype": "c128 Krylov, c64 block-Jacobi+polynomial",
            "per_request": [{"ndofs": int(d), "order": int(p["order"]), "freqs": len(f),
                             "its": int(r[1][0]["iterations"]), "converged": all(x["converged"] == 1 for x in r[1]),
                             "latency_ms": float(l)}
                            for d, (_, p, f), r, l in zip(dofs, reqs, res, lat)]}
    print(json.dumps(line), flush=True)


def main():
    args = parse()
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local_rank = int(os.environ.get("LOCAL_RANK", "0"))
    if args.impl == "reference":
        run_reference(args, rank, world)
        return
    if args.serve:
        if rank == 0:
            run_serve(args, local_rank)
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
