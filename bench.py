#!/usr/bin/env python
"""Benchmark of the B200 FLUPS solve path.

Workload (one step = one solve): 512^3 cell-centred scalar Poisson on [0,1]^3,
unbounded in all six faces, LGF_2 Green's kernel, transforms in FP32
(FP64-computed twiddles, FP32 copy of the FP64 Green's spectrum); the RHS is a
seeded sum of 8 Gaussians (synthetic).  The FP64 mode of the same solve is
timed beside it and gives the FP32 error (relative L2 / Linf).

Reported (one JSON line on rank 0):
  value      grid points per second, input and output resident in HBM
             (flups_solve on device pointers, CUDA events on the solver stream)
  e2e        same metric through flups_solve with pinned host arrays
             (H2D of the RHS and D2H of the field inside every step)
  roofline   the dominant pass: algorithmic bytes per launch / its average
             CUDA-event duration, against the measured HBM copy bandwidth
  cpu_baseline  the reference's own solver (its sources compiled unmodified
             by oracle/build_ref.py against in-repo FFTW/MPI/h3lpr stand-ins,
             one rank, OpenMP on all host threads) on a bounded 128^3 sample;
             the oracle port (numpy/scipy) when that build is absent

  configs    (one GPU) the other measured configurations run after the
             headline in the same process: node513, rot384 and the 64 x 128^3
             batch, one compact record each (--no-configs leaves them out)

--impl reference times the same reference build on the same metric, at the
workload's full grid when its run fits in about four minutes and half the
free host memory, else on a 256^3 or 128^3 sample.  --gpus N runs N independent replicas (one per GPU, weak
scaling).  --workload slab instead splits one solve over the ranks by z
planes (flups_b200/slab.py: NCCL all-to-all of the spectrum; strong scaling).
"""
import argparse
import json
import os
import subprocess
import sys
import threading
import time
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))

METRIC = "grid pts/s per solve FP32 vs FP64 at stated L2 err; %HBM roofline; p50/p99"
UNIT = "grid pts/s"


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--n", type=int, default=512)
    ap.add_argument("--kernel", default="LGF_2")
    ap.add_argument("--sample-n", type=int, default=128, help="grid of the bounded CPU sample")
    ap.add_argument("--profile", action="store_true", help="FP32 solves only (for ncu captures): no FP64, e2e or CPU legs")
    ap.add_argument("--no-configs", action="store_true",
                    help="solve workload: leave out the other measured configurations (node513, rot384, batch) "
                         "that the default single-GPU line carries under 'configs'")
    ap.add_argument("--workload", default="solve", choices=["solve", "batch", "group", "serve", "node513", "rot384", "slab"],
                    help="solve: the 512^3 headline; batch: 64 RHS of 128^3 HEJ_2 FP32 sharing one Green's spectrum; "
                         "serve: 2000 requests of mixed sizes/BCs/kernels/precisions at 500 req/s")
    ap.add_argument("--requests", type=int, default=2000, help="serve: requests in the trace")
    ap.add_argument("--slab-exchange", default="peer", choices=["peer", "alltoall"],
                    help="slab: y passes that store into / load from every rank's column array over CUDA IPC "
                         "(peer; NCCL all-to-all if any rank cannot open the others' arrays), or NCCL all-to-all")
    ap.add_argument("--overlap", type=int, default=0, help="1: overlap the per-x-slab middle passes on three streams")
    ap.add_argument("--rot", action="store_true",
                    help="with --profile --grid: a ROT solve (three components, LGF_4, spectral curl)")
    ap.add_argument("--bcs", type=int, nargs=6, default=None, metavar="BC",
                    help="with --profile --grid: boundary conditions x- x+ y- y+ z- z+ (0 EVEN, 1 ODD, 3 PER, 4 UNB)")
    ap.add_argument("--node", action="store_true", help="with --profile --grid: node-centred data")
    ap.add_argument("--precision", type=int, default=32, choices=[32, 64], help="with --profile --grid: working precision")
    ap.add_argument("--no-xlast", action="store_true", help="with --profile --grid: the reference's pass order")
    ap.add_argument("--grid", type=int, nargs=3, default=None, metavar=("NX", "NY", "NZ"),
                    help="with --profile: an all-unbounded grid NX x NY x NZ instead of n^3 (for ncu captures of one pass "
                         "length on a smaller array, e.g. 256 256 512 runs the 1024-point fused z pass on 1/4 of the lines)")
    return ap.parse_args()


def rhs_gaussians(n, seed=2, device=None):
    """Sum of 8 Gaussians, centres uniform in [0.2,0.8]^3, sigma in [0.03,0.08], amplitude in [-1,1]."""
    rng = np.random.default_rng(seed)
    x = (np.arange(n) + 0.5) / n
    if device is not None:
        import torch
        xs = torch.tensor(x, dtype=torch.float64, device=device)
        out = torch.zeros((n, n, n), dtype=torch.float64, device=device)  # [z][y][x]
        for _ in range(8):
            c = rng.uniform(0.2, 0.8, 3)
            s = rng.uniform(0.03, 0.08)
            a = rng.uniform(-1, 1)
            gx = torch.exp(-(xs - c[0]) ** 2 / s ** 2)
            gy = torch.exp(-(xs - c[1]) ** 2 / s ** 2)
            gz = torch.exp(-(xs - c[2]) ** 2 / s ** 2)
            out += a * gz[:, None, None] * gy[None, :, None] * gx[None, None, :]
        return out
    out = np.zeros((n, n, n))
    for _ in range(8):
        c = rng.uniform(0.2, 0.8, 3)
        s = rng.uniform(0.03, 0.08)
        a = rng.uniform(-1, 1)
        gx = np.exp(-(x - c[0]) ** 2 / s ** 2)
        gy = np.exp(-(x - c[1]) ** 2 / s ** 2)
        gz = np.exp(-(x - c[2]) ** 2 / s ** 2)
        out += a * gz[:, None, None] * gy[None, :, None] * gx[None, None, :]
    return out


class ClockSampler:
    """nvidia-smi clocks and throttle reasons during the timed region."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,clocks_event_reasons.hw_slowdown,"
              "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
              "clocks_event_reasons.sw_power_cap")

    def __init__(self, index):
        self.index = index
        self.proc = None

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.index), f"--query-gpu={self.FIELDS}",
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
        except OSError:
            self.proc = None
        return self

    def __exit__(self, *a):
        self.lines = []
        if self.proc is not None:
            time.sleep(0.25)
            self.proc.terminate()
            try:
                out, _ = self.proc.communicate(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()
                out, _ = self.proc.communicate()
            self.lines = [l for l in out.splitlines() if l.strip()]

    def summary(self):
        sm, smax, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for l in getattr(self, "lines", []):
            f = [v.strip() for v in l.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                smax = float(f[2])
            except ValueError:
                continue
            for nm, v in zip(names, f[5:9]):
                if v.lower() == "active":
                    reasons.add(nm)
        return {"sm_mhz": float(np.median(sm)) if sm else None, "sm_max_mhz": smax, "reasons": sorted(reasons),
                "samples": len(sm)}


# DRAM bytes (read + write) per launch / algorithmic bytes per launch of each pass
# of the 512^3 solve (x-last order), from ncu captures of the same kernel
# instances on quarter-size grids: the fused x rows and the z r2c / c2r pair
# passes on 512 x 128 x 512, the y passes on 128 x 512 x 512 (profiles/); the
# traffic of a 512^3 launch is this ratio times its algorithmic bytes (traffic
# grows with the lines processed).  Ratios below 1: the last writes of a launch
# are still in L2 when it ends.
TRAFFIC_RATIO_512 = {"fused": 1166281472 / 1211634404, "fwd1": 753636352 / 806879232, "bwd1": 781875968 / 806879232,
                     "fwd0": 488390656 / 537395200, "bwd0": 488814336 / 537395200}


def measured_peaks():
    p = ROOT / "MEASURED_PEAKS.json"
    if p.exists():
        d = json.loads(p.read_text())
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


REF_KIND_DESC = {
    "reference": "the reference's own solver (its src/*.cpp compiled unmodified, one rank, OpenMP on all host "
                 "threads) on an in-repo FP64 FFT in place of FFTW (absent here), oracle/_ref/libflups_ref.so",
    "port": "the reference's algorithm restated in numpy/scipy (FP64, all host threads); the reference build "
            "oracle/_ref/libflups_ref.so was absent",
}


def _cpu_solver(n, kernel):
    """A CPU solver of the n^3 all-unbounded cell-centred workload: the reference
    build when it is present (kind "reference"), else the oracle port."""
    from oracle import ref_lib
    from oracle.plans import CELL_CENTER
    from flups_b200.pyflups import GreenType
    bc = [[[4], [4]]] * 3
    if ref_lib.available():
        return ref_lib.RefSolver([n] * 3, 1, bc, [1.0 / n] * 3, [1.0] * 3, CELL_CENTER, int(GreenType[kernel])), "reference"
    from oracle.solver import OracleSolver
    o = OracleSolver([n] * 3, 1, bc, [1.0 / n] * 3, [1.0] * 3, CELL_CENTER)
    o.green_type = int(GreenType[kernel])
    o.setup()
    return o, "port"


def _cpu_time(solver, rhs):
    import scipy.fft as sfft
    with sfft.set_workers(os.cpu_count() or 1):
        t0 = time.perf_counter()
        solver.solve(rhs)
        return time.perf_counter() - t0


def cpu_oracle_sample(n, kernel, steps=3):
    """Time the CPU baseline (the reference build, else the oracle port) on an
    n^3 sample of the workload; returns pts/s, cores, median seconds, kind."""
    cores = os.cpu_count() or 1
    solver, kind = _cpu_solver(n, kernel)
    rhs = rhs_gaussians(n)[None].transpose(0, 3, 2, 1).copy()
    _cpu_time(solver, rhs)
    times = [_cpu_time(solver, rhs) for _ in range(steps)]
    t = float(np.median(times))
    return n ** 3 / t, cores, t, kind


def _mem_available():
    try:
        for ln in open("/proc/meminfo"):
            if ln.startswith("MemAvailable:"):
                return int(ln.split()[1]) * 1024
    except OSError:
        pass
    return 0


def reference_sample_n(args):
    """The largest of n, 256, 128 (n = the workload's grid) whose reference run
    (set-up + warm-up + timed solves) is predicted to end within about four
    minutes and whose arrays fit in half the free host memory, from one timed
    64^3 set-up and solve.  Solves grow with the point count times a log
    factor, the set-up (the lattice Green's function evaluated point by point)
    with the point count: 4.4 / 9.6 / 32.8 s at 96^3 / 128^3 / 192^3 on 8
    cores, 460 s at 512^3 on 16 cores, against 18 s per 512^3 solve."""
    t0 = time.perf_counter()
    solver, _ = _cpu_solver(64, args.kernel)
    ts64 = time.perf_counter() - t0
    rhs = rhs_gaussians(64)[None].transpose(0, 3, 2, 1).copy()
    _cpu_time(solver, rhs)
    t64 = _cpu_time(solver, rhs)
    del solver
    mem = _mem_available()
    for n in (args.n, 256, 128):
        if n > args.n:
            continue
        pts = (n / 64) ** 3
        t_total = (args.warmup + args.steps) * t64 * pts * (1.0 + np.log2(n / 64) / 4.0) + ts64 * pts
        need = 300.0 * (n ** 3) + 16.0 * n ** 3  # measured ~270 B per point in the reference build, + dense copies
        if t_total < 240.0 and (mem == 0 or need < 0.5 * mem):
            return n
    return 128


def run_reference(args):
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    n = reference_sample_n(args)
    cores = os.cpu_count() or 1
    t0 = time.perf_counter()
    solver, kind = _cpu_solver(n, args.kernel)
    setup_s = time.perf_counter() - t0
    rhs = rhs_gaussians(n)[None].transpose(0, 3, 2, 1).copy()
    for _ in range(args.warmup):
        _cpu_time(solver, rhs)
    times = [_cpu_time(solver, rhs) for _ in range(args.steps)]
    tot = sum(times)
    value = args.steps * n ** 3 / tot
    line = {
        "impl": "reference", "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": args.gpus, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": 1e3 * tot / args.steps, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f64", "data": "synthetic (seeded Gaussian sum)",
        "config": {"workload": f"{args.n}^3 cell-centred all-unbounded Poisson, {args.kernel}", "sample": f"{n}^3",
                   "l2_flush": "host run"},
        "cpu_baseline": {"value": value, "unit": UNIT, "cores": cores, "kind": kind,
                         "sample": f"{n}^3 solves of the same workload: {REF_KIND_DESC[kind]}"},
        "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
        "p50_ms": float(np.percentile(times, 50) * 1e3), "p99_ms": float(np.percentile(times, 99) * 1e3),
        "setup_s": setup_s,
    }
    print(json.dumps(line), flush=True)


def make_solver(pf, n, kernel, precision, stream):
    B = pf.BoundaryType
    t = pf.Topology(0, 1, [n, n, n])
    s = pf.Solver(t, [[B.UNB, B.UNB]] * 3, [1.0 / n] * 3, [1.0] * 3)
    s.set_green_type(pf.GreenType[kernel])
    s.set_precision(precision)
    s.set_stream(stream)
    t0 = time.perf_counter()
    s.setup()
    return t, s, time.perf_counter() - t0


def rhs_batch_gaussians(n, nb, seed=4, device=None):
    """nb single Gaussians, centres uniform in [0.3,0.7]^3, sigma uniform in [0.05,0.12]."""
    import torch
    rng = np.random.default_rng(seed)
    xs = torch.tensor((np.arange(n) + 0.5) / n, dtype=torch.float64, device=device)
    out = torch.empty((nb, n, n, n), dtype=torch.float64, device=device)
    for k in range(nb):
        c = rng.uniform(0.3, 0.7, 3)
        sg = rng.uniform(0.05, 0.12)
        gx = torch.exp(-(xs - c[0]) ** 2 / sg ** 2)
        gy = torch.exp(-(xs - c[1]) ** 2 / sg ** 2)
        gz = torch.exp(-(xs - c[2]) ** 2 / sg ** 2)
        out[k] = gz[:, None, None] * gy[None, :, None] * gx[None, None, :]
    return out


def run_batch(args, emit=True):
    """64 right-hand sides of 128^3 (cell, all unbounded, HEJ_2, FP32) sharing one
    Green's spectrum: 64 sequential solves, one batched launch per pass with the
    default and the autotuned CTA tiles, and the autotuned batch replayed from a
    CUDA graph.  One step = one batch of 64 solves."""
    import torch
    from flups_b200 import pyflups as pf
    torch.cuda.set_device(0)
    dev = torch.device("cuda", 0)
    n, nb = 128, 64
    stream = torch.cuda.Stream(device=dev)
    rhs = rhs_batch_gaussians(n, nb, device=dev)
    out = torch.empty_like(rhs)
    t, s, setup_s = make_solver(pf, n, "HEJ_2", 32, stream)
    s.set_async(True)

    def timed(fn, steps):
        with torch.cuda.stream(stream):
            for _ in range(max(3, args.warmup)):
                fn()
        stream.synchronize()
        evs = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(steps)]
        for a, b in evs:
            a.record(stream)
            fn()
            b.record(stream)
        stream.synchronize()
        ms = [a.elapsed_time(b) for a, b in evs]
        return float(np.mean(ms)), float(np.percentile(ms, 50)), float(np.percentile(ms, 99))

    def sequential():
        for k in range(nb):
            s.solve(out[k], rhs[k])

    seq = timed(sequential, max(3, args.steps // 4))
    fixed = timed(lambda: s.solve_batch(out, rhs, nb), args.steps)
    s.set_autotune(True)
    tuned = timed(lambda: s.solve_batch(out, rhs, nb), args.steps)
    graph = timed(lambda: s.solve_graph(out, rhs, nb), args.steps)
    stream.synchronize()
    ref32 = out[:4].clone()
    # per-pass bytes of one batched solve
    s.set_pass_timing(True)
    with torch.cuda.stream(stream):
        for _ in range(3):
            s.solve_batch(out, rhs, nb)
    stream.synchronize()
    stats = s.pass_stats()
    s.set_pass_timing(False)
    tot_bytes = sum(p["bytes"] for p in stats)
    del s, t
    torch.cuda.empty_cache()
    t64, s64, _ = make_solver(pf, n, "HEJ_2", 64, stream)
    out64 = torch.empty_like(rhs[:4])
    s64.solve_batch(out64, rhs[:4].contiguous(), 4)
    torch.cuda.synchronize()
    rel_l2 = float(torch.linalg.vector_norm(ref32 - out64) / torch.linalg.vector_norm(out64))
    del s64, t64
    peak, peak_kind = measured_peaks()
    ms = graph[0]
    line = {
        "metric": METRIC, "value": nb * n ** 3 / (ms * 1e-3), "unit": UNIT, "n_gpus": 1, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": ms, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "f32", "data": "synthetic (64 seeded Gaussians)",
        "config": {"workload": "64 x 128^3 cell-centred all-unbounded HEJ_2, FP32, one shared Green's spectrum, "
                               "autotuned tiles, replayed CUDA graph", "grid": [n, n, n], "batch": nb,
                   "l2_flush": "inputs larger than L2 (512 MiB RHS, 1+ GiB work arrays)"},
        "p50_ms": graph[1], "p99_ms": graph[2],
        "compare_ms_per_batch": {"sequential_64_plain_solves": seq[0], "batched_default_tiles": fixed[0],
                                 "batched_autotuned": tuned[0], "batched_autotuned_graph": graph[0]},
        "accuracy": {"fp32_rel_l2_vs_fp64_first4": rel_l2},
        "roofline": {"bound": "hbm", "kernel": "whole batched solve", "achieved": tot_bytes / (ms * 1e-3) / 1e9,
                     "peak": peak, "unit": "GB/s", "frac": tot_bytes / (ms * 1e-3) / 1e9 / peak, "peak_kind": peak_kind,
                     "bytes_per_step": tot_bytes, "traffic": None},
        "setup_s": setup_s,
    }
    if emit:
        print(json.dumps(line), flush=True)
    return line


def run_group(args):
    """Unevenly sized grids solved as one CUDA graph (flups_b200_solve_group):
    one right-hand side on each of 14 all-unbounded cell-centred grids, two of
    each size in {32, 48, 64, 96, 128, 192, 256}^3 (one HEJ_2, one LGF_2),
    FP32, against the same 14 solves issued one after another on one stream.
    One step = the 14 solves."""
    import torch
    from flups_b200 import pyflups as pf
    torch.cuda.set_device(0)
    dev = torch.device("cuda", 0)
    stream = torch.cuda.Stream(device=dev)
    sizes = [32, 48, 64, 96, 128, 192, 256]
    keep, solvers, rhss, outs = [], [], [], []
    for n in sizes:
        for kernel in ("HEJ_2", "LGF_2"):
            t, s, _ = make_solver(pf, n, kernel, 32, stream)
            s.set_async(True)
            keep.append(t)
            solvers.append(s)
            rhss.append(rhs_gaussians(n, seed=n, device=dev))
            outs.append(torch.empty_like(rhss[-1]))
    pts = sum(n ** 3 for n in sizes) * 2

    def timed(fn, steps):
        with torch.cuda.stream(stream):
            for _ in range(max(3, args.warmup)):
                fn()
        stream.synchronize()
        evs = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(steps)]
        for a, b in evs:
            a.record(stream)
            fn()
            b.record(stream)
        stream.synchronize()
        ms = [a.elapsed_time(b) for a, b in evs]
        return float(np.mean(ms)), float(np.percentile(ms, 50)), float(np.percentile(ms, 99))

    def sequential():
        for s, o, r in zip(solvers, outs, rhss):
            s.solve(o, r)

    seq = timed(sequential, args.steps)
    ref = [o.clone() for o in outs]
    codes = []
    grp = timed(lambda: codes.append(pf.solve_group(solvers, outs, rhss, stream=stream)), args.steps)
    stream.synchronize()
    same = all(torch.equal(a, b) for a, b in zip(outs, ref))
    ms = grp[0]
    line = {
        "metric": METRIC, "value": pts / (ms * 1e-3), "unit": UNIT, "n_gpus": 1, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": ms, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "f32", "data": "synthetic (seeded Gaussian sums)",
        "config": {"workload": "14 uneven all-unbounded cell-centred grids {32..256}^3 x {HEJ_2, LGF_2}, FP32, "
                               "one CUDA graph (flups_b200_solve_group)", "grids": sizes},
        "p50_ms": grp[1], "p99_ms": grp[2],
        "compare_ms_per_step": {"sequential_14_solves_one_stream": seq[0], "group_graph": grp[0]},
        "group_equals_sequential_bitwise": same, "codes_ok": all(c == 0 for c in codes),
    }
    print(json.dumps(line), flush=True)


def node513_rhs(dev):
    """513 x 257 x 257 nodes at i h (h = 1/256) on [0,2]x[0,1]x[0,1]: sum of 8 Gaussians,
    centres uniform in the domain shrunk by 0.2 L per side, sigma in [0.03,0.08], a in [-1,1]."""
    import torch
    rng = np.random.default_rng(2)
    h = 1.0 / 256
    n = (513, 257, 257)
    L = (2.0, 1.0, 1.0)
    ax = [torch.arange(n[d], dtype=torch.float64, device=dev) * h for d in range(3)]
    f = torch.zeros((n[2], n[1], n[0]), dtype=torch.float64, device=dev)
    for _ in range(8):
        c = [rng.uniform(0.2 * L[d], 0.8 * L[d]) for d in range(3)]
        sg = rng.uniform(0.03, 0.08)
        a = rng.uniform(-1.0, 1.0)
        g = [torch.exp(-(ax[d] - c[d]) ** 2 / sg ** 2) for d in range(3)]
        f += a * g[2][:, None, None] * g[1][None, :, None] * g[0][None, None, :]
    return f


def vortex_ring_rhs(n, dev):
    """Vortex ring on n^3 cells of [0,1]^3: centre (0.5,0.5,0.5), axis z, radius
    R(theta) = 0.25 (1 + sum_{m=1..8} a_m cos(m theta + phi_m)), a_m in [-1e-3,1e-3],
    phi_m in [0,2 pi); azimuthal vorticity Gamma/(pi s^2) exp(-d^2/s^2), Gamma = 1,
    s = 0.03, d the distance to the core line.  Returns [3][z][y][x]."""
    import torch
    rng = np.random.default_rng(3)
    am = rng.uniform(-1e-3, 1e-3, 8)
    ph = rng.uniform(0.0, 2 * np.pi, 8)
    x = (torch.arange(n, dtype=torch.float64, device=dev) + 0.5) / n - 0.5
    Z, Y, X = torch.meshgrid(x, x, x, indexing="ij")
    rho = torch.sqrt(X * X + Y * Y)
    th = torch.atan2(Y, X)
    R = torch.full_like(th, 0.25)
    for m in range(8):
        R = R + 0.25 * am[m] * torch.cos((m + 1) * th + ph[m])
    d2 = (rho - R) ** 2 + Z * Z
    s = 0.03
    w = (1.0 / (np.pi * s * s)) * torch.exp(-d2 / (s * s))
    out = torch.stack([-torch.sin(th) * w, torch.cos(th) * w, torch.zeros_like(w)])
    return out.contiguous()


def fast_flags(stats, plan):
    """Kernel family per timed pass, from the host-side plan of the same passes."""
    planned = [q.get("fast", 0) for q in plan.get("passes", []) if q.get("name") != "green"]
    if len(planned) == len(stats):
        return planned
    by_name = {q.get("name"): q.get("fast", 0) for q in plan.get("passes", [])}
    return [by_name.get(p["name"], 0) for p in stats]


def run_config(args, emit=True):
    """node513 (node-centred 513x257x257, EVEN/ODD x, PER y, UNB z, HEJ_4) or
    rot384 (384^3 cell, all UNB, LGF_4, ROT with the spectral curl, 3 components):
    FP32 and FP64 solves of device arrays, the FP32 error against the FP64 mode,
    and the per-pass times (which show the general line-pass kernel where the
    register DFTs do not apply)."""
    import torch
    from flups_b200 import pyflups as pf
    torch.cuda.set_device(0)
    dev = torch.device("cuda", 0)
    stream = torch.cuda.Stream(device=dev)
    B = pf.BoundaryType
    if args.workload == "node513":
        nglob, lda, typ = [513, 257, 257], 1, 0
        bcs = [[B.EVEN, B.ODD], [B.PER, B.PER], [B.UNB, B.UNB]]
        h, L, center, kernel, odiff = [1 / 256] * 3, [2.0, 1.0, 1.0], pf.CenterType.NODE_CENTER, "HEJ_4", pf.DiffType.NOD
        rhs = node513_rhs(dev)
        name = "513x257x257 node-centred, EVEN/ODD x, PER y, UNB z, HEJ_4 (alpha 2)"
    else:
        n = 384
        nglob, lda, typ = [n] * 3, 3, 1
        bcs = [[[B.UNB] * 3, [B.UNB] * 3]] * 3
        h, L, center, kernel, odiff = [1 / n] * 3, [1.0] * 3, pf.CenterType.CELL_CENTER, "LGF_4", pf.DiffType.SPE
        rhs = vortex_ring_rhs(n, dev)
        name = "384^3 cell, all UNB, LGF_4, ROT (spectral curl), 3-component vortex ring"
    torch.cuda.synchronize()
    res = {}
    outs = {}
    for prec in (32, 64):
        t = pf.Topology(0, lda, nglob)
        s = pf.Solver(t, bcs, h, L, order_diff=odiff, center_type=[center] * 3)
        s.set_green_type(pf.GreenType[kernel])
        s.set_precision(prec)
        s.set_stream(stream)
        s.set_async(True)
        t0 = time.perf_counter()
        s.setup()
        setup_s = time.perf_counter() - t0
        out = torch.empty_like(rhs)
        with torch.cuda.stream(stream):
            for _ in range(max(3, args.warmup)):
                s.solve(out, rhs, typ)
        stream.synchronize()
        evs = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(args.steps)]
        for a, b in evs:
            a.record(stream)
            s.solve(out, rhs, typ)
            b.record(stream)
        stream.synchronize()
        ms = [a.elapsed_time(b) for a, b in evs]
        s.set_pass_timing(True)
        with torch.cuda.stream(stream):
            for _ in range(3):
                s.solve(out, rhs, typ)
        stream.synchronize()
        stats = s.pass_stats()
        plan = s.plan_json(typ, 1)
        outs[prec] = out.clone()
        res[prec] = {"ms_per_solve": float(np.mean(ms)), "p50_ms": float(np.percentile(ms, 50)),
                     "p99_ms": float(np.percentile(ms, 99)), "setup_s": setup_s,
                     "passes": [{"name": p["name"], "ms": p["ms_total"] / max(1, p["calls"]), "bytes": p["bytes"],
                                 "kernel": ("register DFT" if f else "line pass")}
                                for p, f in zip(stats, fast_flags(stats, plan))]}
        del s, t
        torch.cuda.empty_cache()
    d = outs[32] - outs[64]
    rel_l2 = float(torch.linalg.vector_norm(d) / torch.linalg.vector_norm(outs[64]))
    rel_linf = float(d.abs().max() / outs[64].abs().max())
    pts = nglob[0] * nglob[1] * nglob[2]
    peak, peak_kind = measured_peaks()
    tot = sum(p["bytes"] for p in res[32]["passes"])
    ms32 = res[32]["ms_per_solve"]
    line = {
        "metric": METRIC, "value": pts / (ms32 * 1e-3), "unit": UNIT, "n_gpus": 1, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": ms32, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "f32", "data": "synthetic (seeded)", "config": {"workload": name, "grid": nglob, "lda": lda},
        "p50_ms": res[32]["p50_ms"], "p99_ms": res[32]["p99_ms"],
        "accuracy": {"fp32_rel_l2_vs_fp64": rel_l2, "fp32_rel_linf_vs_fp64": rel_linf},
        "fp64": {"value": pts / (res[64]["ms_per_solve"] * 1e-3), "ms_per_step": res[64]["ms_per_solve"]},
        "roofline": {"bound": "hbm", "kernel": "whole solve", "achieved": tot / (ms32 * 1e-3) / 1e9, "peak": peak,
                     "unit": "GB/s", "frac": tot / (ms32 * 1e-3) / 1e9 / peak, "peak_kind": peak_kind, "traffic": None},
        "detail": res,
    }
    if emit:
        print(json.dumps(line), flush=True)
    return line


def run_serve(args):
    """Serving trace: Poisson arrivals at 500 req/s; grid n^3 cell-centred with n in
    {32,...,256}; BC sets all-UNB, (PER,PER,UNB), (EVEN,UNB,UNB); HEJ_2 or LGF_2;
    FP32 (0.8) or FP64 (0.2); right-hand sides are seeded Gaussian sums resident on
    the device.  Runs the continuous-batching server from a cold cache, again with
    every key's solver resident, and a serial server (one solve at a time, no
    batching) on the same warm cache; then the same requests as one burst (all
    arriving at t = 0) for the capacity of each.  One step = the whole trace."""
    import torch
    from flups_b200.serving import GpuBackend, Request, Server, latency_stats, make_trace, rhs_pool, run_trace
    torch.cuda.set_device(0)
    dev = torch.device("cuda", 0)
    sizes = (32, 48, 64, 96, 128, 192, 256)
    pool = rhs_pool(sizes, per_size=4, device=dev)
    torch.cuda.synchronize()
    trace = make_trace(n_req=args.requests, rate=500.0, seed=5, sizes=sizes)
    free, total = torch.cuda.mem_get_info()
    budget = int(0.5 * free)
    be = GpuBackend()

    def finish_drop(h, reqs):
        for r in reqs:
            r.out = None  # results are complete; the caller would read them here
    be.finish = finish_drop

    def make(i, key, idx, ta):
        rhs = pool[(key[0], idx)]
        return Request(i, key, rhs, torch.empty_like(rhs), ta)

    def run(srv):
        srv.completed = []
        s0, e0 = srv.setups, srv.evictions
        wall = run_trace(srv, trace, make)
        torch.cuda.synchronize()
        st = latency_stats(srv.completed)
        pts = sum(r.key[0] ** 3 for r in srv.completed)
        return {"wall_s": wall, "solves_per_s": len(srv.completed) / wall, "pts_per_s": pts / wall,
                "mean_batch": float(np.mean([r.batch for r in srv.completed])),
                "setups": srv.setups - s0, "evictions": srv.evictions - e0, **st}

    srv = Server(be, budget, max_batch=16)
    cold = run(srv)
    warm = run(srv)
    serial = Server(be, budget, max_batch=1, max_inflight=1)
    serial.cache, serial.reserved = srv.cache, srv.reserved
    ser = run(serial)
    # capacity: the same requests arriving all at once (a burst), continuous vs
    # serial; the first continuous burst grows every key's batch arrays (one
    # allocation per key), the second runs on them
    burst_trace = [(0.0, key, idx) for _, key, idx in trace]
    saved = trace[:]
    trace[:] = burst_trace
    cap_first = run(srv)
    cap = run(srv)
    cap_serial = run(serial)
    trace[:] = saved
    srv.close()
    line = {
        "metric": METRIC, "value": warm["pts_per_s"], "unit": UNIT, "n_gpus": 1, "steps": 1, "warmup": 1,
        "ms_per_step": warm["wall_s"] * 1e3, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "f32/f64 mix (0.8/0.2)", "data": "synthetic (seeded Gaussian sums, Poisson arrivals, seed 5)",
        "config": {"workload": f"serving trace: {args.requests} requests at 500 req/s, n in {list(sizes)}, BC sets "
                               "all-UNB/(PER,PER,UNB)/(EVEN,UNB,UNB), HEJ_2/LGF_2, fp32/fp64 0.8/0.2",
                   "budget_bytes": budget, "max_batch": 16},
        "p50_ms": warm["p50_ms"], "p99_ms": warm["p99_ms"],
        "serve": {"continuous_warm": warm, "continuous_cold": cold, "serial_warm": ser,
                  "burst_continuous_first": cap_first, "burst_continuous": cap, "burst_serial": cap_serial},
    }
    print(json.dumps(line), flush=True)


def run_slab(args):
    """One n^3 all-unbounded LGF_2 FP32 solve split over the ranks by z planes
    (flups_b200/slab.py): the x and y passes of a rank's planes, an NCCL
    all-to-all of the spectrum, the last-direction pass of its columns, the
    all-to-all back and the inverse passes.  Strong scaling: the same solve
    at every rank count; device arrays (a rank holds its planes of rhs and
    field); the step time is the slowest rank's."""
    import datetime
    import socket

    import torch
    import torch.distributed as dist
    from flups_b200 import pyflups as pf
    from flups_b200.slab import ProcessGroupTransport, SlabRank, connect_peers, solve_connected
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if "MASTER_ADDR" not in os.environ:
        sk = socket.socket()
        sk.bind(("127.0.0.1", 0))
        os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(sk.getsockname()[1]), RANK="0", WORLD_SIZE="1")
        sk.close()
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300), device_id=dev)
    try:
        n = args.n
        B = pf.BoundaryType
        t = pf.Topology(0, 1, [n, n, n])
        s = pf.Solver(t, [[B.UNB, B.UNB]] * 3, [1.0 / n] * 3, [1.0] * 3)
        s.set_green_type(pf.GreenType[args.kernel])
        s.set_precision(32)
        r = SlabRank(s, rank, world)
        rhs = rhs_gaussians(n, device=dev)[r.z0:r.z1].contiguous()
        field = torch.empty_like(rhs)
        tr = ProcessGroupTransport()
        peer = args.slab_exchange == "peer"
        if peer:
            ok = 1
            try:
                connect_peers(r)
            except RuntimeError:
                ok = 0
            flag = torch.tensor([ok], device=dev)
            dist.all_reduce(flag, op=dist.ReduceOp.MIN)
            peer = bool(flag.item())
            if not peer:
                r.s.slab_peers([], [], [])

        def step():
            if peer:
                solve_connected(r, field, rhs)
            else:
                r.solve(field, rhs, tr)

        for _ in range(max(3, args.warmup)):
            step()
        torch.cuda.synchronize()
        dist.barrier()
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        with ClockSampler(local) as cs:
            e0.record()
            for _ in range(args.steps):
                step()
            e1.record()
            torch.cuda.synchronize()
        dist.barrier()
        tt = torch.tensor([e0.elapsed_time(e1) / args.steps], device=dev)
        dist.all_reduce(tt, op=dist.ReduceOp.MAX)
        ms = float(tt.item())
        if rank == 0:
            line = {
                "metric": METRIC, "value": n ** 3 / (ms * 1e-3), "unit": UNIT, "n_gpus": world, "steps": args.steps,
                "warmup": max(3, args.warmup), "ms_per_step": ms, "higher_is_better": True, "scaling": "strong",
                "vs_baseline": None, "dtype": "f32", "data": "synthetic (seeded sum of 8 Gaussians)",
                "config": {"workload": f"{n}^3 cell-centred all-unbounded scalar Poisson, {args.kernel}, FP32, "
                                       f"split over {world} rank(s) by z planes", "grid": [n, n, n],
                           "parallelism": f"z-slab x{world}",
                           "exchange": ("y passes store into / load from the owners' column arrays (CUDA IPC, NVLink)"
                                        if peer else "NCCL all_to_all_single of packed blocks"),
                           "l2_flush": "inputs larger than L2 at n = 512"},
                "e2e": {"value": None, "note": "device arrays only: the slab steps take each rank's planes on its GPU"},
                "gpu_launches": 5 * args.steps,
                "work_bytes_per_rank": int((np.prod(r.planes_shape) + np.prod(r.columns_shape)) * 4),
                "clocks": cs.summary(),
            }
            print(json.dumps(line), flush=True)
        if peer:
            r.s.slab_peers([], [], [])
            from flups_b200 import pyflups as _pf
            for ptr in getattr(r, "_opened", []):
                _pf.load_library().flups_b200_ipc_close(ptr)
        dist.barrier()
        del r, s, t
    finally:
        dist.destroy_process_group()


def run_profile_grid(args):
    """FP32 solves of a seeded random right-hand side on an anisotropic all-unbounded
    grid (cell-centred, h = 1/NX), for ncu captures; prints the mean solve time.
    --rot: a three-component ROT solve (LGF_4, spectral curl)."""
    import torch
    from flups_b200 import pyflups as pf
    nx, ny, nz = args.grid
    torch.cuda.set_device(0)
    B = pf.BoundaryType
    lda, typ = (3, 1) if args.rot else (1, 0)
    t = pf.Topology(0, lda, [nx, ny, nz])
    b6 = args.bcs if args.bcs else [4] * 6
    bc = [[[b6[2 * d]] * lda, [b6[2 * d + 1]] * lda] for d in range(3)]
    m = nx - 1 if args.node else nx
    L = [1.0, (ny - (1 if args.node else 0)) / m, (nz - (1 if args.node else 0)) / m]
    ctr = pf.CenterType.NODE_CENTER if args.node else pf.CenterType.CELL_CENTER
    s = pf.Solver(t, bc, [1.0 / m] * 3, L, order_diff=pf.DiffType.SPE if args.rot else pf.DiffType.NOD,
                  center_type=[ctr] * 3)
    s.set_green_type(pf.GreenType["LGF_4" if args.rot else args.kernel])
    s.set_precision(args.precision)
    if args.no_xlast:
        s.set_xlast(False)
    s.setup()
    g = torch.Generator(device="cuda")
    g.manual_seed(7)
    rhs = torch.randn((lda, nz, ny, nx), dtype=torch.float64, device="cuda", generator=g)
    field = torch.empty_like(rhs)
    for _ in range(max(1, args.warmup)):
        s.solve(field, rhs, typ)
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    for _ in range(args.steps):
        s.solve(field, rhs, typ)
    e1.record()
    torch.cuda.synchronize()
    print(json.dumps({"profile": True, "grid": [nx, ny, nz], "ms_per_step": e0.elapsed_time(e1) / args.steps}), flush=True)


def main():
    args = parse()
    if args.impl == "reference":
        run_reference(args)
        return
    if args.workload == "group":
        run_group(args)
        return
    if args.workload == "batch":
        run_batch(args)
        return
    if args.workload == "serve":
        run_serve(args)
        return
    if args.workload in ("node513", "rot384"):
        run_config(args)
        return
    if args.workload == "slab":
        run_slab(args)
        return
    if args.profile and args.grid:
        run_profile_grid(args)
        return
    import torch
    import torch.distributed as dist

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    if world > 1:
        import datetime
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300), device_id=dev)

    def barrier():
        if world > 1:
            dist.barrier()

    from flups_b200 import pyflups as pf
    n = args.n
    stream = torch.cuda.Stream(device=dev)
    rhs = rhs_gaussians(n, device=dev)
    field = torch.empty_like(rhs)

    # ---------------------------------------------------------------- FP32 (headline)
    t32, s32, setup32 = make_solver(pf, n, args.kernel, 32, stream)
    s32.set_async(True)
    s32.set_overlap(bool(args.overlap))
    with torch.cuda.stream(stream):
        for _ in range(max(3, args.warmup)):
            s32.solve(field, rhs)
    stream.synchronize()
    ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(args.steps)]
    barrier()
    torch.cuda.synchronize()
    with ClockSampler(local) as clk:
        t_all0 = torch.cuda.Event(enable_timing=True)
        t_all1 = torch.cuda.Event(enable_timing=True)
        t_all0.record(stream)
        for k in range(args.steps):
            ev[k][0].record(stream)
            s32.solve(field, rhs)
            ev[k][1].record(stream)
        t_all1.record(stream)
        stream.synchronize()
    torch.cuda.synchronize()
    barrier()
    elapsed = t_all0.elapsed_time(t_all1)  # ms
    step_ms = [a.elapsed_time(b) for a, b in ev]
    if world > 1:
        tt = torch.tensor([elapsed], device=dev)
        dist.all_reduce(tt, op=dist.ReduceOp.MAX)
        elapsed = float(tt.item())
    if args.profile:
        if rank == 0:
            print(json.dumps({"profile": True, "ms_per_step": elapsed / args.steps, "n": n}), flush=True)
        return
    field32 = field.clone()

    # per-pass device timing (separate short run) -> roofline of the dominant pass
    s32.set_pass_timing(True)
    with torch.cuda.stream(stream):
        for _ in range(5):
            s32.solve(field, rhs)
    stream.synchronize()
    stats = s32.pass_stats()
    s32.set_pass_timing(False)
    launches_per_solve = len(stats)
    tot_bytes = sum(p["bytes"] for p in stats)
    dom = max(stats, key=lambda p: p["ms_total"])
    dom_ms = dom["ms_total"] / max(1, dom["calls"])
    peak, peak_kind = measured_peaks()
    achieved = dom["bytes"] / (dom_ms * 1e-3) / 1e9

    # ---------------------------------------------------------------- e2e through the C ABI with host buffers
    # a window of 30 solves (about 0.8 s at 512^3): the first solve's upload and
    # the last one's download cannot overlap a neighbour, and their share of the
    # window shrinks with its length
    e2e_steps = 30
    h_rhs = torch.empty((n, n, n), dtype=torch.float64, pin_memory=True)
    h_rhs.copy_(rhs.cpu())
    h_out = torch.empty_like(h_rhs).pin_memory()
    # async calls: each returns once queued; the library uploads rhs and downloads
    # field in slabs on its copy streams, so one solve's download overlaps the
    # next one's upload; the download's completion is ordered on `stream`
    s32.set_async(True)
    s32.solve(h_out, h_rhs)  # warm the staging buffers and copy streams
    s32.synchronize()
    barrier()
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for _ in range(e2e_steps):
        s32.solve(h_out, h_rhs)
    e1.record(stream)
    e1.synchronize()
    s32.set_async(False)
    e2e_ms = e0.elapsed_time(e1) / e2e_steps
    if world > 1:
        tt = torch.tensor([e2e_ms], device=dev)
        dist.all_reduce(tt, op=dist.ReduceOp.MAX)
        e2e_ms = float(tt.item())
    user_bytes = n ** 3 * 8
    # the bound of that path: the same bytes copied up and down at once on two
    # streams (pinned memory, PCIe both ways), no solve
    d_up = torch.empty_like(rhs)
    cs1, cs2 = torch.cuda.Stream(device=dev), torch.cuda.Stream(device=dev)
    c0 = torch.cuda.Event(enable_timing=True)
    c1 = torch.cuda.Event(enable_timing=True)
    for rep in range(2):
        torch.cuda.synchronize()
        c0.record(cs1)
        cs2.wait_event(c0)
        with torch.cuda.stream(cs1):
            d_up.copy_(h_rhs, non_blocking=True)
        with torch.cuda.stream(cs2):
            h_out.copy_(field, non_blocking=True)
        cs1.wait_stream(cs2)
        c1.record(cs1)
        c1.synchronize()
    pcie_ms = c0.elapsed_time(c1)
    del d_up

    # ---------------------------------------------------------------- FP64 mode and the FP32 error
    del s32, t32
    torch.cuda.empty_cache()
    t64, s64, setup64 = make_solver(pf, n, args.kernel, 64, stream)
    s64.set_async(True)
    field64 = torch.empty_like(rhs)
    with torch.cuda.stream(stream):
        for _ in range(2):
            s64.solve(field64, rhs)
    stream.synchronize()
    f0 = torch.cuda.Event(enable_timing=True)
    f1 = torch.cuda.Event(enable_timing=True)
    k64 = max(3, min(args.steps, 10))
    f0.record(stream)
    for _ in range(k64):
        s64.solve(field64, rhs)
    f1.record(stream)
    f1.synchronize()
    ms64 = f0.elapsed_time(f1) / k64
    diff = field32 - field64
    rel_l2 = float(torch.linalg.vector_norm(diff) / torch.linalg.vector_norm(field64))
    rel_linf = float(diff.abs().max() / field64.abs().max())
    del s64, t64

    if rank != 0:
        if world > 1:
            dist.destroy_process_group()
        return

    cpu_value, cores, cpu_t, cpu_kind = cpu_oracle_sample(args.sample_n, args.kernel)
    ms_per_step = elapsed / args.steps
    value = world * n ** 3 / (ms_per_step * 1e-3)
    clocks = clk.summary()
    line = {
        "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": ms_per_step, "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
        "data": "synthetic (seeded sum of 8 Gaussians)",
        "config": {"workload": f"{n}^3 cell-centred all-unbounded scalar Poisson, {args.kernel}, FP32 transforms",
                   "grid": [n, n, n], "kernel": args.kernel, "l2_flush": "inputs larger than L2 (1 GiB RHS, 2+ GiB work arrays)",
                   "parallelism": f"{world} independent replica(s)"},
        "p50_ms": float(np.percentile(step_ms, 50)), "p99_ms": float(np.percentile(step_ms, 99)),
        "accuracy": {"fp32_rel_l2_vs_fp64": rel_l2, "fp32_rel_linf_vs_fp64": rel_linf,
                     "fp64_pinned_to_oracle": "<=1e-12 rel L2 at 16^3-64^3 (tests/test_gpu_parity.py)"},
        "fp64": {"value": world * n ** 3 / (ms64 * 1e-3), "ms_per_step": ms64},
        "setup_s": {"fp32": setup32, "fp64": setup64},
        "roofline": {"bound": "hbm", "kernel": dom["name"], "achieved": achieved, "peak": peak, "unit": "GB/s",
                     "frac": achieved / peak, "peak_kind": peak_kind,
                     "traffic": (TRAFFIC_RATIO_512[dom["name"]] * dom["bytes"]
                                 if (n == 512 and args.kernel == "LGF_2" and dom["name"] in TRAFFIC_RATIO_512) else None),
                     "traffic_source": "ncu dram__bytes_read.sum+dram__bytes_write.sum of the same kernel instance on a "
                                       "quarter-size grid (fused rows: 512x128x512), scaled by rows",
                     "bytes_per_launch": dom["bytes"], "ms_per_launch": dom_ms,
                     "solve_bytes": tot_bytes, "solve_frac": tot_bytes / (ms_per_step * 1e-3) / 1e9 / peak,
                     "passes": [{"name": p["name"], "ms": p["ms_total"] / max(1, p["calls"]), "bytes": p["bytes"]} for p in stats]},
        "e2e": {"value": world * n ** 3 / (e2e_ms * 1e-3), "unit": UNIT, "h2d_bytes_per_step": user_bytes,
                "d2h_bytes_per_step": user_bytes, "ms_per_step": e2e_ms, "steps": e2e_steps,
                "path": "flups_solve with pinned host rhs/field, async: slab-streamed upload/download overlapped",
                "pcie_bound_ms": pcie_ms,
                "pcie_bound_note": "the step's H2D and D2H bytes copied at once on two streams, no solve"},
        "gpu_launches": launches_per_solve * args.steps,
        "cpu_baseline": {"value": cpu_value, "unit": UNIT, "cores": cores, "kind": cpu_kind,
                         "sample": f"{args.sample_n}^3 solves of the same workload, median of 3: {REF_KIND_DESC[cpu_kind]}"},
        "clocks": clocks,
    }
    if world == 1 and not args.no_configs and n == 512:
        line["configs"] = other_configs(args)
    print(json.dumps(line), flush=True)
    if world > 1:
        dist.destroy_process_group()


def other_configs(args):
    """The other measured configurations, run after the headline in the same
    process and carried on its line (one compact record each): node513
    (513x257x257 node-centred EVEN/ODD-PER-UNB HEJ_4), rot384 (384^3 LGF_4 ROT,
    three components) and batch (64 x 128^3 HEJ_2 sharing one Green's
    spectrum, autotuned tiles, replayed graph).  Each is timed with CUDA events
    on its own stream over 10 steps after 3 warm-ups; a failure is recorded,
    not raised."""
    import copy

    import torch
    out = {}
    for name in ("node513", "rot384", "batch"):
        a = copy.copy(args)
        a.workload, a.steps, a.warmup = name, 10, 3
        torch.cuda.empty_cache()
        try:
            ln = run_batch(a, emit=False) if name == "batch" else run_config(a, emit=False)
        except Exception as e:  # noqa: BLE001 - a record of the failure is the result
            out[name] = {"error": f"{type(e).__name__}: {e}"}
            continue
        rec = {"workload": ln["config"]["workload"], "value": ln["value"], "unit": ln["unit"],
               "ms_per_step": ln["ms_per_step"], "p50_ms": ln.get("p50_ms"), "p99_ms": ln.get("p99_ms"),
               "accuracy": ln.get("accuracy"), "roofline_frac": ln["roofline"]["frac"],
               "roofline_kernel": ln["roofline"]["kernel"], "peak_kind": ln["roofline"]["peak_kind"]}
        if "fp64" in ln:
            rec["fp64_ms_per_step"] = ln["fp64"]["ms_per_step"]
        if "detail" in ln:
            rec["passes_ms"] = {p["name"]: p["ms"] for p in ln["detail"][32]["passes"]}
        if "compare_ms_per_batch" in ln:
            rec["compare_ms_per_batch"] = ln["compare_ms_per_batch"]
        out[name] = rec
    return out


if __name__ == "__main__":
    main()
