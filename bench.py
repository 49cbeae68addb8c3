#!/usr/bin/env python
"""Headline benchmark: the 3D Fourier x Fourier x GLL Helmholtz solve.

Workload (one "step" = one solve): Nx = Ny = 256 Fourier modes, GLL N = 64
(65 points) in z, lambda = 10, homogeneous Dirichlet, f a seeded smooth field
(complex Gaussian Fourier/Legendre coefficients with amplitude (1+|k|^2)^-1.5,
zero mean).  DOF per solve = 256 * 256 * 65 = 4,259,840 grid values of u.

`value` is the FP32 + FP64-residual-refinement solve in GDOF/s with inputs
resident in HBM, the L2 flushed (256 MB write) before every timed solve, and
device time from CUDA events; `fp64` gives the plain FP64 solve beside it.
`e2e` is the same solve through the public API from pinned host memory
(H2D of f and D2H of u of every step inside the timed region; consecutive
steps overlap their copies with the neighbouring solves on separate streams,
as a serving loop does).  Multi-GPU runs are replicas
(the path has no exchange step): every rank solves its own copy, the time is
the max over ranks, and `value` counts all ranks' DOF.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]
"""
from __future__ import annotations

import argparse
import datetime
import json
import math
import os
import re
import signal
import subprocess
import sys
import tempfile
import time

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, HERE)

METRIC = "GDOF/s FP32+refine vs FP64 on B200 at ≤1e-10 rel err; fwd+adjoint ms; %HBM"
NX = NY = 256
NGLL = 65
LAM = 10.0
SEED = 1236
DOM = (0.0, 2 * math.pi, 0.0, 2 * math.pi, 0.0, 2.0)
WORKLOAD = "3D Helmholtz, Fourier 256 x Fourier 256 x GLL 65 (N=64), lambda=10, Dirichlet, seeded smooth field"
FALLBACK_HBM_GBS = 6650.0


def _args():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=200)
    ap.add_argument("--warmup", type=int, default=20)
    ap.add_argument("--impl", choices=("ours", "reference"), default="ours")
    ap.add_argument("--skip-cpu-baseline", action="store_true", help="omit the CPU leg (profiling runs)")
    ap.add_argument("--skip-side", action="store_true", help="omit the batch / adjoint / finite-difference / periodic / derivative legs")
    ap.add_argument("--profile-case", choices=("fp64", "fp32_refine", "fp32", "fd64", "fd64h", "fd32", "fd32x", "batch",
                                               "deriv"),
                    help="run three untimed solves of one workload and exit (a small case for ncu captures)")
    return ap.parse_args()


def profile_case(which: str):
    """Plan creation (with its autotuning), then three solves: the headline
    256 x 256 x 65 workload at one precision, a 256 x 256 x 256 finite-difference
    solve (fd64: a tridiagonal row per warp; fd64h: per half-warp), or the
    512-problem batch; or ("deriv") three rounds of the z, x and y derivatives of
    a 512 x 256 x 65 FP64 field."""
    import torch

    from mpi_b200 import workloads as W

    torch.cuda.set_device(0)
    if which in ("fd64", "fd64h", "fd32", "fd32x"):
        from mpi_b200 import Helmholtz3DFD

        # fd32x: the length-1024 x passes of the FD workload on a 1024 x 512 x 64
        # grid (134 MB FP32 field, larger than L2), FP32 I/O as the bench's FD leg
        nx, ny, nz = (1024, 512, 64) if which == "fd32x" else (256, 256, 256)
        f = torch.from_numpy(W.smooth_field_fd(nx, ny, nz, seed=1239)).cuda()
        p = Helmholtz3DFD(nx, ny, nz, 0.0, 1.0, 0.0, 1.0, 0.0, 1.0, Lambda=1.0,
                          precision="fp64" if which in ("fd64", "fd64h") else "fp32")
        # fd64h: the tridiagonal solves pinned to a row per half-warp (row variant 1)
        p.set_launch_variants(p.launch_variants()["fft"], 1 if which == "fd64h" else 0)
        if which == "fd32x":
            p.set_io_bytes(4)
            f = f.float()
        run = lambda: p.SolvePDE(f)  # noqa: E731
    elif which == "deriv":
        from mpi_b200 import NonPeriodic3D

        # d/dz (GLL), d/dx, d/dy (spectral) of a 512 x 256 x 65 FP64 field
        # (68 MB in, 68 MB out: larger than L2 together)
        p = NonPeriodic3D(512, 256, NGLL, NGLL, *DOM, Lambda=1.0)
        f = torch.randn(512, 256, NGLL, dtype=torch.float64, device="cuda")
        o = torch.empty_like(f)

        def run():
            p.FirstDerivativeZ(f, out=o)
            p.FirstDerivativeX(f, out=o)
            p.FirstDerivativeY(f, out=o)
    elif which == "batch":
        from mpi_b200 import BatchNonPeriodic2D

        Nx, P, lam, fs, _ = W.batch_2d(512, seed=1237)
        p = BatchNonPeriodic2D(Nx, P, lam, 0.0, 2 * math.pi, -1.0, 1.0, precision="fp32_refine")
        f = p.pack([torch.from_numpy(x) for x in fs]).cuda()
        run = lambda: p.solve(f)  # noqa: E731
    else:
        from mpi_b200 import NonPeriodic3D

        f = torch.from_numpy(W.smooth_field_3d(NX, NY, NGLL, seed=SEED)).cuda()
        p = NonPeriodic3D(NX, NY, NGLL, NGLL, *DOM, Lambda=LAM, precision=which)
        run = lambda: p.SolvePDE(f)  # noqa: E731
    run()
    torch.cuda.synchronize()
    # the profiler range (ncu --profile-from-start off) holds the three solves
    # only, not plan creation and its autotuning
    torch.cuda.profiler.start()
    for _ in range(3):
        run()
    torch.cuda.synchronize()
    torch.cuda.profiler.stop()
    print("profile case done:", which, flush=True)


def _dist():
    ws = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return ws, rank, local


# ----------------------------------------------------------------- clocks --
class ClockSampler:
    """nvidia-smi sampling (200 ms) of SM clocks and throttle reasons."""

    FIELDS = ("clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,clocks_event_reasons.hw_slowdown,"
              "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
              "clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_id: str):
        self.path = tempfile.mktemp(suffix=".csv")
        self.proc = None
        self.gpu_id = gpu_id

    def start(self):
        try:
            self.fh = open(self.path, "w")
            self.proc = subprocess.Popen(["nvidia-smi", "-i", self.gpu_id, f"--query-gpu={self.FIELDS}",
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=self.fh, stderr=subprocess.DEVNULL)
        except Exception:
            self.proc = None

    def stop(self) -> dict:
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"], "samples": 0}
        self.proc.send_signal(signal.SIGTERM)
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        self.fh.close()
        rows = []
        for line in open(self.path):
            parts = [p.strip() for p in line.split(",")]
            if len(parts) >= 8:
                rows.append(parts)
        os.unlink(self.path)
        if not rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": [], "samples": 0}
        sm = [float(r[0]) for r in rows if r[0].replace(".", "").isdigit()]
        smax = [float(r[1]) for r in rows if r[1].replace(".", "").isdigit()]
        power = [float(r[2]) for r in rows if re.match(r"^[\d.]+$", r[2])]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[i] for r in rows for i in range(4) if r[4 + i].lower().startswith("active")})
        loaded = [s for s, p in zip(sm, power) if p > 250.0] or sm
        loaded.sort()
        return {"sm_mhz": loaded[len(loaded) // 2] if loaded else None, "sm_max_mhz": max(smax) if smax else None,
                "reasons": reasons, "samples": len(rows), "power_w_max": max(power) if power else None}


# ------------------------------------------------------------- reference --
def _ref_worker_init():
    # one thread per worker process (the reference is single-threaded; numpy's
    # BLAS would otherwise start a pool per process)
    for v in ("OMP_NUM_THREADS", "OPENBLAS_NUM_THREADS", "MKL_NUM_THREADS"):
        os.environ[v] = "1"
    sys.path.insert(0, HERE)


_REF_CACHE = {}


def _ref_solve_slab(ny: int):
    """One reference SolvePDE of the 256 x ny x 65 slab of the workload (seeded;
    the input is generated once per worker process)."""
    import numpy as np

    from mpi_b200 import workloads as W
    from oracle import oracle as O

    key = ("slab", ny)
    if key not in _REF_CACHE:
        _REF_CACHE[key] = W.smooth_field_3d(NX, ny, NGLL, seed=SEED)
    f = _REF_CACHE[key]
    z = np.zeros((NX, ny))
    t = time.perf_counter()
    if O.have_reference():
        O.ref_solve3d(f, z, z, xl=DOM[0], xr=DOM[1], yl=DOM[2], yr=DOM[3], zl=DOM[4], zr=DOM[5], lam=LAM)
    else:
        O.solve3d(f, z, z, Lx=DOM[1] - DOM[0], Ly=DOM[3] - DOM[2], Lz=DOM[5] - DOM[4], lam=LAM)
    return time.perf_counter() - t


def run_reference_arm(args, ws, rank):
    """The reference's own CPU solver (oracle/_ref, compiled from its sources;
    the C restatement when the reference was not available at build time) on
    every host core: each worker process runs one SolvePDE per step."""
    if rank != 0:
        return
    import multiprocessing as mp

    from oracle import oracle as O

    O.build()
    kind = "reference" if O.have_reference() else "port"
    cores = max(1, min(os.cpu_count() or 1, 64))
    # calibrate one 256 x 32 x 65 slab and size the per-worker sample so the
    # (steps + warmup) rounds stay near two minutes
    t32 = _ref_solve_slab(32)
    budget = 120.0 / max(1, args.steps + args.warmup)
    ny = 32
    while ny < NY and t32 * (2 * ny / 32) <= budget:
        ny *= 2
    ctx = mp.get_context("spawn")
    with ctx.Pool(cores, initializer=_ref_worker_init) as pool:
        for _ in range(args.warmup):
            pool.map(_ref_solve_slab, [ny] * cores)
        times = []
        for _ in range(args.steps):
            t = time.perf_counter()
            pool.map(_ref_solve_slab, [ny] * cores)
            times.append(time.perf_counter() - t)
    dof = NX * ny * NGLL * cores
    ms = 1e3 * sum(times) / len(times)
    val = dof / (ms * 1e-3) / 1e9
    sample = f"{cores} processes x one SolvePDE of the 256x{ny}x65 slab of the workload per step"
    line = {
        "impl": "reference", "metric": METRIC, "value": val, "unit": "GDOF/s", "n_gpus": ws, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": ms, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "f64", "data": "synthetic", "config": {"workload": WORKLOAD, "precision": "fp64", "device": "cpu"},
        "cpu_baseline": {"value": val, "unit": "GDOF/s", "cores": cores, "kind": kind, "sample": sample},
        "e2e": {"value": val, "unit": "GDOF/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


# ------------------------------------------------------------------- ours --
_T0 = time.perf_counter()


def _log(msg):
    """Progress with elapsed wall time, on stderr (the JSON line goes to stdout)."""
    sys.stderr.write(f"[bench {time.perf_counter() - _T0:7.1f} s] {msg}\n")
    sys.stderr.flush()


def rank_max(times, ws, device):
    """Element-wise max of per-rank timings over the process group (the replica
    whose GPU finished last sets the job time); the input list when ws == 1."""
    import torch

    t = torch.tensor([float(v) for v in times], dtype=torch.float64, device=device)
    if ws > 1:
        import torch.distributed as dist

        dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return [float(v) for v in t.cpu()]


def job_gdofs(dof_per_rank, ws, ms_per_step):
    """Whole-job throughput of ws replicas, each solving dof_per_rank per step."""
    return ws * dof_per_rank / (ms_per_step * 1e-3) / 1e9


def _peak_hbm():
    try:
        with open(os.path.join(HERE, "MEASURED_PEAKS.json")) as fh:
            return float(json.load(fh)["hbm_gbs"]), "measured"
    except Exception:
        return FALLBACK_HBM_GBS, "fallback"


def _traffic_from_profiles(stage: str):
    """DRAM bytes per launch of a stage's kernel at this workload, from the
    committed ncu summary (profiles/), or None."""
    path = os.path.join(HERE, "profiles", "traffic_256x256x65.txt")
    out = {}
    try:
        for line in open(path):
            m = re.match(r"^\s*(\w+)\s+(fp64|fp32_refine|fp32)\s+([\d.eE+]+)\s*$", line)
            if m and m.group(1) == stage:
                out[m.group(2)] = float(m.group(3))
    except OSError:
        pass
    return out or None


def _stage_model(eig: bool, spec_bytes: float, io_bytes: float) -> dict:
    """Kernel, algorithmic HBM bytes (inputs read once, outputs written once) and
    FP64 flops of each timed stage of the headline solve.  Five-kernel pipeline:
    x FFT, y FFT, row solves, inverse y, inverse x.  Eigen-basis pipeline: the
    GLL transform + x FFT (stage event 0-1), the y convolution (1-2) and the
    inverse (4-5); the coefficient spectrum holds 64 complex values per row."""
    nkx = NX // 2 + 1
    if not eig:
        rows_flops = 2.0 * nkx * NY * 2 * (NGLL - 2) ** 2  # folded transforms: n^2 MAC per real row
        fft_x = 2.5 * NGLL * NY * NX * math.log2(NX)       # R2C: 5 N log2 N per complex pair of columns
        fft_y = 5.0 * nkx * NGLL * NY * math.log2(NY)
        return {"fft_x": {"kernel": "fft_x", "bytes": io_bytes + spec_bytes, "flops": fft_x},
                "fft_y": {"kernel": "fft_y", "bytes": 2 * spec_bytes, "flops": fft_y},
                "rows": {"kernel": "rows", "bytes": 2 * spec_bytes, "flops": rows_flops},
                "ifft_y": {"kernel": "ifft_y", "bytes": 2 * spec_bytes, "flops": fft_y},
                "ifft_x": {"kernel": "ifft_x", "bytes": spec_bytes + io_bytes, "flops": fft_x}}
    s_bytes = 16.0 * nkx * NY * 64
    gll = 2.0 * NX * NY * 2 * 32 * 32                     # two 32 x 32 folded products per real row
    fft_x = 5.0 * 32 * NY * NX * math.log2(NX)           # 32 complex column pairs per plane
    fft_y = 2 * 5.0 * nkx * 64 * NY * math.log2(NY)      # forward and inverse
    return {"fft_x": {"kernel": "eig_fwd_kernel", "bytes": io_bytes + s_bytes, "flops": gll + fft_x},
            "fft_y": {"kernel": "eig_conv_kernel", "bytes": 2 * s_bytes, "flops": fft_y},
            "ifft_x": {"kernel": "eig_inv_kernel", "bytes": s_bytes + io_bytes, "flops": gll + fft_x}}


def _fp64_peak(dev) -> float:
    """Dense FP64 throughput of this GPU (TFLOP/s): torch.matmul float64 4096^3
    (cuBLAS DGEMM), best of 5, CUDA events."""
    import torch

    n = 4096
    a = torch.randn(n, n, dtype=torch.float64, device=dev)
    b = torch.randn(n, n, dtype=torch.float64, device=dev)
    c = torch.empty_like(a)
    torch.matmul(a, b, out=c)
    best = 1e30
    for _ in range(5):
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        torch.matmul(a, b, out=c)
        e1.record()
        torch.cuda.synchronize()
        best = min(best, e0.elapsed_time(e1))
    return 2.0 * n ** 3 / (best * 1e-3) / 1e12


def run_ours(args, ws, rank, local):
    import numpy as np
    import torch

    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    if ws > 1:
        import torch.distributed as dist

        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300))
    from mpi_b200 import NonPeriodic3D
    from mpi_b200 import workloads as W

    fnp = W.smooth_field_3d(NX, NY, NGLL, seed=SEED)
    f = torch.from_numpy(fnp).to(dev)
    dof = NX * NY * NGLL
    # plan creation: host setup (GLL grid, eigen-decompositions, per-shift data),
    # uploads and, the first time a shape is seen in the process, the autotuner
    plans, plan_ms = {}, {}
    for prec in ("fp32_refine", "fp64"):
        t0 = time.perf_counter()
        plans[prec] = NonPeriodic3D(NX, NY, NGLL, NGLL, *DOM, Lambda=LAM, precision=prec)
        torch.cuda.synchronize()
        plan_ms[prec + "_with_autotune"] = 1e3 * (time.perf_counter() - t0)
    t0 = time.perf_counter()
    NonPeriodic3D(NX, NY, NGLL, NGLL, *DOM, Lambda=LAM, precision="fp64").DestroyPDEPlan()
    torch.cuda.synchronize()
    plan_ms["fp64_autotune_cached"] = 1e3 * (time.perf_counter() - t0)
    fp64_peak = _fp64_peak(dev)
    outs = {k: p.SolvePDE(f) for k, p in plans.items()}
    torch.cuda.synchronize()
    flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device=dev)
    stream = torch.cuda.current_stream()
    uuid = str(torch.cuda.get_device_properties(local).uuid)
    clocks = ClockSampler(uuid if uuid.startswith("GPU-") else f"GPU-{uuid}")
    clocks.start()

    def barrier():
        torch.cuda.synchronize()
        if ws > 1:
            import torch.distributed as dist

            dist.barrier()
        torch.cuda.synchronize()

    def timed(fn):
        for _ in range(args.warmup):
            flush.add_(1.0)
            fn()
        barrier()
        evs = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(args.steps)]
        for e0, e1 in evs:
            flush.add_(1.0)  # evicts L2 (126 MB) between steps
            e0.record(stream)
            fn()
            e1.record(stream)
        barrier()
        return sum(e0.elapsed_time(e1) for e0, e1 in evs)

    res = {}
    for name, p in plans.items():
        # the headline's timed region is the profiler range (ncu --profile-from-start off)
        if name == "fp32_refine":
            torch.cuda.profiler.start()
        total_ms = timed(lambda p=p, name=name: p.SolvePDE(f, out=outs[name]))
        if name == "fp32_refine":
            torch.cuda.profiler.stop()
        res[name] = total_ms
    kernels = {k: p.kernels() for k, p in plans.items()}
    launches = len(kernels["fp32_refine"].split()) * args.steps  # the headline's timed solves

    # end to end through the public API: every step copies its f from pinned host
    # memory (H2D), solves, and reads its u back (D2H).  Steps are pipelined the
    # way a serving loop runs them: the H2D of step i + 1 and the D2H of step i - 1
    # run on their own streams (copy engines) while step i solves; device
    # buffers are double-buffered and every reuse waits on an event.
    fh = torch.from_numpy(fnp).pin_memory()
    uh = torch.empty_like(fh).pin_memory()
    fds = [torch.empty_like(f), torch.empty_like(f)]
    uds = [torch.empty_like(f), torch.empty_like(f)]
    s_in, s_out = torch.cuda.Stream(), torch.cuda.Stream()
    ev = {k: [torch.cuda.Event(), torch.cuda.Event()] for k in ("in", "solved", "out")}

    def e2e_run(n):
        for i in range(n):
            b = i & 1
            with torch.cuda.stream(s_in):
                if i >= 2:
                    s_in.wait_event(ev["solved"][b])  # solve i - 2 has read fds[b]
                fds[b].copy_(fh, non_blocking=True)
                ev["in"][b].record(s_in)
            stream.wait_event(ev["in"][b])
            if i >= 2:
                stream.wait_event(ev["out"][b])  # D2H i - 2 has read uds[b]
            plans["fp32_refine"].SolvePDE(fds[b], out=uds[b], stream=stream)
            ev["solved"][b].record(stream)
            with torch.cuda.stream(s_out):
                s_out.wait_event(ev["solved"][b])
                uh.copy_(uds[b], non_blocking=True)
                ev["out"][b].record(s_out)
        stream.wait_stream(s_in)
        stream.wait_stream(s_out)

    e2e_run(max(args.warmup, 3))
    barrier()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    e2e_run(args.steps)
    e1.record(stream)
    barrier()
    e2e_ms = e0.elapsed_time(e1)
    e2e_ok = bool(torch.equal(uds[(args.steps - 1) & 1].cpu(), uh))

    # the PCIe bound of e2e: the same pipelined H2D / D2H traffic with no solve
    def copy_run(n):
        for i in range(n):
            b = i & 1
            with torch.cuda.stream(s_in):
                if i >= 2:
                    s_in.wait_event(ev["out"][b])
                fds[b].copy_(fh, non_blocking=True)
                ev["in"][b].record(s_in)
            with torch.cuda.stream(s_out):
                s_out.wait_event(ev["in"][b])
                uh.copy_(fds[b], non_blocking=True)
                ev["out"][b].record(s_out)
        stream.wait_stream(s_in)
        stream.wait_stream(s_out)

    copy_run(3)
    barrier()
    e0.record(stream)
    copy_run(args.steps)
    e1.record(stream)
    barrier()
    copy_ms = e0.elapsed_time(e1) / args.steps

    # per-stage device time of the refined solve (events on its stream)
    pref = plans["fp32_refine"]
    pref.enable_stage_timing(True)
    acc = {}
    nst = max(5, min(args.steps, 50))
    for _ in range(nst):
        flush.add_(1.0)
        pref.SolvePDE(f, out=outs["fp32_refine"])
        for k, v in pref.stage_times().items():
            acc[k] = acc.get(k, 0.0) + v / nst
    pref.enable_stage_timing(False)
    side = {}
    if ws == 1 and not args.skip_side:
        st, wu = max(3, min(args.steps, 20)), 3
        _log("headline done")
        side["batch"] = _leg_batch(dev, flush, stream, st, wu, cpu=not args.skip_cpu_baseline)
        _log("batch leg done")
        side["adjoint"] = _leg_adjoint(dev, flush, stream, max(st, 50), wu)
        _log("adjoint leg done")
        side["fd"] = _leg_fd(dev, flush, stream, st, wu, cpu=not args.skip_cpu_baseline)
        _log("fd leg done")
        side["periodic"] = _leg_periodic(dev, flush, stream, st, wu, cpu=not args.skip_cpu_baseline)
        _log("periodic leg done")
        side["derivatives"] = _leg_derivatives(dev, flush, stream, st, wu)
        _log("derivatives leg done")
    clk = clocks.stop()

    # max over ranks
    t_ref, t_64, t_e2e = rank_max([res["fp32_refine"], res["fp64"], e2e_ms], ws, dev)
    ms_ref, ms_64, ms_e2e = t_ref / args.steps, t_64 / args.steps, t_e2e / args.steps

    # accuracy of the refined solve against the FP64 solve (and the reference below)
    u32 = outs["fp32_refine"].double()
    u64 = outs["fp64"]
    rel_vs_fp64 = float((u32 - u64).norm() / u64.norm())

    if rank == 0:
        peak, peak_kind = _peak_hbm()
        spec_bytes = 16.0 * (NX // 2 + 1) * NY * NGLL
        io_bytes = 8.0 * dof
        eig = kernels["fp32_refine"].startswith("eig_")
        stages = _stage_model(eig, spec_bytes, io_bytes)
        acc = {stages[k]["kernel"]: v for k, v in acc.items() if k in stages}
        dom = max(acc, key=acc.get)
        alg = {v["kernel"]: v["bytes"] for v in stages.values()}[dom]
        flops = {v["kernel"]: v["flops"] for v in stages.values()}[dom]
        achieved = alg / (acc[dom] * 1e-3) / 1e9
        traffic = _traffic_from_profiles(dom)
        refine_fp64 = "fdm_tc_refine_kernel" not in kernels["fp32_refine"]
        line = {
            "metric": METRIC,
            "value": job_gdofs(dof, ws, ms_ref),
            "unit": "GDOF/s",
            "n_gpus": ws,
            "steps": args.steps,
            "warmup": args.warmup,
            "ms_per_step": ms_ref,
            "higher_is_better": True,
            "scaling": "weak",
            "vs_baseline": None,
            "dtype": "f64" if refine_fp64 else "f32 solves + f64 residuals/FFTs",
            "data": "synthetic",
            "config": {"workload": WORKLOAD, "precision": "fp32_refine", "method": pref.info()["method"],
                       "refine_sweeps": 1, "l2": "256 MB buffer written before every timed solve",
                       "parallelism": f"replicas x{ws}", "dof_per_solve": dof,
                       "kernels": kernels["fp32_refine"],
                       "rows_kernel": ("FP64 arithmetic (the autotuner picked an FP64 path for the refined plan: "
                                       "faster than its FP32 tensor-core refinement kernel at this shape)"
                                       if refine_fp64 else "FP32 tensor-core solves + FP64 residual sweep")},
            "fp64": {"value": ws * dof / (ms_64 * 1e-3) / 1e9, "ms_per_step": ms_64,
                     "method": plans["fp64"].info()["method"], "kernels": kernels["fp64"]},
            "refine_over_fp64": ms_64 / ms_ref,
            "rel_l2_refine_vs_fp64": rel_vs_fp64,
            "plan_ms": plan_ms,
            "stage_ms": acc,
            "stage_hbm_frac": {k: {v["kernel"]: v["bytes"] for v in stages.values()}[k] / (t * 1e-3) / 1e9 / peak
                               for k, t in acc.items() if t > 0},
            "roofline": {"kernel": dom, "bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                         "frac": achieved / peak, "peak_source": f"{peak_kind} (MEASURED_PEAKS.json hbm_gbs)",
                         "algorithmic_bytes": alg, "traffic": (traffic or {}).get("fp32_refine"),
                         "compute": {"flops": flops, "achieved_tflops": flops / (acc[dom] * 1e-3) / 1e12,
                                     "fp64_peak_tflops": fp64_peak,
                                     "frac": flops / (acc[dom] * 1e-3) / 1e12 / fp64_peak,
                                     "peak_source": "measured here: torch.matmul float64 4096^3, best of 5"}},
            "e2e": {"value": ws * dof / (ms_e2e * 1e-3) / 1e9, "unit": "GDOF/s", "ms_per_step": ms_e2e,
                    "pipelined": "H2D of step i+1 and D2H of step i-1 overlap the solve of step i",
                    "last_result_read_back": e2e_ok,
                    "h2d_bytes_per_step": int(fh.numel() * 8), "d2h_bytes_per_step": int(uh.numel() * 8),
                    "copy_only_ms_per_step": copy_ms,
                    "frac_of_copy_bound": copy_ms / ms_e2e,
                    "bound": "pcie: the same pinned H2D + D2H per step with no solve"},
            "gpu_launches": launches,
            "clocks": clk,
        }
        line.update(side)
        if not args.skip_cpu_baseline and ws == 1:
            line["cpu_baseline"], ref_u = _cpu_baseline(fnp)
            _log("cpu baseline done")
            line["rel_l2_refine_vs_reference"] = float(np.linalg.norm(u32.cpu().numpy() - ref_u) / np.linalg.norm(ref_u))
            line["rel_l2_fp64_vs_reference"] = float(np.linalg.norm(u64.cpu().numpy() - ref_u) / np.linalg.norm(ref_u))
        print(json.dumps(line), flush=True)
    for p in plans.values():
        p.DestroyPDEPlan()
    if ws > 1:
        import torch.distributed as dist

        dist.barrier()
        dist.destroy_process_group()


# ------------------------------------------------------ side workloads --
# Measured on one GPU beside the headline and reported under their own keys.
BATCH_WORKLOAD = ("512 independent 2D problems, Nx from {32..512}, GLL order from {16..128}, lambda log-uniform "
                  "in [1e-2, 1e4], manufactured sin(3x)(1-y^2)e^y f on [0,2pi) x [-1,1], Dirichlet")
ADJ_WORKLOAD = ("3D Fourier 128 x Fourier 128 x GLL 65 (N=64), lambda=5, L = 0.5 ||u - u_obs||^2; forward solve, "
                "then dL/df and dL/dlambda by helm_solve_adjoint_misfit")
FD_WORKLOAD = "finite-difference FFT/Thomas, 1024 x 1024 periodic x 256 interior points, Dirichlet, lambda=1"
PER_WORKLOAD = ("3D Helmholtz periodic in all three directions, Fourier 256 x Fourier 256 x GLL 65 (N=64, one "
                "element), lambda=10, seeded smooth field; plus the reference's stock Periodic3D test "
                "(64 x 32 x 250, N=10: 25 elements, cyclic interface sweep)")
DER_WORKLOAD = "derivatives of a 256 x 256 x 65 FP64 field on the GLL grid of the headline plan"


def _ev_ms(fn, flush, stream, steps, warmup):
    """Mean device ms of fn over `steps` calls (CUDA events on `stream`), the L2
    flushed before each call."""
    import torch

    for _ in range(warmup):
        flush.add_(1.0)
        fn()
    torch.cuda.synchronize()
    evs = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(steps)]
    for e0, e1 in evs:
        flush.add_(1.0)
        e0.record(stream)
        fn()
        e1.record(stream)
    torch.cuda.synchronize()
    return sum(e0.elapsed_time(e1) for e0, e1 in evs) / steps


def _leg_batch(dev, flush, stream, steps, warmup, cpu):
    import numpy as np
    import torch

    from mpi_b200 import BatchNonPeriodic2D
    from mpi_b200 import workloads as W

    Nx, P, lam, fs, us = W.batch_2d(512, seed=1237)
    dof = sum(a * b for a, b in zip(Nx, P))
    res, sol, info = {}, {}, None
    for prec in ("fp32_refine", "fp64"):
        b = BatchNonPeriodic2D(Nx, P, lam, 0.0, 2 * math.pi, -1.0, 1.0, precision=prec)
        f = b.pack([torch.from_numpy(x) for x in fs]).to(dev)
        u = b.solve(f)
        res[prec] = _ev_ms(lambda b=b, f=f, u=u: b.solve(f, out=u), flush, stream, steps, warmup)
        sol[prec] = [x.cpu().numpy() for x in b.unpack(u)]
        info = b.info()
        b.destroy()

    def rel(a, c):
        return float(np.linalg.norm(a - c) / np.linalg.norm(c))

    out = {
        "workload": BATCH_WORKLOAD, "precision": "fp32_refine", "dof_per_solve": dof,
        "value": dof / (res["fp32_refine"] * 1e-3) / 1e9, "unit": "GDOF/s", "ms_per_step": res["fp32_refine"],
        "fp64": {"value": dof / (res["fp64"] * 1e-3) / 1e9, "ms_per_step": res["fp64"]},
        "max_rel_l2_refine_vs_fp64": max(rel(a, c) for a, c in zip(sol["fp32_refine"], sol["fp64"])),
        "max_rel_l2_fp64_vs_exact": max(rel(a, c) for a, c in zip(sol["fp64"], us)),
        "launch": "one cudaGraphLaunch per solve; size classes on concurrent streams inside the graph",
        "classes": info["classes"], "kernels_per_solve": info["kernels_per_solve"],
        "l2": "256 MB buffer written before every timed solve",
    }
    if cpu:
        from oracle import oracle as O

        O.build()
        if O.have_reference():
            t, errs = 0.0, []
            for f, la, u in zip(fs, lam, sol["fp32_refine"]):
                z = np.zeros(f.shape[0])
                r, ms = O.ref_solve2d(f, z, z, xl=0.0, xr=2 * math.pi, yl=-1.0, yr=1.0, lam=la, return_time=True)
                t += ms
                errs.append(rel(u, r))
            out["cpu_baseline"] = {"value": dof / (t * 1e-3) / 1e9, "unit": "GDOF/s", "cores": 1, "kind": "reference",
                                   "sample": "the reference's SolvePDE of each of the 512 problems, one core, "
                                             "its own SolvePDE clock summed"}
            out["max_rel_l2_refine_vs_reference"] = max(errs)
            # the same 512 reference solves spread over the host's cores (spawned
            # processes, one share each; wall time of the pool's map, pool warm)
            import multiprocessing as mp

            cores = max(1, min(os.cpu_count() or 1, 64))
            if cores > 1:
                shares = [list(range(i, len(Nx), cores)) for i in range(cores)]
                with mp.get_context("spawn").Pool(cores, initializer=_ref_worker_init) as pool:
                    pool.map(_ref_batch_share, [[0]] * cores)
                    t0 = time.perf_counter()
                    pool.map(_ref_batch_share, shares)
                    wall = time.perf_counter() - t0
                out["cpu_baseline_all_cores"] = {"value": dof / wall / 1e9, "unit": "GDOF/s", "cores": cores,
                                                 "kind": "reference",
                                                 "sample": "the 512 reference SolvePDE calls split over the cores, "
                                                           "wall time"}
    return out


def _ref_batch_share(idx):
    """The reference's plan + SolvePDE for the listed problems of the 512-problem batch."""
    import numpy as np

    from mpi_b200 import workloads as W
    from oracle import oracle as O

    if "batch" not in _REF_CACHE:  # generated once per worker (the warm-up map)
        _REF_CACHE["batch"] = W.batch_2d(512, seed=1237)
    Nx, P, lam, fs, _ = _REF_CACHE["batch"]
    for i in idx:
        z = np.zeros(fs[i].shape[0])
        O.ref_solve2d(fs[i], z, z, xl=0.0, xr=2 * math.pi, yl=-1.0, yr=1.0, lam=lam[i])
    return len(idx)


def _leg_adjoint(dev, flush, stream, steps, warmup):
    import torch

    from mpi_b200 import NonPeriodic3D
    from mpi_b200 import workloads as W

    n, P, la = 128, 65, 5.0
    f = torch.from_numpy(W.smooth_field_3d(n, n, P, seed=11)).to(dev)
    uobs = torch.from_numpy(W.smooth_field_3d(n, n, P, seed=12)).to(dev)
    out = {"workload": ADJ_WORKLOAD}
    for prec in ("fp32", "fp64"):
        p = NonPeriodic3D(n, n, P, P, *DOM, Lambda=la, precision=prec)
        u = p.SolvePDE(f)
        fwd = _ev_ms(lambda: p.SolvePDE(f, out=u), flush, stream, steps, warmup)
        def both():
            # forward, then dL/df and dL/dlambda of L = 1/2 ||u - u_obs||^2 (the
            # misfit u - u_obs is formed inside the adjoint's first pass)
            p.SolvePDE(f, out=u)
            p.SolveAdjointMisfit(u, uobs)

        fb = _ev_ms(both, flush, stream, steps, warmup)
        out[prec] = {"forward_ms": fwd, "forward_plus_adjoint_ms": fb, "ratio": fb / fwd}
        p.DestroyPDEPlan()
    return out


def _leg_fd(dev, flush, stream, steps, warmup, cpu=False):
    import torch

    from mpi_b200 import Helmholtz3DFD
    from mpi_b200 import workloads as W

    Nx, Ny, Nz = 1024, 1024, 256
    f = torch.from_numpy(W.smooth_field_fd(Nx, Ny, Nz, seed=1239)).to(dev)
    dof = Nx * Ny * Nz
    out = {"workload": FD_WORKLOAD, "dof_per_solve": dof}
    us = {}
    peak, _ = _peak_hbm()
    f32 = f.float()
    for prec in ("fp32", "fp32_refine", "fp64"):
        p = Helmholtz3DFD(Nx, Ny, Nz, 0.0, 1.0, 0.0, 1.0, 0.0, 1.0, Lambda=1.0, precision=prec)
        # the FP32 plan reads f and writes u in FP32 (4 B per point each way)
        fi = f
        if prec == "fp32":
            p.set_io_bytes(4)
            fi = f32
        u = p.SolvePDE(fi)
        fwd = _ev_ms(lambda: p.SolvePDE(fi, out=u), flush, stream, steps, warmup)
        ubar = u.double()  # the adjoint takes and returns FP64 arrays
        adj = _ev_ms(lambda: p.SolveAdjoint(ubar), flush, stream, steps, warmup)
        out[prec] = {"value": dof / (fwd * 1e-3) / 1e9, "unit": "GDOF/s", "forward_ms": fwd, "adjoint_ms": adj}
        if prec == "fp32_refine":
            # FP32 solve + 2 sweeps of FP64 stencil residual and FP32 correction
            out[prec]["kernels"] = p.kernels()
            us[prec] = u
            p.DestroyPDEPlan()
            continue
        # per-pass HBM fraction at this size: algorithmic bytes = input + output of each pass
        p.enable_stage_timing(True)
        st = {}
        for _ in range(3):
            flush.add_(1.0)
            p.SolvePDE(fi, out=u)
            for k, v in p.stage_times().items():
                st[k] = st.get(k, 0.0) + v / 3
        p.enable_stage_timing(False)
        eb = 8 if prec == "fp64" else 4
        real_b, spec_b = dof * eb, (Nx // 2 + 1) * Ny * Nz * 2 * eb
        pass_bytes = {"fft_x": real_b + spec_b, "fft_y": 2 * spec_b, "rows": 2 * spec_b, "ifft_y": 2 * spec_b,
                      "ifft_x": spec_b + real_b}
        out[prec]["stage_ms"] = st
        out[prec]["stage_hbm_frac"] = {k: pass_bytes[k] / (st[k] * 1e-3) / 1e9 / peak for k in st if st[k] > 0}
        us[prec] = u.double()
        p.DestroyPDEPlan()
    out["rel_l2_fp32_vs_fp64"] = float((us["fp32"] - us["fp64"]).norm() / us["fp64"].norm())
    out["rel_l2_fp32_refine_vs_fp64"] = float((us["fp32_refine"] - us["fp64"]).norm() / us["fp64"].norm())
    if cpu:
        # no reference implementation of a direct FD solve exists (HypreFDM is
        # iterative and needs HYPRE): the C restatement on one core, 256 x 256 x 256
        import numpy as np

        from oracle import oracle as O

        O.build()
        n = 256
        fs = W.smooth_field_fd(n, n, Nz, seed=1239)
        z = np.zeros((n, n))
        t0 = time.perf_counter()
        O.fd3d_solve(fs, z, z, Lx=1.0, Ly=1.0, Lz=1.0, lam=1.0)
        t = time.perf_counter() - t0
        out["cpu_baseline"] = {"value": n * n * Nz / t / 1e9, "unit": "GDOF/s", "cores": 1, "kind": "port",
                               "sample": "the C restatement's FFT/tridiagonal solve of 256 x 256 x 256 (the "
                                         "workload's z size, 1/16 of its x-y plane), one core"}
    return out


def _leg_periodic(dev, flush, stream, steps, warmup, cpu=False):
    import numpy as np
    import torch

    from mpi_b200 import Periodic3D
    from mpi_b200 import workloads as W

    f = torch.from_numpy(W.smooth_field_3d(NX, NY, NGLL, seed=SEED)).to(dev)
    dof = NX * NY * NGLL
    out = {"workload": PER_WORKLOAD, "dof_per_solve": dof}
    us = {}
    for prec in ("fp64", "fp32_refine"):
        p = Periodic3D(NX, NY, NGLL, NGLL, *DOM, Lambda=LAM, precision=prec)
        u = p.SolvePDE(f)
        ms = _ev_ms(lambda: p.SolvePDE(f, out=u), flush, stream, steps, warmup)
        out[prec] = {"value": dof / (ms * 1e-3) / 1e9, "unit": "GDOF/s", "ms_per_solve": ms}
        us[prec] = u
        p.DestroyPDEPlan()
    out["rel_l2_refine_vs_fp64"] = float((us["fp32_refine"] - us["fp64"]).norm() / us["fp64"].norm())
    fs, ue = W.stock_periodic_3d()
    ps = Periodic3D(64, 32, 250, 10, 0.0, 1.0, 0.0, 1.0, 0.0, 1.0, Lambda=1.0)
    fsd = torch.from_numpy(fs).to(dev)
    us_ = ps.SolvePDE(fsd)
    ms = _ev_ms(lambda: ps.SolvePDE(fsd, out=us_), flush, stream, steps, warmup)
    out["stock_periodic_3d"] = {"value": fs.size / (ms * 1e-3) / 1e9, "unit": "GDOF/s", "ms_per_solve": ms,
                                "max_err_vs_exact": float(np.abs(us_.cpu().numpy() - ue).max())}
    ps.DestroyPDEPlan()
    if cpu:
        from oracle import oracle as O

        O.build()
        n = 64
        fsmall = W.smooth_field_3d(n, n, NGLL, seed=SEED)
        kind = "reference" if O.have_reference() else "port"
        t0 = time.perf_counter()
        if kind == "reference":
            O.ref_psolve3d(fsmall, xl=DOM[0], xr=DOM[1], yl=DOM[2], yr=DOM[3], zl=DOM[4], zr=DOM[5], lam=LAM)
        else:
            O.psolve3d(fsmall, Lx=DOM[1] - DOM[0], Ly=DOM[3] - DOM[2], Lz=DOM[5] - DOM[4], lam=LAM)
        t = time.perf_counter() - t0
        out["cpu_baseline"] = {"value": n * n * NGLL / t / 1e9, "unit": "GDOF/s", "cores": 1, "kind": kind,
                               "sample": "the reference's Periodic3D SolvePDE of 64 x 64 x 65 (1/16 of the "
                                         "workload's x-y plane), one core"}
    return out


def _leg_derivatives(dev, flush, stream, steps, warmup):
    """GLL-direction and spectral derivatives at the headline shape; HBM roofline
    with algorithmic bytes = one read and one write of the field per call."""
    import torch

    from mpi_b200 import NonPeriodic3D

    p = NonPeriodic3D(NX, NY, NGLL, NGLL, *DOM, Lambda=LAM)
    u = torch.randn(NX, NY, NGLL, dtype=torch.float64, device=dev)
    du = torch.empty_like(u)
    peak, src = _peak_hbm()
    nbytes = 2 * u.numel() * 8
    out = {"workload": DER_WORKLOAD, "algorithmic_bytes": nbytes, "peak_gbs": peak, "peak_source": src}
    for name, axis in (("d_dz_gll", "Z"), ("d_dx_fourier", "X"), ("d_dy_fourier", "Y")):
        for order in (1, 2):
            fn = getattr(p, ("First" if order == 1 else "Second") + "Derivative" + axis)
            ms = _ev_ms(lambda: fn(u, out=du), flush, stream, steps, warmup)
            gbs = nbytes / (ms * 1e-3) / 1e9
            out[f"{name}_{order}"] = {"ms": ms, "achieved_gbs": gbs, "frac": gbs / peak, "launches": 1}
    p.DestroyPDEPlan()
    return out


def _cpu_baseline(fnp):
    """The reference's own FP64 CPU solve (oracle/_ref) of the full workload on
    one host core, twice; its output is also the error reference."""
    import numpy as np

    from oracle import oracle as O

    O.build()
    z = np.zeros((NX, NY))
    kind = "reference" if O.have_reference() else "port"
    times = []
    u = None
    for _ in range(2):
        t = time.perf_counter()
        if kind == "reference":
            u = O.ref_solve3d(fnp, z, z, xl=DOM[0], xr=DOM[1], yl=DOM[2], yr=DOM[3], zl=DOM[4], zr=DOM[5], lam=LAM)
        else:
            u = O.solve3d(fnp, z, z, Lx=DOM[1] - DOM[0], Ly=DOM[3] - DOM[2], Lz=DOM[5] - DOM[4], lam=LAM)
        times.append(time.perf_counter() - t)
    t = min(times)
    return ({"value": NX * NY * NGLL / t / 1e9, "unit": "GDOF/s", "cores": 1, "kind": kind,
             "sample": "two full SolvePDE calls of the 256x256x65 workload on one core (best)"}, u)


def main():
    args = _args()
    ws, rank, local = _dist()
    if args.profile_case:
        profile_case(args.profile_case)
    elif args.impl == "reference":
        run_reference_arm(args, ws, rank)
    else:
        run_ours(args, ws, rank, local)


if __name__ == "__main__":
    main()
