"""Throughput benchmark of the channel-DNS time step on B200.

Workload (one instance per GPU): 128x128 Fourier modes (192x192 physical
with the 3/2 pad), ny = 153 on the reference's stretched grid, Re_tau = 180
(Re = 180/sqrt(3.0675e-3)), fixed dt = 5e-4, seeded perturbed-laminar
initial state.  A step is one RK3 step (3 substeps).  The metric counts
grid points Nx*Nz*ny times substeps per second over the whole job.

  value  device-resident state, one CUDA graph per step, CUDA events on the
         engine's stream, max over ranks
  e2e    the host-buffer C-ABI call lh_step_host: pinned host arrays in the
         reference column layout are uploaded, stepped and downloaded every
         step
  --impl reference   the reference algorithm on the host cores (the C
         restatement, all threads), on a bounded sample of the same workload

Usage: python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]
N > 1 runs under torchrun, one independent instance per rank (weak scaling).
"""
from __future__ import annotations

import argparse
import math
import json
import os
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(ROOT, "final-single-block-_b200"))

METRIC = "FP64 grid-pt·substeps/s: served batch vs plain 1-instance on B200; p50/p99 lat"
UNIT = "grid-pt*substeps/s"
RE_TAU = 180.0
MPGX = -3.0675e-3


def workload_desc(n: int = 128):
    """The plain workload: Nx = Nz = n Fourier modes (128: the headline
    configuration), ny = 153, Re_tau = 180, dt = 5e-4."""
    from lh_b200 import Desc, re_from_retau
    return Desc(Nx=n, Nz=n, ny=153, Re=re_from_retau(RE_TAU, MPGX), mpgx=MPGX, dt_mode=1, dt=5e-4)


def config_dict(desc, n_gpus):
    m = 3 * desc.Nx // 2
    return {
        "workload": f"plain drop-in, one channel instance per GPU: Nx=Nz={desc.Nx} modes ({m}x{m} physical, 3/2 "
                    "pad), ny=153 polynomial-stretched y (dyq=10, p=5), Re_tau=180, dt=5e-4, RK3, seeded "
                    "perturbed-laminar initial state",
        "Nx": desc.Nx, "Nz": desc.Nz, "ny": desc.ny, "Re": desc.Re, "dt": desc.dt,
        "grid_points": desc.points(), "substeps_per_step": 3,
        "instances_per_gpu": 1, "parallelism": f"replicas x{n_gpus}",
        "l2": ("state and per-substep traffic (~0.45 GB resident) exceed the 126 MB L2; no flush"
               if desc.Nx >= 128 else "diagnostic size: the state fits in the 126 MB L2 (not the headline workload)"),
    }


class ClockSampler:
    """nvidia-smi clock/throttle samples while the timed region runs."""

    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index: int):
        self.index = index
        self.rows = []
        self.proc = None

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.index), f"--query-gpu={self.Q}",
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except OSError:
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.rows.append([x.strip() for x in line.split(",")])

    def __exit__(self, *a):
        if self.proc:
            time.sleep(0.25)
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()
            self.t.join(timeout=2)

    def summary(self):
        if not self.rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"], "samples": 0}
        sm = [float(r[1]) for r in self.rows if len(r) >= 9 and r[1].replace(".", "").isdigit()]
        mx = [float(r[2]) for r in self.rows if len(r) >= 9 and r[2].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = set()
        for r in self.rows:
            for k, n in enumerate(names):
                if len(r) >= 9 and r[5 + k].lower().startswith("active"):
                    reasons.add(n)
        return {"sm_mhz": float(np.median(sm)) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": sorted(reasons), "samples": len(self.rows)}


def peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        with open(p) as f:
            j = json.load(f)
        return float(j["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


def fp64_peak_tflops(n: int = 8192, reps: int = 5) -> float:
    """FP64 denominator measured on this GPU: a float64 GEMM of n^3 (2 n^3
    flops), best of `reps`, timed with CUDA events."""
    import torch
    a = torch.randn(n, n, dtype=torch.float64, device="cuda")
    b = torch.randn(n, n, dtype=torch.float64, device="cuda")
    torch.matmul(a, b)
    best = float("inf")
    for _ in range(reps):
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        torch.matmul(a, b)
        e1.record()
        e1.synchronize()
        best = min(best, e0.elapsed_time(e1) * 1e-3)
    del a, b
    torch.cuda.empty_cache()
    return 2.0 * n ** 3 / best / 1e12


def fft_flops_per_substep(desc) -> float:
    """FFT flops of one substep counted as 5 N log2 N per complex transform of
    length N (2.5 N log2 N per real one): 12 ny [Mz 2.5 Mx log2 Mx + (Nx/2+1)
    5 Mz log2 Mz] -- twelve 2-D transforms per plane pair, the z transforms
    pruned to the Nx/2+1 retained x modes."""
    Mx, Mz = 3 * desc.Nx // 2, 3 * desc.Nz // 2
    return 12.0 * desc.ny * (Mz * 2.5 * Mx * math.log2(Mx) + (desc.Nx // 2 + 1) * 5.0 * Mz * math.log2(Mz))


TRAFFIC_SUMMARY = os.path.join(ROOT, "profiles", "dram_traffic_plain_128x128x153.md")


def ncu_traffic():
    """Measured DRAM bytes (read + write) per substep for each kernel class,
    from the committed ncu summary: lines ``dram_bytes_per_substep[<class>]: N``."""
    out = {}
    if os.path.exists(TRAFFIC_SUMMARY):
        with open(TRAFFIC_SUMMARY) as f:
            for line in f:
                line = line.strip().strip("`")
                if line.startswith("dram_bytes_per_substep[") and "]:" in line:
                    key, val = line[len("dram_bytes_per_substep["):].split("]:", 1)
                    try:
                        out[key] = float(val)
                    except ValueError:
                        pass
    return out


def cpu_rate(desc, sample_steps: int, threads: int):
    """Reference algorithm on the host (oracle, OpenMP) -> (rate, seconds, cores)."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle as O
    from lh_b200.state import perturbed_laminar  # numpy only: the engine library is not loaded
    cfg = O.Config(Nx=desc.Nx, Nz=desc.Nz, ny=desc.ny, Re=desc.Re, mpgx=desc.mpgx, dt_mode=O.DT_FIXED,
                   dt_fixed=desc.dt, nthreads=threads)
    o = O.Oracle(cfg, threaded=True)
    yu, yv = o.array(0), o.array(1)  # the oracle's own ygrid
    ic = perturbed_laminar(desc, 20260002, yu, yv)
    o.load_state(*ic)
    o.step(1)  # warm caches and page in
    t0 = time.perf_counter()
    o.step(sample_steps)
    dt = time.perf_counter() - t0
    return desc.points() * 3 * sample_steps / dt, dt


def run_reference(args, rank, world):
    if rank != 0:
        return
    desc = workload_desc(args.nx)
    threads = os.cpu_count() or 1
    steps = max(1, args.steps)
    warm = max(0, min(args.warmup, 1))
    # bounded sample: each timed step is one RK3 step of the full workload
    sample = min(steps, 3)
    rate, secs = cpu_rate(desc, sample, threads)
    line = {
        "impl": "reference", "metric": METRIC, "value": rate, "unit": UNIT, "n_gpus": world,
        "steps": sample, "warmup": warm, "ms_per_step": 1e3 * secs / sample, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": config_dict(desc, world),
        "cpu_baseline": {"value": rate, "unit": UNIT, "cores": threads, "kind": "port",
                         "sample": f"{sample} RK3 steps of the full 128x128x153 workload, C restatement "
                                   f"of the reference (OpenMP, {threads} threads); the Fortran build needs "
                                   f"a Fortran compiler and MPI, absent here"},
        "e2e": {"value": rate, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


def field_bytes(desc):
    """F: one complex FP64 field over every column and y row."""
    return 16 * desc.ncols * desc.ny


def substep_alg_bytes(desc):
    """Algorithmic HBM bytes of one RK3 substep, 20 F: the plane pass reads
    u1 u2 u3 and writes Nu1 Nu2 Nu3 (6 F); the column pass reads u1 u2 u3 p,
    the new and the previous Nu (10 F) and writes u1 u2 u3 p (4 F)."""
    return 20 * field_bytes(desc)


# HBM bytes each kernel class of this design moves per substep, in units of
# F: the z-inverse reads the three velocity planes, the x-products kernel
# works on the L2-resident staging only, the z-forward writes the x/z parts
# of Nu and the three y-flux spectra, the column pass reads 13 fields and
# writes 7 (u1 u2 u3 p, Nu x3).
FIELD_PASSES = {"z_inverse": 3, "x_products": 0, "z_forward": 6, "dt": 0, "column": 20}


def _batch_rate(b, pts, K):
    """grid-pt*substeps/s of a batch over K timed steps (after 3 warm steps)."""
    b.step(3)
    b.synchronize()
    t0 = time.perf_counter()
    b.step(K)
    b.synchronize()
    bt = time.perf_counter() - t0
    return pts * 3 * K / bt, 1e3 * bt / K


def plain_small():
    """The first configuration: one 32x32x153 instance, dt = 1e-3, Re_tau = 180,
    device-resident, CUDA events on the engine's stream (it fits in L2)."""
    import torch
    from lh_b200 import Desc, Engine, grids, perturbed_laminar, re_from_retau
    d = Desc(Nx=32, Nz=32, ny=153, Re=re_from_retau(RE_TAU, MPGX), mpgx=MPGX, dt_mode=1, dt=1e-3)
    e = Engine(d)
    e.upload(*perturbed_laminar(d, 20260001, *grids(d)))
    e.step(5)
    e.synchronize()
    st = torch.cuda.ExternalStream(e.stream())
    a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    K = 100
    a.record(st)
    e.step(K)
    b.record(st)
    b.synchronize()
    e.synchronize()
    ms = a.elapsed_time(b) / K
    e.close()
    return {"workload": "plain, one 32x32x153 instance, dt 1e-3, Re_tau 180, 100 timed steps (the configuration's "
                        "100-step run), state L2-resident", "value": d.points() * 3 / (ms * 1e-3), "unit": UNIT,
            "ms_per_step": ms}


def batched_and_served(args):
    """Throughput of the batched engine on the uniform batch (64 instances of
    32x32x153, Re_tau and dt drawn per instance) and on the uneven batch (16 x
    32^2, 8 x 64^2, 4 x 128^2 at ny = 153 and 1 x 256^2 x 257, Re_tau in
    [180, 550], tanh(2) grid), and of the serving loop on a Poisson stream,
    next to the plain single-instance path on the same stream and clock."""
    from lh_b200 import Batch, Desc, grids, perturbed_laminar, re_from_retau
    from lh_b200.serve import Request, poisson_stream, run_plain, serve
    rng = np.random.default_rng(20260003)
    b = Batch()
    pts = 0
    for k in range(64):
        d = Desc(Nx=32, Nz=32, ny=153, Re=re_from_retau(rng.uniform(100, 400), MPGX), mpgx=MPGX, dt_mode=1,
                 dt=rng.uniform(5e-4, 2e-3))
        yu, yv = grids(d)
        b.add(d, *perturbed_laminar(d, 20260003 + 1000 * k, yu, yv))
        pts += d.points()
    rate, ms = _batch_rate(b, pts, 10)
    b.close()
    batched = {"workload": "64 instances of 32x32x153, Re_tau~U[100,400], dt~U[5e-4,2e-3], one launch per "
                           "kernel class and chunk round per substep, CUDA graph",
               "value": rate, "unit": UNIT, "ms_per_step": ms}
    rng = np.random.default_rng(20260004)
    b = Batch()
    pts = 0
    k = 0
    for n, ny, count in ((32, 153, 16), (64, 153, 8), (128, 153, 4), (256, 257, 1)):
        for _ in range(count):
            d = Desc(Nx=n, Nz=n, ny=ny, Re=re_from_retau(rng.uniform(180, 550), MPGX), mpgx=MPGX, grid_type=1,
                     gamma=2.0, dt_mode=1, dt=2.5e-4 if n >= 128 else 5e-4)
            yu, yv = grids(d)
            b.add(d, *perturbed_laminar(d, 20260004 + 1000 * k, yu, yv))
            pts += d.points()
            k += 1
    rate_u, ms_u = _batch_rate(b, pts, 10)
    b.close()
    uneven = {"workload": "16 x 32x32x153, 8 x 64x64x153, 4 x 128x128x153 and 1 x 256x256x257, Re_tau~U[180,550], "
                          "tanh(2) y grid, dt 5e-4 (2.5e-4 at 128^2 and above), shared substep launches, CUDA graph; "
                          "10 timed steps (the configuration's 500-step run measured on a sample)",
              "value": rate_u, "unit": UNIT, "ms_per_step": ms_u}
    n_req = args.serve_requests
    steps = (200, 5000) if args.serve_full_steps else (20, 200)
    scale = args.serve_time_scale
    mk = lambda: poisson_stream(n_req, 4.0, np.random.default_rng(20260005), [32, 64, 128, 192], [97, 153, 257],
                                steps=steps, dt=(2e-4, 5e-4))
    # one short request of every grid through both paths first, so neither timed
    # run pays the first launches of a size's kernels or its first plans
    warm = [Request(k, Desc(Nx=n, Nz=n, ny=ny, Re=re_from_retau(180.0, MPGX), mpgx=MPGX, dt_mode=1, dt=2e-4),
                    777 + k, 2, 0.0)
            for k, (n, ny) in enumerate((n, ny) for n in (32, 64, 128, 192) for ny in (97, 153, 257))]
    serve(warm, hbm_budget=150 << 30, max_chunk=50, keep_results=False)
    run_plain(warm, keep_results=False)
    reqs = mk()
    st = serve(reqs, hbm_budget=150 << 30, max_chunk=50, keep_results=False, time_scale=scale)
    reqs2 = mk()
    tp = run_plain(reqs2, keep_results=False, time_scale=scale)
    work = sum(r.work for r in reqs2)
    ttc_plain = [r.finished - r.arrival * scale for r in reqs2]
    served = {"workload": f"{n_req} requests, Poisson arrivals (4/s, replayed at {scale:g}x the arrival times), "
                          f"grids {{32,64,128,192}}^2 x ny {{97,153,257}}, Re_tau~U[100,550], dt~U[2e-4,5e-4] "
                          f"(the configuration names no dt; the reference's CFL rule diverges on laminar starts at "
                          f"high Re_tau), steps "
                          f"log-U[{steps[0]},{steps[1]}], 150 GB budget; both paths warmed first by one 2-step request "
                          f"of every grid",
              "value": st.throughput, "unit": UNIT, "p50_ttc_s": st.p50, "p99_ttc_s": st.p99,
              "mean_live": st.mean_live, "max_live": st.max_live, "wall_s": st.wall,
              "plain_same_stream": work / tp, "plain_wall_s": tp,
              "plain_p50_ttc_s": float(np.percentile(ttc_plain, 50)),
              "plain_p99_ttc_s": float(np.percentile(ttc_plain, 99)),
              "served_over_plain": st.throughput / (work / tp),
              "diverged": [{"N": r.desc.Nx, "ny": r.desc.ny, "Re_tau": round(r.desc.Re * math.sqrt(-MPGX), 1),
                            "steps": r.nsteps} for r in reqs if r.error],
              "diverged_plain": sum(1 for r in reqs2 if r.error)}
    return batched, uneven, served


def max_over_ranks(vals, world, device):
    """Element-wise maximum of a list of floats over all ranks (all_reduce MAX);
    the identity at world size 1."""
    import torch
    t = torch.tensor(vals, dtype=torch.float64, device=device)
    if world > 1:
        import torch.distributed as tdist
        tdist.all_reduce(t, op=tdist.ReduceOp.MAX)
    return [float(x) for x in t.tolist()]


def job_rate(world, units_per_rank, seconds):
    """Whole-job throughput: the units all ranks processed over the slowest
    rank's time (each rank runs its own instance, weak scaling)."""
    return world * units_per_rank / seconds


def run_ours(args, rank, world, local_rank):
    import torch
    from lh_b200 import Engine, grids, perturbed_laminar
    torch.cuda.set_device(local_rank)
    desc = workload_desc(args.nx)
    yu, yv = grids(desc)
    ic = perturbed_laminar(desc, 20260002 + 1000 * rank, yu, yv)
    e = Engine(desc)
    e.upload(*ic)
    # launch shapes from the autotuner (measured on a scratch instance before
    # the timed region, or read from its cache)
    tuned = None if args.no_tune else e.autotune()
    st = torch.cuda.ExternalStream(e.stream())
    W, K = args.warmup, args.steps
    e.step(W)
    e.synchronize()
    pts_sub = desc.points() * 3
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    dist = world > 1
    if dist:
        import torch.distributed as tdist
        tdist.barrier()
    torch.cuda.synchronize()
    with ClockSampler(local_rank) as clk:
        ev0.record(st)
        e.step(K)
        ev1.record(st)
        ev1.synchronize()
    torch.cuda.synchronize()
    ms = ev0.elapsed_time(ev1)
    e.synchronize()  # error word: non-finite state fails the run
    (ms_max,) = max_over_ranks([ms], world, "cuda")
    value = job_rate(world, pts_sub * K, ms_max * 1e-3)
    launches_per_step = None

    # per-kernel breakdown with CUDA events on the engine's stream
    prof = e.profile(2)
    launches_per_step = sum(n for _, n in prof.values()) // 2
    dom = max(prof.items(), key=lambda kv: kv[1][0])
    hbm, src = peaks()
    F = field_bytes(desc)
    alg = substep_alg_bytes(desc)
    sub_s = ms_max * 1e-3 / (3 * K)  # one substep, from the timed region
    achieved = alg / sub_s / 1e9
    # the committed ncu summary covers the 128x128x153 workload only
    traffic = ncu_traffic() if desc.Nx == 128 else {}
    traffic_sub = sum(traffic.values()) if traffic else None
    kernels = {}
    for name, (kms, kn) in prof.items():
        per_sub = kms / 6.0  # 2 steps x 3 substeps
        kb = FIELD_PASSES[name] * F
        kernels[name] = {"ms_per_substep": per_sub, "launches_per_substep": kn / 6.0,
                         "share": kms / sum(v[0] for v in prof.values()),
                         "design_hbm_bytes_per_substep": kb,
                         "achieved_gbs": kb / (per_sub * 1e-3) / 1e9 if per_sub > 0 else None,
                         "ncu_dram_bytes_per_substep": traffic.get(name)}

    # end to end through the host-buffer call
    nu, nv, nc = desc.nyu, desc.nyv, desc.ncols
    shapes = [(nc, nu + 2), (nc, nv + 2), (nc, nu + 2), (nc, nu)]
    host = []
    for shp, src_arr in zip(shapes, ic):
        t = torch.empty(int(np.prod(shp)) * 2, dtype=torch.float64, pin_memory=True)
        t.numpy()[:] = np.ascontiguousarray(src_arr).view(np.float64).ravel()
        host.append(t)
    addrs = [t.data_ptr() for t in host]
    nbytes = sum(t.numel() * 8 for t in host)
    Ke = max(2, min(K, 10))
    e.step_host(addrs, 1)  # warm
    if dist:
        tdist.barrier()
    # device time on the engine's stream around the host-buffer calls: each
    # call uploads, steps and downloads on that stream before it returns
    ev2, ev3 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    torch.cuda.synchronize()
    ev2.record(st)
    for _ in range(Ke):
        e.step_host(addrs, 1)
    ev3.record(st)
    ev3.synchronize()
    (e2e_ms,) = max_over_ranks([ev2.elapsed_time(ev3)], world, "cuda")
    e2e_val = job_rate(world, pts_sub * Ke, e2e_ms * 1e-3)

    batched = uneven = served = small = None
    if rank == 0 and world == 1 and not args.no_serve:
        small = plain_small()
        batched, uneven, served = batched_and_served(args)

    fp64 = None
    if rank == 0 and world == 1:
        fl = fft_flops_per_substep(desc)
        pk = fp64_peak_tflops()
        fp64 = {"kernel": "the FFT flops of one substep (plane pass k_zinv/k_xprod/k_zfwd) over the whole substep time",
                "achieved": fl / sub_s / 1e12, "peak": pk, "unit": "TFLOP/s", "frac": fl / sub_s / 1e12 / pk,
                "flops_per_substep": fl,
                "peak_source": "measured on this GPU: float64 GEMM 8192^3 (torch.matmul), best of 5"}

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu:
        threads = os.cpu_count() or 1
        rate, secs = cpu_rate(desc, 2, threads)
        cpu = {"value": rate, "unit": UNIT, "cores": threads, "kind": "port",
               "sample": f"2 RK3 steps of the same 128x128x153 workload on the host, C restatement of the "
                         f"reference path (OpenMP, {threads} threads), {secs:.1f} s"}
    if rank == 0:
        line = {
            "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": K, "warmup": W,
            "ms_per_step": ms_max / K, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": "f64", "data": "synthetic", "config": config_dict(desc, world),
            "e2e": {"value": e2e_val, "unit": UNIT, "h2d_bytes_per_step": nbytes, "d2h_bytes_per_step": nbytes},
            "gpu_launches": launches_per_step * K,
            "tuned": tuned,
            "roofline": {"bound": "hbm", "kernel": "one RK3 substep (plane pass k_zinv/k_xprod/k_zfwd + column pass "
                                                  "k_column), the unit the 20 F algorithmic bytes are counted on",
                         "achieved": achieved, "peak": hbm, "peak_source": src, "unit": "GB/s",
                         "frac": achieved / hbm, "traffic": traffic_sub, "alg_bytes": alg,
                         "avg_duration_ms": sub_s * 1e3},
            "fp64": fp64,
            "kernels": kernels,
            "dominant_kernel": dom[0],
            "cpu_baseline": cpu,
            "plain_32x32x153": small,
            "batched": batched,
            "batched_uneven": uneven,
            "served": served,
            "clocks": clk.summary(),
        }
        print(json.dumps(line), flush=True)
    e.close()


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=30)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--no-cpu", action="store_true", help="skip the CPU-baseline sample")
    ap.add_argument("--no-serve", action="store_true", help="skip the batched and served measurements")
    ap.add_argument("--no-tune", action="store_true", help="default launch shapes instead of the autotuner's")
    ap.add_argument("--nx", type=int, default=128,
                    help="Fourier modes Nx = Nz of the plain workload (128: the headline configuration)")
    ap.add_argument("--serve-requests", type=int, default=30)
    ap.add_argument("--serve-full-steps", action="store_true",
                    help="served stream with the configuration's step counts log-U[200,5000] (default 20..200)")
    ap.add_argument("--serve-time-scale", type=float, default=0.05,
                    help="arrival times are replayed at this factor (<1: compressed)")
    args = ap.parse_args()
    args.warmup = max(args.warmup, 3)
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local_rank = int(os.environ.get("LOCAL_RANK", "0"))
    if world != args.gpus and world == 1 and args.gpus > 1:
        print(json.dumps({"error": "run N>1 under torchrun"}))
        sys.exit(2)
    if args.impl == "reference":
        run_reference(args, rank, world)
        return
    if world > 1:
        import datetime

        import torch
        import torch.distributed as tdist
        torch.cuda.set_device(local_rank)
        tdist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))
    try:
        run_ours(args, rank, world, local_rank)
    finally:
        if world > 1:
            import torch.distributed as tdist
            tdist.destroy_process_group()


if __name__ == "__main__":
    main()
