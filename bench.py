"""Benchmark: solves/s of the FFT-accelerated dipole solve on one B200.

Workload (one step = one complete rigorous solve):
  inhomogeneous cube 64x64x64 (262,144 dipoles), d = 10 nm, lambda 632.8 nm,
  permittivity from the seeded Gaussian random field (mean 2.25, std 0.1,
  lc = 50 nm, SUNIF seed 4*7+1), plane wave theta = 20 deg p-polarised, RR
  polarisability, FFT grid 128^3, GPBICG1 to true residual 1e-4, solved with
  the FP32 mat-vec / inner Krylov inside FP64 iterative refinement
  (headline `value`), next to the plain FP64 drop-in (`fp64` block).
Inputs (FF0, polarisability) are resident in HBM for `value`; `e2e` runs the
same solve through the C-ABI (ifdda_inverserig) with pinned host buffers and
the host<->device copies inside the timed region.  L2 is flushed (256 MiB
write) before every timed step.  `--impl reference` times the CPU
restatement of the reference path (oracle, all host threads) on the same
workload.  With torchrun, every rank solves its own copy (replicas, weak
scaling); times are the max over ranks.
"""
import argparse
import json
import math
import os
import statistics
import subprocess
import sys
import threading
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(ROOT, "if-dda_b200"))

import numpy as np  # noqa: E402

METRIC = "solves/s & p99 latency, mixed vs FP64 at rel. residual 1e-4; matvec HBM GB/s"
WORKLOAD = ("C2 inhomogeneous GRF cube 64^3 (262,144 dipoles), d=10 nm, lambda=632.8 nm, "
            "theta=20 deg p-pol, RR, GPBICG1 to true residual 1e-4, FFT grid 128^3")
LAMBDA = 632.8e-9
N_EDGE = 64
TOL = 1e-4


def build_object():
    from ifdda import objects
    k0 = 2 * math.pi / LAMBDA
    ob = objects.inhomocuboid(N_EDGE, N_EDGE, N_EDGE, 10e-9, 2.25 + 0j, 50e-9, 0.1, 7, k0, "RR")
    E0, _ = objects.irradiance(1.0, 10 * LAMBDA)
    return ob, k0, E0


def measured_peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        d = json.load(open(p))
        return float(d["hbm_gbs"]), "MEASURED_PEAKS.json hbm_gbs (copy, burst)"
    return 6650.0, "fallback 6.65 TB/s"


def profile_traffic():
    """dram bytes per zconv launch from the committed ncu summary, if any."""
    p = os.path.join(ROOT, "profiles", "zconv_c2_fp32.md")
    if not os.path.exists(p):
        return None
    for line in open(p):
        if line.startswith("traffic_bytes_per_launch:"):
            try:
                return float(line.split(":", 1)[1])
            except ValueError:
                return None
    return None


class ClockSampler:
    """nvidia-smi samples (every 100 ms) during the timed region."""

    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index):
        self.gpu = gpu_index
        self.proc = None
        self.lines = []

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", f"--query-gpu={self.Q}", "--format=csv,noheader,nounits",
                                          "-lms", "100", "-i", str(self.gpu)], stdout=subprocess.PIPE,
                                         stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except OSError:
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def __exit__(self, *a):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()

    def summary(self):
        sm, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            f = [x.strip() for x in ln.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                mx = float(f[2])
            except ValueError:
                continue
            for nm, v in zip(names, f[5:9]):
                if v.lower().startswith("active"):
                    reasons.add(nm)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": mx, "reasons": sorted(reasons),
                "samples": len(sm)}


def dist_setup():
    ws = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return ws, rank, local


def max_over_ranks(v, ws, device=None):
    if ws == 1:
        return v
    import torch
    import torch.distributed as dist
    t = torch.tensor([v], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def barrier(ws):
    if ws > 1:
        import torch.distributed as dist
        dist.barrier()


# ----------------------------------------------------------------- CPU arm --
def cpu_oracle_sample(ob, k0, E0, ncompte_full, n_mv=4):
    """Times the oracle (C restatement of the reference path, FP64, OpenMP on
    every host thread): the Green spectrum once, then GPBICG1 stopped after
    n_mv mat-vecs; a full solve is extrapolated with the solve's mat-vec
    count.  Returns (solves/s, seconds sampled, cores, sample string)."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle
    cores = os.cpu_count() or 1
    oracle.set_threads(cores)
    n = ob.nx
    t0 = time.perf_counter()
    G = oracle.greencalculfft(n, n, n, ob.aretecube, k0)
    t_green = time.perf_counter() - t0
    ff0 = oracle.incident(ob.xs, ob.ys, ob.zs, k0, E0, 1.0, 0, 20.0, 0.0)
    t0 = time.perf_counter()
    oracle.inverserig(G, n, n, n, ob.nbsphere, ob.polarisa, ob.nmax, ff0, "GPBICG1", TOL, max_matvecs=n_mv)
    t_mv = (time.perf_counter() - t0) / n_mv
    t_solve = t_green + t_mv * ncompte_full
    sample = (f"oracle FP64 on {cores} host threads: greencalculfft 128^3 ({t_green:.2f} s) + GPBICG1 stopped "
              f"after {n_mv} mat-vecs ({t_mv:.3f} s/mat-vec incl. Krylov vector work); full solve "
              f"extrapolated to ncompte={ncompte_full} mat-vecs = {t_solve:.1f} s")
    return 1.0 / t_solve, t_green + t_mv * n_mv, cores, sample


def run_reference(args):
    ws, rank, _ = dist_setup()
    if rank != 0:
        return 0
    ob, k0, E0 = build_object()
    # GPBICG1 on this workload needs 34 mat-vecs (16 iterations) in FP64, the
    # same count for the oracle and the GPU drop-in
    ncompte = 34
    vals = []
    for i in range(args.warmup + args.steps):
        v, secs, cores, sample = cpu_oracle_sample(ob, k0, E0, ncompte, n_mv=2)
        if i >= args.warmup:
            vals.append(v)
    value = statistics.mean(vals)
    line = {"metric": METRIC, "value": value, "unit": "solves/s", "n_gpus": args.gpus, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": 1000.0 / value, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "c128", "data": "synthetic (seeded GRF, ng=7)", "impl": "reference",
            "config": {"workload": WORKLOAD, "precision": "fp64", "parallelism": "cpu"},
            "cpu_baseline": {"value": value, "unit": "solves/s", "cores": cores, "kind": "port", "sample": sample},
            "e2e": {"value": value, "unit": "solves/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)
    return 0


# ----------------------------------------------------------------- GPU arm --
def run_gpu(args):
    import torch
    import ctypes as C
    import ifdda
    from ifdda import IFDDA_FP64, IFDDA_MIXED, _capi

    ws, rank, local = dist_setup()
    torch.cuda.set_device(local)
    if ws > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))
    dev = torch.device("cuda", local)
    ob, k0, E0 = build_object()
    ctx = ifdda.Context(local)
    lib = ctx.lib
    stream = torch.cuda.ExternalStream(ctx.stream(), device=dev)
    t0 = time.perf_counter()
    g = ctx.green(ob.nx, ob.ny, ob.nz, ob.aretecube, k0)
    green_ms = (time.perf_counter() - t0) * 1e3
    ff0_h = ctx.planewaves(ob.xs, ob.ys, ob.zs, k0, E0, [0], [20.0], [0.0], [1.0])[0]
    nb, nmax = ob.nbsphere, ob.nmax
    pol_h = ob.polarisa
    ff0_d = torch.from_numpy(ff0_h).to(dev)
    pol_d = torch.from_numpy(pol_h).to(dev)
    ff_d = torch.empty_like(ff0_d)
    loc_d = torch.empty_like(ff0_d)
    flush = torch.empty(64 * 1024 * 1024, dtype=torch.float32, device=dev)  # 256 MiB > L2
    torch.cuda.synchronize()

    def solve_dev(prec):
        r = g.inverserig_device(1, nb, nmax, None, pol_d.data_ptr(), ff0_d.data_ptr(), ff_d.data_ptr(),
                                loc_d.data_ptr(), "GPBICG1", TOL, precision=prec)
        if r["nstop"] != 0:
            raise RuntimeError(f"solve failed: {r['infostr'].strip()}")
        return r

    def timed(prec, steps, warmup, count_launches=False):
        for _ in range(warmup):
            solve_dev(prec)
        torch.cuda.synchronize()
        barrier(ws)
        torch.cuda.synchronize()
        times, infos = [], []
        l0 = lib.ifdda_launch_count()
        for _ in range(steps):
            with torch.cuda.stream(stream):
                flush.zero_()
                e0 = torch.cuda.Event(enable_timing=True)
                e1 = torch.cuda.Event(enable_timing=True)
                e0.record(stream)
            infos.append(solve_dev(prec))
            with torch.cuda.stream(stream):
                e1.record(stream)
            e1.synchronize()
            times.append(e0.elapsed_time(e1))
        launches = lib.ifdda_launch_count() - l0
        torch.cuda.synchronize()
        barrier(ws)
        return times, infos, launches

    # headline: mixed precision, iterations replayed as CUDA graphs
    with ClockSampler(local) as clk:
        t_mixed, info_mixed, launches = timed(IFDDA_MIXED, args.steps, args.warmup)
    # the dominant kernel (zconv, FP32) bracketed by CUDA events on the
    # solver's stream during further complete solves (plain launches)
    lib.ifdda_timing_enable(_capi.PASS_ZCONV, _capi.IFDDA_FP32)
    timed(IFDDA_MIXED, max(3, min(args.steps, 10)), 0)
    nl, tot = C.c_int(0), C.c_double(0)
    lib.ifdda_timing_read(C.byref(nl), C.byref(tot))
    lib.ifdda_timing_enable(0, -1)
    zconv_ms = tot.value / max(nl.value, 1)

    fp64_steps = max(1, min(args.steps, 5))
    t_fp64, info_fp64, _ = timed(IFDDA_FP64, fp64_steps, min(args.warmup, 3))

    total_ms = max_over_ranks(sum(t_mixed), ws, dev)
    value = ws * args.steps / (total_ms / 1e3)
    fp64_total = max_over_ranks(sum(t_fp64), ws, dev)
    fp64_value = ws * fp64_steps / (fp64_total / 1e3)

    # mat-vec throughput (whole mat-vec, algorithmic bytes) at both precisions
    N = ob.nx * ob.ny * ob.nz
    Np = (ob.nx + 1) * (ob.ny + 1) * (ob.nz + 1)
    M = 8 * N
    mv = {}
    for prec, dt, s in ((2, torch.complex64, 8), (0, torch.complex128, 16)):
        x = torch.randn(3 * N, dtype=dt, device=dev)
        b = torch.randn(3 * N, dtype=dt, device=dev)
        for _ in range(3):
            g.matvec_device(1, N, x.data_ptr(), b.data_ptr(), precision=prec)
        ctx.synchronize()
        reps = 20
        with torch.cuda.stream(stream):
            e0 = torch.cuda.Event(enable_timing=True)
            e1 = torch.cuda.Event(enable_timing=True)
            e0.record(stream)
        for _ in range(reps):
            g.matvec_device(1, N, x.data_ptr(), b.data_ptr(), precision=prec)
        with torch.cuda.stream(stream):
            e1.record(stream)
        e1.synchronize()
        ms = e0.elapsed_time(e1) / reps
        balg = s * (7 * N + 6 * Np + 6 * M)
        mv["fp32" if prec == 2 else "fp64"] = {"ms": round(ms, 4), "alg_bytes": balg,
                                                "GB_s": round(balg / ms / 1e6, 1)}

    # end to end through the C-ABI with pinned host buffers
    ff0_pin = torch.from_numpy(ff0_h).pin_memory()
    pol_pin = torch.from_numpy(pol_h).pin_memory()
    e2e_steps = max(1, min(args.steps, 5))
    g.inverserig(nb, pol_pin.numpy(), nmax, ff0_pin.numpy(), "GPBICG1", TOL, precision=IFDDA_MIXED)
    barrier(ws)
    te = []
    for _ in range(e2e_steps):
        t0 = time.perf_counter()
        r = g.inverserig(nb, pol_pin.numpy(), nmax, ff0_pin.numpy(), "GPBICG1", TOL, precision=IFDDA_MIXED)
        te.append(time.perf_counter() - t0)
        if r.nstop != 0:
            raise RuntimeError(r.infostr)
    e2e_total = max_over_ranks(sum(te), ws, dev)
    e2e_value = ws * e2e_steps / e2e_total
    h2d = ff0_h.nbytes + nb * 16  # FF0 + the compact isotropic polarisability
    d2h = 2 * ff0_h.nbytes        # FF and FFloc

    peak, peak_src = measured_peaks()
    zc_bytes = 8 * (2 * 3 * ob.nz * (2 * ob.ny) * (2 * ob.nx) + 6 * Np)
    achieved = zc_bytes / (zconv_ms * 1e6) if zconv_ms > 0 else None
    traffic = profile_traffic()
    cpu = None
    if rank == 0 and ws == 1 and not args.no_cpu:
        ncompte64 = int(info_fp64[0]["ncompte"][0])
        v, secs, cores, sample = cpu_oracle_sample(ob, k0, E0, ncompte64)
        cpu = {"value": v, "unit": "solves/s", "cores": cores, "kind": "port", "sample": sample}

    lat = sorted(t_mixed)
    p50 = statistics.median(lat)
    p99 = lat[min(len(lat) - 1, int(math.ceil(0.99 * len(lat))) - 1)]
    im = info_mixed[-1]
    i64 = info_fp64[-1]
    line = {
        "metric": METRIC, "value": value, "unit": "solves/s", "n_gpus": ws, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": total_ms / args.steps, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "c64 inner / c128 outer", "data": "synthetic (seeded GRF, ng=7)",
        "config": {"workload": WORKLOAD, "precision": "mixed FP32/FP64 refinement", "l2": "flushed before each step",
                   "parallelism": f"replicas x{ws}" if ws > 1 else "single GPU"},
        "latency_ms": {"p50": p50, "p99": p99},
        "mixed": {"solves_s": value, "nloop": int(im["nloop"][0]), "ncompte": int(im["ncompte"][0]),
                  "tol1": float(im["tol1"][0])},
        "fp64": {"solves_s": fp64_value, "ms_per_solve": fp64_total / fp64_steps, "nloop": int(i64["nloop"][0]),
                 "ncompte": int(i64["ncompte"][0]), "tol1": float(i64["tol1"][0])},
        "matvec": mv,
        "green_build_ms": green_ms,
        "roofline": {"bound": "hbm", "kernel": "k_zconv<float,128> (z FFT + 3x3 spectrum multiply + inverse z FFT)",
                     "achieved": achieved, "peak": peak, "unit": "GB/s",
                     "frac": (achieved / peak) if achieved else None, "traffic": traffic,
                     "alg_bytes_per_launch": zc_bytes, "avg_launch_ms": zconv_ms, "launches_timed": nl.value,
                     "peak_source": peak_src},
        "cpu_baseline": cpu,
        "e2e": {"value": e2e_value, "unit": "solves/s", "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": d2h},
        "gpu_launches": int(launches),
        "clocks": clk.summary(),
    }
    if rank == 0:
        print(json.dumps(line), flush=True)
    g.close()
    ctx.close()
    if ws > 1:
        import torch.distributed as dist
        dist.destroy_process_group()
    return 0


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=60)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ifdda", choices=["ifdda", "reference"])
    ap.add_argument("--no-cpu", action="store_true", help="skip the CPU oracle sample")
    args = ap.parse_args()
    if args.impl == "reference":
        return run_reference(args)
    return run_gpu(args)


if __name__ == "__main__":
    sys.exit(main())
