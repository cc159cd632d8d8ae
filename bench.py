"""Benchmark: solves/s of the FFT-accelerated dipole solve on one B200.

Default workload (one step = one complete rigorous solve of the inhomogeneous cube):
  inhomogeneous cube 64x64x64 (262,144 dipoles), d = 10 nm, lambda 632.8 nm,
  permittivity from the seeded Gaussian random field (mean 2.25, std 0.1,
  lc = 50 nm, SUNIF seed 4*7+1), plane wave theta = 20 deg p-polarised, RR
  polarisability, FFT grid 128^3, GPBICG1 to true residual 1e-4, solved with
  the FP32 mat-vec / inner Krylov inside FP64 iterative refinement
  (headline `value`), next to the plain FP64 drop-in (`fp64` block).
Other workloads (--workload): c1 (sphere 16^3, inside-only dipoles), c3
(128 plane waves on a 96x96x64 ellipsoid lattice, one batched solve per
step), c5 (192^3 concentric spheres, GPBICG1), c4 (request stream
through the continuous-batching server), mic (bright-field microscope image
of the c3 object: every illumination of the condenser solved in batches, FFT
lens, 512^2 image; one step = one image).
Inputs are resident in HBM for `value`; `e2e` runs the same solve through the
C-ABI (ifdda_inverserig) with pinned host inputs and the host<->device copies
inside the timed region.  L2 is flushed (256 MiB write) before every timed
step.  `--impl reference` times the CPU restatement of the reference path
(oracle, all host threads) on the same workload.  With torchrun, every rank
solves its own copy (replicas, weak scaling); times are the max over ranks.
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
from dataclasses import dataclass, field

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(ROOT, "if-dda_b200"))

import numpy as np  # noqa: E402

METRIC = "solves/s & p99 latency, mixed vs FP64 at rel. residual 1e-4; matvec HBM GB/s"
TOL = 1e-4


# ----------------------------------------------------------------- workloads --
@dataclass
class Workload:
    key: str
    desc: str
    ob: object
    k0: float
    E0: float
    beams: list            # [(beam, a1, a2, pp)] one per right-hand side
    method: str
    fp64_nrhs: int         # right-hand sides solved for the FP64 comparison
    cpu_mv: int = 4        # oracle mat-vecs timed for the CPU baseline
    extra: dict = field(default_factory=dict)

    @property
    def nrhs(self):
        return len(self.beams)


def wl_c1():
    from ifdda import objects
    lam = 632.8e-9
    k0 = 2 * math.pi / lam
    ob = objects.sphere(100e-9, 2.25 + 0j, 16, k0, "RR", na=-1)
    E0, _ = objects.irradiance(1.0, 10 * lam)
    return Workload("c1", "C1 sphere eps 2.25, R=100 nm, 16^3 lattice, 2176 dipoles inside, lambda=632.8 nm, "
                    "normal incidence x-pol, RR, GPBICG1 to 1e-4, FFT grid 32^3", ob, k0, E0,
                    [(0, 0.0, 0.0, 1.0)], "GPBICG1", 1)


def wl_c2():
    from ifdda import objects
    lam = 632.8e-9
    k0 = 2 * math.pi / lam
    ob = objects.inhomocuboid(64, 64, 64, 10e-9, 2.25 + 0j, 50e-9, 0.1, 7, k0, "RR")
    E0, _ = objects.irradiance(1.0, 10 * lam)
    return Workload("c2", "C2 inhomogeneous GRF cube 64^3 (262,144 dipoles), d=10 nm, lambda=632.8 nm, "
                    "theta=20 deg p-pol, RR, GPBICG1 to true residual 1e-4, FFT grid 128^3", ob, k0, E0,
                    [(0, 20.0, 0.0, 1.0)], "GPBICG1", 1)


def wl_c3(nrhs_pairs=64):
    from ifdda import objects
    lam = 500e-9
    k0 = 2 * math.pi / lam
    ob = objects.ellipsoid_lattice(96, 96, 64, 10e-9, 400e-9, 300e-9, 200e-9, 2.0, 2.6, 33, k0, "RR")
    E0, _ = objects.irradiance(1.0, 10 * lam)
    rng = np.random.Generator(np.random.PCG64(3))
    r = 0.9 * k0 * np.sqrt(rng.uniform(0, 1, nrhs_pairs))
    t = rng.uniform(0, 2 * np.pi, nrhs_pairs)
    beams = []
    for kx, ky in zip(r * np.cos(t), r * np.sin(t)):
        beams.append((1, float(kx), float(ky), 0.0))  # s
        beams.append((1, float(kx), float(ky), 1.0))  # p
    return Workload("c3", f"C3 batched brightfield sweep: ellipsoid 400/300/200 nm on a 96x96x64 lattice, d=10 nm, "
                    f"eps U[2.0,2.6] (seed 33), lambda=500 nm, {len(beams)} plane waves ({nrhs_pairs} (kx,ky) on the "
                    f"NA 0.9 disk, seed 3, x s/p) in one batched solve, GPBICG1 to 1e-4, FFT grid 192x192x128",
                    ob, k0, E0, beams, "GPBICG1", 8, cpu_mv=2)


def wl_c5():
    from ifdda import objects
    lam = 632.8e-9
    k0 = 2 * math.pi / lam
    ob = objects.concentric([0.9e-6, 1.9e-6], [3.0 + 0.01j, 2.0 + 0j], 192, k0, "RR", na=0)
    E0, _ = objects.irradiance(1.0, 10 * lam)
    return Workload("c5", "C5 concentric spheres (core eps 3+0.01i r=0.9 um, shell eps 2 r=1.9 um) on the full "
                    "192^3 lattice (7.08M dipoles, d = 2 r_out/192 = 19.79 nm as the reference sizes it), "
                    "lambda=632.8 nm, normal incidence, GPBICG1 to 1e-4 (QMR-BiCGSTAB, the configured method, does "
                    "not converge on this object: QMRBICGSTAB2 stands at true residual 4.2e-2 after 3000 FP64 "
                    "iterations, QMRBICGSTAB1 breaks down), FFT grid 384^3",
                    ob, k0, E0, [(0, 0.0, 0.0, 1.0)], "GPBICG1", 1, cpu_mv=1)


WORKLOADS = {"c1": wl_c1, "c2": wl_c2, "c3": wl_c3, "c5": wl_c5}


# ------------------------------------------------------------------ helpers --
def measured_peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        d = json.load(open(p))
        return float(d["hbm_gbs"]), "MEASURED_PEAKS.json hbm_gbs (copy, burst)"
    return 6650.0, "fallback 6.65 TB/s"


def profile_traffic(key):
    """dram bytes per zconv launch from the committed ncu summary, if any."""
    p = os.path.join(ROOT, "profiles", f"zconv_{key}_fp32.md")
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
def cpu_oracle_solves(w: Workload, max_solves: int, budget_s: float):
    """Times the oracle (C restatement of the reference path, FP64, OpenMP on
    every host thread) doing what one cdmlib call does for one right-hand
    side of the workload: greencalculfft, then the complete solve
    (inverserig / inverserigopt with the workload's method) to TOL.  Runs
    whole solves, at least one, until max_solves or budget_s seconds.
    Returns (seconds per solve list, cores, info of the last solve)."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle
    cores = os.cpu_count() or 1
    oracle.set_threads(cores)
    ob = w.ob
    times, info = [], None
    t_all = time.perf_counter()
    for i in range(max_solves):
        bm, a1, a2, pp = w.beams[i % len(w.beams)]
        ff0 = oracle.incident(ob.xs, ob.ys, ob.zs, w.k0, w.E0, pp, bm, a1, a2)
        t0 = time.perf_counter()
        G = oracle.greencalculfft(ob.nx, ob.ny, ob.nz, ob.aretecube, w.k0)
        t_green = time.perf_counter() - t0
        r = oracle.inverserig(G, ob.nx, ob.ny, ob.nz, ob.nbsphere, ob.polarisa, ob.nmax, ff0, w.method, TOL,
                              tabdip=ob.tabdip_or_none)
        times.append(time.perf_counter() - t0)
        del G
        info = {"green_s": t_green, "ncompte": int(r["ncompte"]), "nloop": int(r["nloop"]),
                "tol1": float(r["tol1"]), "nstop": int(r["nstop"])}
        if time.perf_counter() - t_all > budget_s:
            break
    return times, cores, info


def cpu_sample_text(w, times, cores, info):
    return (f"oracle FP64 on {cores} host threads: {len(times)} complete solve(s) of one right-hand side of "
            f"{w.key}, each greencalculfft ({info['green_s']:.2f} s) + {w.method} to true residual {TOL:g} "
            f"(nloop {info['nloop']}, ncompte {info['ncompte']}, tol1 {info['tol1']:.2e}); "
            f"{statistics.mean(times):.2f} s per solve")


def run_reference(args):
    """The reference arm: the CPU restatement of cdmlib's rigorous path timed
    as whole solves (greencalculfft + the complete Krylov solve), one
    right-hand side per step.  A full solve takes seconds, so the run is
    bounded: one untimed warm-up solve, then timed solves until --steps or
    about 150 s; the line's `steps` is the number actually timed."""
    ws, rank, _ = dist_setup()
    if rank != 0:
        return 0
    w = WORKLOADS[args.workload]()
    if args.warmup > 0:
        cpu_oracle_solves(w, 1, 0.0)
    times, cores, info = cpu_oracle_solves(w, max(1, args.steps), 150.0)
    value = len(times) / sum(times)
    sample = cpu_sample_text(w, times, cores, info)
    line = {"metric": METRIC, "value": value, "unit": "solves/s", "n_gpus": args.gpus, "steps": len(times),
            "steps_requested": args.steps, "warmup": min(args.warmup, 1), "ms_per_step": 1000.0 / value,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "c128",
            "data": "synthetic (seeded)", "impl": "reference",
            "config": {"workload": w.desc, "precision": "fp64", "parallelism": "cpu",
                       "step": "greencalculfft + complete solve of one right-hand side"},
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
    w = WORKLOADS[args.workload]()
    ob, k0, E0 = w.ob, w.k0, w.E0
    ctx = ifdda.Context(local)
    lib = ctx.lib
    stream = torch.cuda.ExternalStream(ctx.stream(), device=dev)
    t0 = time.perf_counter()
    g = ctx.green(ob.nx, ob.ny, ob.nz, ob.aretecube, k0)
    green_ms = (time.perf_counter() - t0) * 1e3  # first build: allocation and twiddle tables included
    ff0_h = ctx.planewaves(ob.xs, ob.ys, ob.zs, k0, E0, [b[0] for b in w.beams], [b[1] for b in w.beams],
                           [b[2] for b in w.beams], [b[3] for b in w.beams])
    nb, nmax, nrhs = ob.nbsphere, ob.nmax, w.nrhs
    pol_h = ob.polarisa
    ff0_d = torch.from_numpy(ff0_h).to(dev)
    pol_d = torch.from_numpy(pol_h).to(dev)
    tab_d = torch.from_numpy(ob.tabdip).to(dev) if ob.inside_only else None
    ff_d = torch.empty_like(ff0_d)
    loc_d = torch.empty_like(ff0_d)
    flush = torch.empty(64 * 1024 * 1024, dtype=torch.float32, device=dev)  # 256 MiB > L2
    torch.cuda.synchronize()

    def solve_dev(prec, k=nrhs):
        r = g.inverserig_device(k, nb, nmax, tab_d.data_ptr() if tab_d is not None else None, pol_d.data_ptr(),
                                ff0_d.data_ptr(), ff_d.data_ptr(), loc_d.data_ptr(), w.method, TOL, precision=prec)
        if r["nstop"] != 0:
            raise RuntimeError(f"solve failed: {r['infostr'].strip()}")
        return r

    def timed(prec, steps, warmup, k=nrhs, green=False):
        """steps complete solves; with green, each step first recomputes the
        spectrum in place (greencalculfft, which cdmlib runs on every call)."""
        for _ in range(warmup):
            if green:
                g.recompute(ob.aretecube, k0)
            solve_dev(prec, k)
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
            if green:
                g.recompute(ob.aretecube, k0)
            infos.append(solve_dev(prec, k))
            with torch.cuda.stream(stream):
                e1.record(stream)
            e1.synchronize()
            times.append(e0.elapsed_time(e1))
        launches = lib.ifdda_launch_count() - l0
        torch.cuda.synchronize()
        barrier(ws)
        return times, infos, launches

    # headline: mixed precision, iterations replayed as CUDA graphs; a step
    # is one object: its Green spectrum (recomputed in place, as cdmlib
    # calls greencalculfft on every run) and the solve of its right-hand sides
    with ClockSampler(local) as clk:
        t_mixed, info_mixed, launches = timed(IFDDA_MIXED, args.steps, args.warmup, green=True)
    # the same solves with the spectrum resident (a cached spectrum)
    t_mixed_solve, _, _ = timed(IFDDA_MIXED, args.steps, 1)
    # the dominant kernel (zconv, FP32) bracketed by CUDA events on the
    # solver's stream during further complete solves (plain launches)
    lib.ifdda_timing_enable(_capi.PASS_ZCONV, _capi.IFDDA_FP32)
    timed(IFDDA_MIXED, max(1, min(args.steps, 5)), 0)
    nl, tot = C.c_int(0), C.c_double(0)
    lib.ifdda_timing_read(C.byref(nl), C.byref(tot))
    lib.ifdda_timing_enable(0, -1)
    zconv_ms = tot.value / max(nl.value, 1)
    g.release_workspace()
    kacc = w.fp64_nrhs
    loc_mixed, ff_mixed = loc_d[:kacc].cpu().numpy(), ff_d[:kacc].cpu().numpy()

    fp64_steps = max(1, min(args.steps, 5))
    t_fp64, info_fp64, _ = timed(IFDDA_FP64, fp64_steps, min(args.warmup, 2), k=w.fp64_nrhs, green=True)
    loc64, ff64 = loc_d[:kacc].cpu().numpy(), ff_d[:kacc].cpu().numpy()
    t_fp64_solve, _, _ = timed(IFDDA_FP64, fp64_steps, 0, k=w.fp64_nrhs)
    # the plain FP64 drop-in called once per right-hand side, as the
    # reference's incidence loop calls inverserig (microsbf.f:214-280)
    # the plain FP64 drop-in called once per right-hand side, as the
    # reference's incidence loop calls inverserig (microsbf.f:214-280), at
    # the bench tolerance and at a fifth of it (its local-field error is
    # compared with the converged field below)
    bytes_rhs = 3 * nb * 16
    nser = w.fp64_nrhs
    serial = {}

    def serial_pass(tol):
        ts, locs = [], []
        for r in range(nser):
            with torch.cuda.stream(stream):
                e0 = torch.cuda.Event(enable_timing=True)
                e1 = torch.cuda.Event(enable_timing=True)
                e0.record(stream)
            rr = g.inverserig_device(1, nb, nmax, tab_d.data_ptr() if tab_d is not None else None,
                                     pol_d.data_ptr(), ff0_d.data_ptr() + r * bytes_rhs,
                                     ff_d.data_ptr() + r * bytes_rhs, loc_d.data_ptr() + r * bytes_rhs, w.method,
                                     tol, precision=IFDDA_FP64)
            if rr["nstop"] != 0:
                raise RuntimeError(rr["infostr"].strip())
            with torch.cuda.stream(stream):
                e1.record(stream)
            e1.synchronize()
            ts.append(e0.elapsed_time(e1))
            locs.append(loc_d[r].cpu().numpy())
        return ts, locs
    for tol_s in (TOL, TOL / 5):
        serial_pass(tol_s)
        ts, locs = serial_pass(tol_s)
        serial[f"tol_{tol_s:g}"] = {"solves_s": nser / (sum(ts) / 1e3), "rhs": nser, "ms_per_solve": statistics.mean(ts),
                                    "_locs": locs}
    # accuracy against a converged FP64 solve (true residual 1e-10; the FP64
    # drop-in is the path the parity tests hold to the oracle): local field
    # and Cext of the mixed solve, and of the FP64 solve stopped at TOL
    rc = g.inverserig_device(kacc, nb, nmax, tab_d.data_ptr() if tab_d is not None else None, pol_d.data_ptr(),
                             ff0_d.data_ptr(), ff_d.data_ptr(), loc_d.data_ptr(), w.method, 1e-10,
                             precision=IFDDA_FP64)
    if rc["nstop"] != 0:
        raise RuntimeError(f"converged solve failed: {rc['infostr'].strip()}")
    locc, ffc = loc_d[:kacc].cpu().numpy(), ff_d[:kacc].cpu().numpy()
    g.release_workspace()
    acc = {"reference": "FP64 drop-in solved to true residual 1e-10", "rhs_compared": kacc,
           "converged_tol1_max": float(np.max(rc["tol1"]))}
    for name, loc, ff in (("mixed", loc_mixed, ff_mixed), ("fp64", loc64, ff64)):
        el, ec = 0.0, 0.0
        for r in range(kacc):
            el = max(el, float(np.linalg.norm(loc[r] - locc[r]) / np.linalg.norm(locc[r])))
            cm, _ = ctx.cross_sections(ff0_h[r], ff[r], loc[r], k0, abs(E0) ** 2)
            cc, _ = ctx.cross_sections(ff0_h[r], ffc[r], locc[r], k0, abs(E0) ** 2)
            ec = max(ec, abs(cm - cc) / abs(cc))
        acc[f"local_field_rel_l2_{name}"] = el
        acc[f"cext_rel_diff_{name}"] = ec
    for key, blk in serial.items():
        locs = blk.pop("_locs")
        blk["local_field_rel_l2"] = max(float(np.linalg.norm(locs[r] - locc[r]) / np.linalg.norm(locc[r]))
                                        for r in range(min(nser, kacc)))
    # the precision comparison: the mixed batched solver against the FP64
    # drop-in one right-hand side per call, at matching accuracy (the loosest
    # tolerance whose local field is as close to the converged field as the
    # mixed solve's, or within 1e-4 of it)
    bar = max(1e-4, acc["local_field_rel_l2_mixed"])
    match = next((k for k in serial if serial[k]["local_field_rel_l2"] <= bar), None)

    total_ms = max_over_ranks(sum(t_mixed), ws, dev)
    value = ws * args.steps * nrhs / (total_ms / 1e3)
    solve_only = ws * args.steps * nrhs / (max_over_ranks(sum(t_mixed_solve), ws, dev) / 1e3)
    fp64_total = max_over_ranks(sum(t_fp64), ws, dev)
    fp64_value = ws * fp64_steps * w.fp64_nrhs / (fp64_total / 1e3)
    fp64_solve_only = ws * fp64_steps * w.fp64_nrhs / (max_over_ranks(sum(t_fp64_solve), ws, dev) / 1e3)

    # mat-vec throughput (whole mat-vec, algorithmic bytes, one right-hand side)
    N = ob.nx * ob.ny * ob.nz
    Np = (ob.nx + 1) * (ob.ny + 1) * (ob.nz + 1)
    M = 8 * N
    mv = {}
    pk, _ = measured_peaks()
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
        # the unpruned algorithm's bytes (x, alpha, y; the full 6-component
        # spectrum; the padded 3-component field written and read once)
        bdense = s * (7 * N + 12 * M)
        mv["fp32" if prec == 2 else "fp64"] = {"ms": round(ms, 4), "alg_bytes": balg,
                                                "GB_s": round(balg / ms / 1e6, 1),
                                                "frac": round(balg / ms / 1e6 / pk, 3),
                                                "alg_bytes_unpruned": bdense,
                                                "GB_s_unpruned": round(bdense / ms / 1e6, 1),
                                                "frac_unpruned": round(bdense / ms / 1e6 / pk, 3)}
        del x, b
    g.release_workspace()

    # end to end through the C-ABI with pinned host inputs
    e2e_value, h2d, d2h = None, 0, 0
    if not args.no_e2e:
        ff0_pin = torch.from_numpy(ff0_h).pin_memory()
        pol_pin = torch.from_numpy(pol_h).pin_memory()
        # the fields come back into pinned arrays allocated once, as the
        # reference's FF / FFloc arrays are
        out_pin = (torch.empty(ff0_h.shape, dtype=torch.complex128).pin_memory().numpy(),
                   torch.empty(ff0_h.shape, dtype=torch.complex128).pin_memory().numpy())
        e2e_steps = max(1, min(args.steps, 20, int(10000.0 / max(total_ms / args.steps, 1.0))))  # ~10 s at most
        tab_h = ob.tabdip_or_none
        g.recompute(ob.aretecube, k0)
        g.inverserig(nb, pol_pin.numpy(), nmax, ff0_pin.numpy(), w.method, TOL, tabdip=tab_h, precision=IFDDA_MIXED,
                     out=out_pin)
        barrier(ws)
        te = []
        for _ in range(e2e_steps):
            t0 = time.perf_counter()
            # what one cdmlib call does on the path: greencalculfft, then the solve
            g.recompute(ob.aretecube, k0)
            r = g.inverserig(nb, pol_pin.numpy(), nmax, ff0_pin.numpy(), w.method, TOL, tabdip=tab_h,
                             precision=IFDDA_MIXED, out=out_pin)
            te.append(time.perf_counter() - t0)
            if r.nstop != 0:
                raise RuntimeError(r.infostr)
        e2e_total = max_over_ranks(sum(te), ws, dev)
        e2e_value = ws * e2e_steps * nrhs / e2e_total
        h2d = ff0_h.nbytes + nb * 16 + (ob.tabdip.nbytes if ob.inside_only else 0)  # FF0, compact alpha, Tabdip
        d2h = 2 * ff0_h.nbytes  # FF and FFloc
        g.release_workspace()

    peak, peak_src = measured_peaks()
    Z, Y, X = 2 * ob.nz, 2 * ob.ny, 2 * ob.nx
    zc_bytes = 8 * (2 * 3 * ob.nz * Y * X * nrhs + 6 * Np)
    achieved = zc_bytes / (zconv_ms * 1e6) if zconv_ms > 0 else None
    cpu = None
    if rank == 0 and ws == 1 and not args.no_cpu:
        times, cores, info = cpu_oracle_solves(w, 1, 0.0)
        cpu = {"value": len(times) / sum(times), "unit": "solves/s", "cores": cores, "kind": "port",
               "sample": cpu_sample_text(w, times, cores, info)}

    lat = sorted(t_mixed)
    p50 = statistics.median(lat)
    p99 = lat[min(len(lat) - 1, int(math.ceil(0.99 * len(lat))) - 1)]
    im = info_mixed[-1]
    i64 = info_fp64[-1]
    line = {
        "metric": METRIC, "value": value, "unit": "solves/s", "n_gpus": ws, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": total_ms / args.steps, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "c64 inner / c128 outer", "data": "synthetic (seeded)",
        "config": {"workload": w.desc, "nrhs_per_step": nrhs, "precision": "mixed FP32/FP64 refinement",
                   "step": "Green spectrum recomputed in place (greencalculfft) + solve of the step's right-hand "
                           "sides, as one cdmlib call", "l2": "flushed before each step",
                   "parallelism": f"replicas x{ws}" if ws > 1 else "single GPU"},
        "latency_ms": {"p50": p50, "p99": p99},
        "mixed": {"solves_s": value, "solves_s_spectrum_resident": solve_only, "nloop_max": int(np.max(im["nloop"])),
                  "ncompte_max": int(np.max(im["ncompte"])), "tol1_max": float(np.max(im["tol1"]))},
        "fp64": {"solves_s": fp64_value, "solves_s_spectrum_resident": fp64_solve_only, "nrhs": w.fp64_nrhs,
                 "ms_per_step": fp64_total / fp64_steps, "nloop_max": int(np.max(i64["nloop"])),
                 "ncompte_max": int(np.max(i64["ncompte"])), "tol1_max": float(np.max(i64["tol1"]))},
        "accuracy": acc,
        "fp64_one_rhs_per_call": serial,
        "mixed_over_fp64_one_rhs_per_call": {
            "at_bench_tol": solve_only / serial[f"tol_{TOL:g}"]["solves_s"],
            "at_matching_accuracy": (solve_only / serial[match]["solves_s"]) if match else None,
            "fp64_tol_matching": match, "spectrum": "resident in both"},
        "matvec": mv,
        "tile_chooser": {name: dict(zip(("zconv_variant", "ypass_variant", "ms_z0_z1_y0_y1"), g.tiles(pr)))
                         for name, pr in (("fp32", _capi.IFDDA_FP32), ("fp64", _capi.IFDDA_FP64))},
        "green_build_ms": green_ms,
        "roofline": {"bound": "hbm", "kernel": f"k_zconv<float,{Z}> (z FFT + 3x3 spectrum multiply + inverse z FFT)",
                     "achieved": achieved, "peak": peak, "unit": "GB/s",
                     "frac": (achieved / peak) if achieved else None, "traffic": profile_traffic(w.key),
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


def run_matvec(args):
    """Mat-vec only: the five passes of --nrhs right-hand sides (one batched
    launch sequence) on the workload's grid, FP32 then FP64 (--precs), each
    pass timed with CUDA events on the solver stream (also the target of the
    ncu commands in profiles/)."""
    import ctypes as C
    import torch
    import ifdda
    from ifdda import _capi

    ws, rank, local = dist_setup()
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    w = WORKLOADS[args.workload]()
    ob = w.ob
    ctx = ifdda.Context(local)
    lib = ctx.lib
    g = ctx.green(ob.nx, ob.ny, ob.nz, ob.aretecube, w.k0)
    N = ob.nx * ob.ny * ob.nz
    Np = (ob.nx + 1) * (ob.ny + 1) * (ob.nz + 1)
    names = {1: "fwd_x", 2: "fwd_y", 3: "zconv", 4: "inv_y", 5: "inv_x"}
    out = {}
    R = args.nrhs
    for prec, dt, s in ((_capi.IFDDA_FP32, torch.complex64, 8), (_capi.IFDDA_FP64, torch.complex128, 16)):
        if str(prec) not in args.precs.split(","):
            continue
        x = torch.randn(R * 3 * N, dtype=dt, device=dev)
        b = torch.randn(R * 3 * N, dtype=dt, device=dev)
        for _ in range(args.warmup):
            g.matvec_device(R, N, x.data_ptr(), b.data_ptr(), precision=prec)
        ctx.synchronize()
        # per launch: every right-hand side's share, the spectrum once
        balg = {1: 9 * N * s * R, 2: 18 * N * s * R, 3: (24 * N * R + 6 * Np) * s, 4: 18 * N * s * R,
                5: 12 * N * s * R}
        passes = {}
        for ps in range(1, 6):
            lib.ifdda_timing_enable(ps, prec)
            for _ in range(args.steps):
                g.matvec_device(R, N, x.data_ptr(), b.data_ptr(), precision=prec)
            ctx.synchronize()
            nl, ms = C.c_int(0), C.c_double(0)
            lib.ifdda_timing_read(C.byref(nl), C.byref(ms))
            avg = ms.value / max(nl.value, 1)
            passes[names[ps]] = {"ms": round(avg, 5), "alg_GB_s": round(balg[ps] / avg / 1e6, 1)}
        # every zconv variant the tile chooser weighs, timed the same way
        zv, yv, tms = g.tiles(prec)
        zvar = {}
        for v in range(3):
            try:
                g.set_tiles(prec, v, yv)
            except ifdda.IfddaError:  # the grid's z length has fewer variants
                break
            lib.ifdda_timing_enable(3, prec)
            for _ in range(args.steps):
                g.matvec_device(R, N, x.data_ptr(), b.data_ptr(), precision=prec)
            ctx.synchronize()
            nl, ms = C.c_int(0), C.c_double(0)
            lib.ifdda_timing_read(C.byref(nl), C.byref(ms))
            zvar[v] = round(ms.value / max(nl.value, 1), 5)
        g.set_tiles(prec, zv, yv)
        lib.ifdda_timing_enable(0, -1)
        passes["tile_chooser"] = {"zconv_variant": zv, "ypass_variant": yv, "ms_z0_z1_y0_y1": tms,
                                  "zconv_ms_by_variant": zvar}
        out["fp32" if s == 8 else "fp64"] = passes
        del x, b
    if rank == 0:
        print(json.dumps({"mode": "matvec", "workload": w.desc, "nrhs": R, "passes": out}), flush=True)
    g.close()
    ctx.close()
    return 0


def run_solve_passes(args):
    """The five mat-vec passes inside complete solves of the workload's first
    right-hand side (mixed, then FP64): each pass's launches timed with CUDA
    events (the library then runs the solver loop without CUDA graphs, so the
    pass kernels carry their fused Krylov work as in the solve), next to the
    solve time with graphs.  Also the target of the per-iteration launch list
    in profiles/."""
    import ctypes as C
    import torch
    import ifdda
    from ifdda import IFDDA_FP32, IFDDA_FP64, IFDDA_MIXED

    ws, rank, local = dist_setup()
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    w = WORKLOADS[args.workload]()
    ob = w.ob
    ctx = ifdda.Context(local)
    lib = ctx.lib
    stream = torch.cuda.ExternalStream(ctx.stream(), device=dev)
    g = ctx.green(ob.nx, ob.ny, ob.nz, ob.aretecube, w.k0)
    bm, a1, a2, pp = w.beams[0]
    ff0 = ctx.planewaves(ob.xs, ob.ys, ob.zs, w.k0, w.E0, [bm], [a1], [a2], [pp])
    ff0_d = torch.from_numpy(ff0).to(dev)
    pol_d = torch.from_numpy(ob.polarisa).to(dev)
    tab_d = torch.from_numpy(ob.tabdip).to(dev) if ob.inside_only else None
    ff_d, loc_d = torch.empty_like(ff0_d), torch.empty_like(ff0_d)

    def solve(prec):
        r = g.inverserig_device(1, ob.nbsphere, ob.nmax, tab_d.data_ptr() if tab_d is not None else None,
                                pol_d.data_ptr(), ff0_d.data_ptr(), ff_d.data_ptr(), loc_d.data_ptr(), w.method, TOL,
                                precision=prec)
        if r["nstop"] != 0:
            raise RuntimeError(r["infostr"].strip())
        return r

    names = {1: "fwd_x", 2: "fwd_y", 3: "zconv", 4: "inv_y", 5: "inv_x"}
    out = {}
    for name, prec, pbits in (("mixed", IFDDA_MIXED, IFDDA_FP32), ("fp64", IFDDA_FP64, IFDDA_FP64)):
        for _ in range(args.warmup):
            solve(prec)
        ts = []
        for _ in range(args.steps):
            torch.cuda.synchronize()
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            r = solve(prec)
            e1.record(stream)
            e1.synchronize()
            ts.append(e0.elapsed_time(e1))
        res = {"ms_per_solve": statistics.median(ts), "nloop": int(r["nloop"][0]), "ncompte": int(r["ncompte"][0])}
        for ps in range(1, 6):
            lib.ifdda_timing_enable(ps, pbits)
            solve(prec)
            torch.cuda.synchronize()
            nl, ms = C.c_int(0), C.c_double(0)
            lib.ifdda_timing_read(C.byref(nl), C.byref(ms))
            res[names[ps]] = {"launches": nl.value, "us_per_launch": round(1e3 * ms.value / max(nl.value, 1), 2)}
        lib.ifdda_timing_enable(0, -1)
        out[name] = res
    if rank == 0:
        print(json.dumps({"mode": "passes", "workload": w.desc, "solve": out}), flush=True)
    g.close()
    ctx.close()
    return 0


def run_serving(args):
    """Config 4: a seeded request stream through the continuous-batching
    server, mixed precision then plain FP64 on the same stream."""
    import torch
    from ifdda import IFDDA_FP64, IFDDA_MIXED
    from ifdda import serve

    ws, rank, local = dist_setup()
    torch.cuda.set_device(local)
    reqs = serve.make_stream(args.requests, args.rate, seed=4)
    # page-locked read-back buffers for the largest local field of the
    # stream, one per slot, made before the timed stream
    serve.prewarm_readback(max(48 * r.n ** 3 * len(r.incidences) for r in reqs), args.slots)
    out = {}
    for name, prec in (("mixed", IFDDA_MIXED), ("fp64", IFDDA_FP64)):
        srv = serve.Server(slots=args.slots, device=local, precision=prec, ragged=args.ragged, policy=args.policy)
        # warm-up: one request per lattice size compiles nothing but fills caches
        srv.run(reqs[:args.slots], realtime=False, keep_fields=False)
        t0 = time.perf_counter()
        # every local field is read back to the host, then dropped
        res = srv.run(reqs, realtime=True, keep_fields=False)
        wall = time.perf_counter() - t0
        srv.close()
        out[name] = serve.latency_stats(res, wall)
        out[name]["wall_s"] = wall
    desc = (f"C4 serving stream: {args.requests} requests, Poisson arrivals at {args.rate}/s (seed 4), sphere or "
            f"cube, edge in {{16..96}}, d=10 nm, eps' U[1.5,4] eps'' U[0,0.5], lambda U[400,800] nm, 1-32 "
            f"incidences on the NA 0.9 disk, GPBICG1 to 1e-4, {args.slots} concurrent slots, HBM-budget admission"
            + (", ragged batches (every arrived request of the head's box in one solve)" if args.ragged else "")
            + (", least-work-first admission (5 s wait cap)" if args.policy == "sjf" else ", FIFO admission"))
    m = out["mixed"]
    line = {"metric": METRIC, "value": m["solves_per_s"], "unit": "solves/s", "n_gpus": 1, "steps": args.requests,
            "warmup": args.slots, "ms_per_step": m["wall_s"] * 1e3 / args.requests, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "c64 inner / c128 outer", "data": "synthetic (seeded)",
            "config": {"workload": desc, "parallelism": "single GPU"},
            "latency_ms": {"p50": m["p50_ms"], "p99": m["p99_ms"]}, "serving": out}
    if rank == 0:
        print(json.dumps(line), flush=True)
    return 0


def run_microscope(args):
    """Bright-field microscope (microsbf.f with the FFT lens) of the c3
    ellipsoid: one step = one complete image, every illumination solved.  The
    call is the C-ABI's ifdda_microscope with host inputs and the image read
    back, so the timed region is end to end; it is timed with CUDA events on
    the library's stream (the call returns after its last kernel)."""
    import torch
    import ifdda
    from ifdda import IFDDA_FP64, IFDDA_MIXED

    ws, rank, local = dist_setup()
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    w = wl_c3()
    ob, k0 = w.ob, w.k0
    lam = 2 * math.pi / k0
    mo = dict(ntypemic=1, nfft2d=512, numaper=0.9, numaperinc=0.5, gross=100.0, zlens=0.0, P0=1.0, w0=10 * lam)
    ctx = ifdda.Context(local)
    stream = torch.cuda.ExternalStream(ctx.stream(), device=dev)
    g = ctx.green(ob.nx, ob.ny, ob.nz, ob.aretecube, k0)
    lib = ctx.lib
    out = {}
    for name, prec in (("mixed", IFDDA_MIXED), ("fp64", IFDDA_FP64)):
        steps = args.steps if name == "mixed" else max(1, min(args.steps, 3))
        for _ in range(args.warmup if name == "mixed" else 1):
            r = g.microscope(ob.xs, ob.ys, ob.zs, ob.polarisa, w.method, TOL, precision=prec, **mo)
            if r.nstop != 0:
                raise RuntimeError(r.infostr.strip())
        times = []
        l0 = lib.ifdda_launch_count()
        with ClockSampler(local) as clk:
            for _ in range(steps):
                e0 = torch.cuda.Event(enable_timing=True)
                e1 = torch.cuda.Event(enable_timing=True)
                e0.record(stream)
                r = g.microscope(ob.xs, ob.ys, ob.zs, ob.polarisa, w.method, TOL, precision=prec, **mo)
                e1.record(stream)
                e1.synchronize()
                times.append(e0.elapsed_time(e1))
        launches = (lib.ifdda_launch_count() - l0) // steps
        ms = statistics.mean(times)
        out[name] = dict(images_per_s=1e3 / ms, ms_per_image=ms, illuminations=2 * len(r.kxinc),
                         last_ncompte=r.ncompte, launches_per_image=launches, clocks=clk.summary())
    m = out["mixed"]
    nill = m["illuminations"]
    cpu = None
    if not args.no_cpu and rank == 0:
        times, cores, info = cpu_oracle_solves(w, 1, 0.0)
        cpu = {"value": len(times) / sum(times) / nill, "unit": "images/s", "cores": cores, "kind": "port",
               "sample": cpu_sample_text(w, times, cores, info) +
               f"; one image = {nill} such solves (the oracle's image formation not counted)"}
    desc = (f"bright-field microscope (microsbf.f, FFT lens) of the c3 ellipsoid (96x96x64 full box, d=10 nm, "
            f"lambda=500 nm): objective NA 0.9, condenser NA 0.5, {nill} illuminations (s and p), image "
            f"512x512, magnification 100, GPBICG1 to 1e-4")
    line = {"metric": "microscope images/s", "value": m["images_per_s"], "unit": "images/s", "n_gpus": 1,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": m["ms_per_image"], "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "c64 inner / c128 outer", "data": "synthetic (seeded)",
            "config": {"workload": desc, "parallelism": "single GPU", "l2": "inputs > L2 (590k dipoles)"},
            "gpu_launches": m["launches_per_image"], "clocks": m["clocks"], "microscope": out,
            "cpu_baseline": cpu}
    g.close()
    ctx.close()
    if rank == 0:
        print(json.dumps(line), flush=True)
    return 0


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=60)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ifdda", choices=["ifdda", "reference"])
    ap.add_argument("--workload", default="c2", choices=["c1", "c2", "c3", "c4", "c5", "mic"])
    ap.add_argument("--no-cpu", action="store_true", help="skip the CPU oracle sample")
    ap.add_argument("--no-e2e", action="store_true", help="skip the end-to-end (host buffers) measurement")
    ap.add_argument("--requests", type=int, default=2000, help="c4: stream length")
    ap.add_argument("--rate", type=float, default=3.0, help="c4: Poisson arrival rate (requests/s)")
    ap.add_argument("--policy", default="fifo", choices=("fifo", "sjf"),
                    help="c4: admission order (oldest first, or least work first with a 5 s wait cap)")
    ap.add_argument("--slots", type=int, default=4, help="c4: concurrent solver slots")
    ap.add_argument("--ragged", action="store_true", help="c4: solve arrived requests of one box as ragged batches")
    ap.add_argument("--nrhs", type=int, default=1, help="matvec mode: right-hand sides per batched mat-vec")
    ap.add_argument("--precs", default="2,0", help="matvec mode: precisions (2 FP32, 0 FP64)")
    ap.add_argument("--mode", default="solve", choices=["solve", "matvec", "passes"],
                    help="matvec: time the five mat-vec passes only; passes: the passes inside solves")
    args = ap.parse_args()
    if args.impl == "reference":
        if args.workload in ("c4", "mic"):
            args.workload = "c2"
        return run_reference(args)
    if args.workload == "c4":
        return run_serving(args)
    if args.workload == "mic":
        return run_microscope(args)
    if args.mode == "matvec":
        return run_matvec(args)
    if args.mode == "passes":
        return run_solve_passes(args)
    return run_gpu(args)


if __name__ == "__main__":
    sys.exit(main())
