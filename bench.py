#!/usr/bin/env python
"""Benchmark of the VIE solve on B200 (one JSON line on rank 0).

Workload (default ``c3``): 256^3 organic solar cell (PEDOT 40 nm, P3HT:PCBM
120 nm, 16 Ag spheres r = 20 nm seeded in the active layer), 1 nm voxels,
padded 512^3, x-polarised plane wave at 550 nm, the reference's CORS driver
(CORS_FFT) to relative residual 1e-8 from x0 = 0.  Synthetic geometry from
vie_fft_b200.geometry.

One step = one full solve on inputs resident in HBM: FP32-complex inner CORS
inside FP64 defect correction (``value``, solves/s).  The all-FP64 CORS solve
of the same system is timed after it for the speed-up, and the operator
application (the hot op) is timed on its own for the roofline.  ``extras``
holds the same pair for BiCGSTAB (the reference's default driver) and short
summaries of the batched (C4) and gradient (C5) workloads.

``e2e`` times the same solve through the C ABI with host buffers: every step
copies the incident field from pinned host memory to the device and the
solution back (both inside the timed region).

``--impl reference`` times the reference's own CPU code (oracle/_ref: the
reference vie_fft compiled against the MKL shim; the C restatement when the
reference build is absent) on a bounded sample of the same workload: one
L_DC_Dq block (two 512^3 FFTs, the spectral multiply, the crop) per process,
one process per usable host core, scaled to solves/s with the operator's nine
blocks per application and the FP64 iteration count of this workload.

Multi-GPU: replicas only (instances are independent, like the reference's
per-wavelength process farm); value = total solves / max time over ranks.
"""
from __future__ import annotations

import argparse
import json
import multiprocessing as mp
import os
import statistics
import subprocess
import sys
import tempfile
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "solves/s & matvec ms to rel-res 1e-8: mixed vs FP64 on 1 B200; % HBM peak"
TOL = 1e-8
# the 32^3 sphere is solved to 1e-6 by BiCGSTAB, as the reference's CPU case is
# specified; the 128^3 and 256^3 lines time the reference's CORS driver (CORS_FFT,
# CG_Iteration.h:780-1073), the fastest of its drivers to 1e-8 on these grids
# (256^3 to 1e-8: FP64 CORS 4.98 s, BiCGSTAB 7.62 s; mixed CORS 2.47 s, mixed
# BiCGSTAB 4.20 s), with the BiCGSTAB figures of the 256^3 case in `extras`
WORKLOAD_TOL = {"c1": 1e-6}
WORKLOAD_SOLVER = {"c1": "bicgstab", "c2": "cors", "c3": "cors"}
# iterations of the FP64 solve of these workloads (driver and tolerance above):
# 256^3 CORS 279 and 128^3 CORS 17 measured on the GPU, 32^3 BiCGSTAB 24 the
# reference's own (its 23 steps + 1); used only to scale the CPU sample to solves/s
FP64_ITERS = {"c3": 279, "c2": 17, "c1": 24}


def tol_of(name):
    return WORKLOAD_TOL.get(name, TOL)


def solver_of(name):
    return WORKLOAD_SOLVER.get(name, "bicgstab")


def workload(name):
    from vie_fft_b200 import geometry as G
    if name.startswith("grid:"):
        # synthetic operator of any shape for kernel timing: random metal voxels, all edges flagged
        import numpy as np
        shape = tuple(int(v) for v in name[5:].split(","))
        rng = np.random.default_rng(0)
        mat = (rng.random(shape) < 0.3).astype(np.uint8) * 2
        flags = np.ones((3,) + shape, np.uint8)
        d = float(G.nm(1.0))
        w = G.Workload("grid", shape, (d, d, d), G.k0_of(550.0), mat, flags,
                       np.array([G.AIR_DUMMY, 2.0, G.to_reference_eps(-8.5 + 0.3j), 2.0]))
        return w, f"synthetic {shape} operator (random metal voxels)"
    if name == "c3":
        return G.solar_cell(), "256^3 organic solar cell (PEDOT/P3HT:PCBM, 16 Ag spheres r=20nm), 1 nm voxels, " \
                               "padded 512^3, x-pol 550 nm, CORS to rel-res 1e-8"
    if name == "c2":
        return G.sphere_cluster(), "128^3 cluster of 40 Au spheres (r 5-15 nm, seed 2) in eps_b=1.77, 1 nm voxels, " \
                                   "padded 256^3, x-pol 500 nm, CORS to rel-res 1e-8"
    if name == "c1":
        return G.single_sphere(), "32^3 Ag sphere r=18 nm, 1.25 nm voxels, padded 64^3, x-pol 400 nm, " \
                                  "BiCGSTAB to rel-res 1e-6"
    raise SystemExit(f"unknown workload {name}")


def bytes_per_matvec(shape, e):
    """Algorithmic HBM bytes of one operator application (five pruned passes):
    e*(3*(3a + 4b + 4c) + g) + a, a = NxNyNz, b = NxNy*2Nz, c = Nx*2Ny*2Nz,
    g = the (Nx+1)(Ny+1)(Nz+1) Green octant, + a bytes of edge flags."""
    nx, ny, nz = shape
    a = nx * ny * nz
    b = nx * ny * 2 * nz
    c = nx * 2 * ny * 2 * nz
    g = (nx + 1) * (ny + 1) * (nz + 1)
    return e * (3 * (3 * a + 4 * b + 4 * c) + g) + a


def measured_peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        with open(p) as f:
            d = json.load(f)
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


class ClockSampler:
    """nvidia-smi clock / throttle samples during the timed region."""

    def __init__(self, gpu_index):
        self.f = tempfile.NamedTemporaryFile("w+", suffix=".csv", delete=False)
        q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")
        try:
            self.p = subprocess.Popen(["nvidia-smi", f"--id={gpu_index}", f"--query-gpu={q}", "--format=csv,noheader,nounits",
                                       "-lms", "200"], stdout=self.f, stderr=subprocess.DEVNULL)
        except FileNotFoundError:
            self.p = None

    def stop(self):
        if self.p is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.p.terminate()
        self.p.wait()
        self.f.seek(0)
        rows = [l.strip().split(", ") for l in self.f.read().splitlines() if l.strip()]
        os.unlink(self.f.name)
        sm, smax, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for r in rows:
            try:
                sm.append(float(r[1]))
                smax = float(r[2])
                for nm_, v in zip(names, r[5:9]):
                    if v.strip() == "Active":
                        reasons.add(nm_)
            except (ValueError, IndexError):
                continue
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": smax, "reasons": sorted(reasons),
                "samples": len(sm)}


# ---------------------------------------------------------------------------
# reference / CPU baseline
# ---------------------------------------------------------------------------
def _block_worker(args):
    shape, d, k0, use_ref = args
    from oracle import oracle as O
    return O.time_block(O.Grid(*shape, *d, k0), use_reference=use_ref)


def cpu_block_sample(w, procs, use_ref=True):
    """Time one L_DC_Dq block of workload w in `procs` concurrent processes."""
    ctx = mp.get_context("spawn")
    t0 = time.perf_counter()
    with ctx.Pool(procs) as pool:
        res = pool.map(_block_worker, [(w.shape, w.d, w.k0, use_ref)] * procs)
    wall = time.perf_counter() - t0
    return res, wall


def usable_cores(w):
    n = os.cpu_count() or 1
    try:
        import psutil
        mem = psutil.virtual_memory().available
    except Exception:
        mem = 8 << 30
    per = 16 * 8 * w.a * 2 + 16 * w.a * 4  # Green + padded array + vectors of one block
    return max(1, min(n, int(mem * 0.6 // per), 64))


def cpu_solves_per_s(block_seconds, iters):
    # one BiCGSTAB or CORS iteration = 2 operator applications = 2 x 9 blocks
    return 1.0 / (block_seconds * 9 * 2 * iters)


def workload_config(w, desc, tol=TOL, solver="bicgstab"):
    """The workload both arms time: grid, padding, driver and tolerance."""
    return {"workload": desc, "grid": list(w.shape), "padded": [2 * s for s in w.shape], "solver": solver,
            "tol": tol}


def run_reference(args, rank, world):
    if rank != 0:
        return
    w, desc = workload(args.workload)
    from oracle import oracle as O
    use_ref = O.ref_available()
    kind = "reference" if use_ref else "port"
    iters = args.fp64_iters or FP64_ITERS.get(args.workload) or 0
    procs = usable_cores(w)
    # warm-up: the same block on a 64^3 grid (pages in code and allocator)
    for _ in range(max(args.warmup, 1)):
        _block_worker(((64, 64, 64), w.d, w.k0, use_ref))
    times = []
    for _ in range(args.steps):
        res, wall = cpu_block_sample(w, procs, use_ref)
        per = max(r["seconds"] for r in res)
        times.append(per)
    block = statistics.median(times)
    # aggregate over the processes that ran concurrently
    value = procs * cpu_solves_per_s(block, iters) if iters else None
    line = {"impl": "reference", "metric": METRIC, "value": value, "unit": "solves/s", "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": block * 1e3, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "c128", "data": "synthetic",
            "config": workload_config(w, desc, tol_of(args.workload), solver_of(args.workload)),
            "arm": {"precision": "c128 (the reference's double-complex path on the MKL shim)",
                    "parallelism": f"{procs} host processes"},
            "cpu_baseline": {"value": value, "unit": "solves/s", "cores": procs, "kind": kind,
                             "sample": f"one L_DC_Dq block (two {2*w.shape[0]}^3 FFTs + multiply + crop) per "
                                       f"process, {procs} processes; solves/s = procs / (block_s * 9 blocks * "
                                       f"2 matvecs * {iters} FP64 iterations)",
                             "block_seconds": block},
            "e2e": {"value": value, "unit": "solves/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


# ---------------------------------------------------------------------------
# GPU arm
# ---------------------------------------------------------------------------
def run_gpu(args, rank, world, local_rank):
    import numpy as np
    import torch

    import vie_fft_b200 as V
    from vie_fft_b200 import post

    torch.cuda.set_device(local_rank)
    dist = None
    if world > 1:
        import torch.distributed as dist
    w, desc = workload(args.workload)
    if world > 1:
        # replicas: each rank solves its own wavelength of the same geometry
        from vie_fft_b200 import geometry as G
        from vie_fft_b200.replicas import replica_wavelength
        w.k0 = G.k0_of(replica_wavelength(w.meta["wavelength_nm"], rank))
    c = V.Context(*w.shape, *w.d, w.k0, device=local_rank)
    c.set_flags(w.flags)
    if w.eps_voxel is not None:
        c.set_eps(w.eps_voxel)
    else:
        c.set_material(w.material, w.eps_table)
    t0 = time.perf_counter()
    c.green()
    green_s = time.perf_counter() - t0
    c.incident(w.theta, w.phi, w.psi, copy=False)
    stream = torch.cuda.ExternalStream(c.stream_ptr())
    # FFT schedule of this grid picked by the autotuner (outside the timed region)
    t0 = time.perf_counter()
    schedule = c.autotune() if not args.no_autotune else "defaults"
    tune_s = time.perf_counter() - t0

    def barrier():
        torch.cuda.synchronize()
        if dist is not None:
            dist.barrier()

    def solve(precision, true_residual=False, out=None, solver=None):
        r = c.solve(solver or solver_of(args.workload), tol=tol_of(args.workload), precision=precision,
                    copy=out is not None, out=out, true_residual=true_residual)
        return r

    if args.only_matvec:
        # operator applications only (profiling entry): FP32 then FP64, W warm-up + K timed each
        res = {}
        for name, dt, prec in (("fp32", torch.complex64, V.PREC_MIXED), ("fp64", torch.complex128, V.PREC_FP64)):
            x = torch.randn((3,) + w.shape, dtype=dt, device="cuda")
            y = torch.zeros_like(x)
            torch.cuda.synchronize()
            for _ in range(args.warmup):
                c.matvec_dev(x.data_ptr(), y.data_ptr(), precision=prec)
            c.sync()
            a0, a1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            a0.record(stream)
            for _ in range(args.steps):
                c.matvec_dev(x.data_ptr(), y.data_ptr(), precision=prec)
            a1.record(stream)
            a1.synchronize()
            ms = a0.elapsed_time(a1) / args.steps
            B = bytes_per_matvec(w.shape, 8 if name == "fp32" else 16)
            res[name] = {"ms": ms, "GBps": B / ms / 1e6, "hbm_frac": B / ms / 1e6 / measured_peaks()[0]}
            del x, y
        if rank == 0:
            print(json.dumps({"mode": "matvec", "workload": args.workload, "grid": list(w.shape), **res}), flush=True)
        c.close()
        return

    # ---- warm-up
    for _ in range(args.warmup):
        last = solve(V.PREC_MIXED)
    # ---- timed region: K mixed solves
    barrier()
    sampler = ClockSampler(local_rank) if rank == 0 else None
    launches0 = V.launch_count()
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    ev0.record(stream)
    infos = []
    for _ in range(args.steps):
        infos.append(solve(V.PREC_MIXED).info)
    ev1.record(stream)
    ev1.synchronize()
    barrier()
    launches = V.launch_count() - launches0
    clocks = sampler.stop() if sampler else None
    ms = ev0.elapsed_time(ev1) / args.steps
    from vie_fft_b200.replicas import throughput
    value, ms_max = throughput(1.0, ms, device="cuda")
    x_mixed = c.solution()

    # ---- FP64 reference solve of the same system (speed-up and accuracy)
    solve(V.PREC_FP64)
    barrier()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    n64 = max(1, min(2, args.steps))
    for _ in range(n64):
        r64 = solve(V.PREC_FP64)
    e1.record(stream)
    e1.synchronize()
    ms64 = e0.elapsed_time(e1) / n64
    x64 = c.solution()
    rel64 = {"true_relres": c.residual()}

    # ---- operator roofline (the hot op of each precision), inputs > L2
    def time_matvec(dtype, prec, reps=10):
        x = torch.randn((3,) + w.shape, dtype=dtype, device="cuda")
        y = torch.zeros_like(x)
        torch.cuda.synchronize()
        for _ in range(3):
            c.matvec_dev(x.data_ptr(), y.data_ptr(), precision=prec)
        c.sync()
        a0, a1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a0.record(stream)
        for _ in range(reps):
            c.matvec_dev(x.data_ptr(), y.data_ptr(), precision=prec)
        a1.record(stream)
        a1.synchronize()
        del x, y
        return a0.elapsed_time(a1) / reps

    mv32 = time_matvec(torch.complex64, V.PREC_MIXED)
    mv64 = time_matvec(torch.complex128, V.PREC_FP64)
    peak, peak_kind = measured_peaks()
    B32, B64 = bytes_per_matvec(w.shape, 8), bytes_per_matvec(w.shape, 16)
    ach32 = B32 / (mv32 * 1e-3) / 1e9
    ach64 = B64 / (mv64 * 1e-3) / 1e9
    traffic = None
    tf = os.path.join(ROOT, "profiles", "matvec_dram_bytes.json")
    if os.path.exists(tf):
        with open(tf) as f:
            tj = json.load(f)
        traffic = tj.get(args.workload, {}).get("fp32")

    # ---- end to end through the C ABI with pinned host buffers
    e2e = None
    if args.e2e_steps > 0:
        h_rhs = torch.empty((3,) + w.shape, dtype=torch.complex128, pin_memory=True)
        h_x = torch.empty((3,) + w.shape, dtype=torch.complex128, pin_memory=True)
        e_host = c.incident(w.theta, w.phi, w.psi, copy=True)
        h_rhs.numpy()[...] = e_host
        xn = h_x.numpy()
        barrier()
        f0, f1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        tw0 = time.perf_counter()
        f0.record(stream)
        for _ in range(args.e2e_steps):
            c.set_rhs(h_rhs.numpy())
            c.solve(solver_of(args.workload), tol=tol_of(args.workload), precision=V.PREC_MIXED, out=xn,
                    true_residual=False)
        f1.record(stream)
        f1.synchronize()
        wall = (time.perf_counter() - tw0) / args.e2e_steps
        ms_e2e = f0.elapsed_time(f1) / args.e2e_steps
        e2e_value, _ = throughput(1.0, ms_e2e, device="cuda")
        e2e = {"value": e2e_value, "unit": "solves/s",
               "h2d_bytes_per_step": int(h_rhs.numel() * 16), "d2h_bytes_per_step": int(h_x.numel() * 16),
               "wall_ms_per_step": wall * 1e3}

    if rank != 0:
        return
    # ---- accuracy of the mixed solve against FP64
    cs_mixed = post.cross_sections(w, x_mixed)
    cs_64 = post.cross_sections(w, x64)
    xerr = {k: abs(cs_mixed[k] - cs_64[k]) / max(abs(cs_64[k]), 1e-300) for k in cs_64}
    field_rel = float(np.linalg.norm(x_mixed - x64) / np.linalg.norm(x64))
    # ---- post-processing of the solution on the GPU (FarField1, FarField2, NearField)
    post_ms = {}
    for name, fn in (("farfield1", lambda: c.farfield1(w.theta, w.phi, w.psi)), ("farfield2", lambda: c.farfield2(w.phi)),
                     ("nearfield", lambda: c.nearfield(w.material))):
        fn()
        t0 = time.perf_counter()
        fn()
        post_ms[name] = (time.perf_counter() - t0) * 1e3

    # ---- CPU baseline (bounded sample), rank 0 at N = 1 only
    cpu = None
    if world == 1 and not args.no_cpu:
        from oracle import oracle as O
        use_ref = O.ref_available()
        res, wall = cpu_block_sample(w, 1, use_ref)
        blk = res[0]["seconds"]
        iters64 = r64.info["iterations"]
        cpu = {"value": cpu_solves_per_s(blk, iters64), "unit": "solves/s", "cores": 1, "kind": res[0]["kind"],
               "sample": f"one L_DC_Dq block at {w.shape} ({2*w.shape[0]}^3 padded FFT pair, {blk:.1f} s), "
                         f"scaled by 9 blocks x 2 matvecs x {iters64} FP64 {solver_of(args.workload)} iterations",
               "block_seconds": blk}

    info = infos[-1]
    line = {
        "metric": METRIC, "value": value, "unit": "solves/s", "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": ms_max, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "c64 inner + c128 refine", "data": "synthetic",
        "config": workload_config(w, desc, tol_of(args.workload), solver_of(args.workload)),
        "arm": {"precision": "mixed (FP32 inner Krylov, FP64 "
                             + ("reliable updates)" if solver_of(args.workload) == "bicgstab" else "defect correction)"),
                "l2": "inputs larger than L2 (FP32 vectors 403 MB, FP64 805 MB each)",
                "parallelism": "replicas" if world > 1 else "single"},
        "roofline": {"bound": "hbm", "achieved": ach32, "peak": peak, "unit": "GB/s", "frac": ach32 / peak,
                     "traffic": traffic, "kernel": "FP32 operator application (5 pruned FFT passes)",
                     "peak_source": peak_kind, "algorithmic_bytes": B32},
        "e2e": e2e,
        "gpu_launches": launches,
        "clocks": clocks,
        "cpu_baseline": cpu,
        "fp64": {"solves_per_s": 1e3 / ms64, "ms_per_solve": ms64, "iterations": r64.info["iterations"],
                 "true_relres": rel64["true_relres"]},
        "speedup_mixed_vs_fp64": ms64 / ms_max,
        "mixed": {"iterations": info["iterations"], "outer": info["outer"], "matvecs_fp32": info["matvecs_fp32"],
                  "matvecs_fp64": info["matvecs_fp64"], "true_relres": info["true_relres"]},
        "matvec_ms": {"fp32": mv32, "fp64": mv64},
        "matvec_hbm_frac": {"fp32": ach32 / peak, "fp64": ach64 / peak},
        "xsec_rel_err_mixed_vs_fp64": xerr, "field_rel_diff_mixed_vs_fp64": field_rel,
        "green_setup_s": green_s, "fft_schedule": schedule, "autotune_s": tune_s,
        "post_ms_gpu": post_ms,
    }
    bicgstab = None
    if world == 1 and args.workload == "c3" and not args.no_extras:
        # the reference's default driver on the same system: mixed and FP64 BiCGSTAB
        # (one warm-up solve each for the graph capture, then one timed)
        bicgstab = {}
        for name, prec in (("mixed", V.PREC_MIXED), ("fp64", V.PREC_FP64)):
            solve(prec, solver="bicgstab")
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            rb = solve(prec, solver="bicgstab")
            e1.record(stream)
            e1.synchronize()
            bicgstab[name] = {"solves_per_s": 1e3 / e0.elapsed_time(e1), "ms": e0.elapsed_time(e1),
                              "iterations": rb.info["iterations"], "outer": rb.info["outer"]}
        bicgstab["speedup_mixed_vs_fp64"] = bicgstab["fp64"]["ms"] / bicgstab["mixed"]["ms"]
        bicgstab["speedup_mixed_cors_vs_fp64_bicgstab"] = bicgstab["fp64"]["ms"] / ms_max
    c.close()
    if world == 1 and args.workload == "c3" and not args.no_extras:
        line["extras"] = extra_configs(args, rank, world, local_rank)
        line["extras"]["bicgstab_256"] = bicgstab
    print(json.dumps(line), flush=True)


def extra_configs(args, rank, world, local_rank):
    """Summaries of the batched (C4) and adjoint-gradient (C5) workloads, run
    after the headline measurement so that their figures are recorded with it:
    one warm-up and one timed step each, C5 without its finite-difference pass
    (tests/test_c5_fd_gpu.py holds that check)."""
    ex = argparse.Namespace(**vars(args))
    ex.steps, ex.warmup = 1, 1
    ex.workload = "c4"
    l4 = run_gpu_batch(ex, rank, world, local_rank, emit=False)
    ex.workload = "c5"
    l5 = run_gpu_gradient(ex, rank, world, local_rank, emit=False, fd_check=False)
    return {
        "note": "1 warm-up + 1 timed step each, host wall time of the batch / gradient call",
        "c4": {"workload": l4["config"]["workload"], "instances": l4["config"]["instances"],
               "instances_per_s_mixed": l4["value"], "instances_per_s_fp64": l4["fp64"]["instances_per_s"],
               "speedup_mixed_vs_fp64": l4["speedup_mixed_vs_fp64"],
               "xsec_max_rel_err_mixed_vs_fp64": l4["xsec_max_rel_err_mixed_vs_fp64"],
               "iterations_min_max_mixed": l4["mixed"]["iterations_min_max"],
               "operator_GBps": l4["operator_GBps"],
               "failed": l4["mixed"]["failed"], "gpu_launches": l4["gpu_launches"]},
        "c5": {"workload": l5["config"]["workload"], "gradients_per_s_mixed": l5["value"],
               "gradients_per_s_fp64": l5["fp64"]["gradients_per_s"],
               "speedup_mixed_vs_fp64": l5["speedup_mixed_vs_fp64"],
               "grad_rel_diff_mixed_vs_fp64": l5["grad_rel_diff_mixed_vs_fp64"],
               "power_rel_diff_mixed_vs_fp64": l5["power"]["rel_diff"], "gpu_launches": l5["gpu_launches"],
               "iterations_fwd_adj_mixed": l5["mixed"]["iterations_fwd_adj"],
               "iterations_fwd_adj_fp64": l5["fp64"]["iterations_fwd_adj"]},
    }


def batch_workloads(name):
    """Batched workloads: c4 = the wavelength x polarisation sweep (64 x 2 over a
    96x96x48 solar cell, Drude silver) plus 48 single spheres on uneven grids
    (edges 16..96 step 8); c4i / c4ii = either part alone."""
    from vie_fft_b200 import geometry as G
    sweep = G.batch_sweep() if name in ("c4", "c4i") else []
    spheres = G.batch_spheres() if name in ("c4", "c4ii") else []
    desc = []
    if sweep:
        desc.append("64 wavelengths (350-800 nm, Drude Ag) x 2 polarisations over a 96x96x48 solar cell")
    if spheres:
        desc.append("48 single spheres, grid edge 16..96 (step 8), eps Re[-6,-1] Im[0.1,1]")
    return sweep + spheres, " + ".join(desc) + "; BiCGSTAB to rel-res 1e-8, one CUDA graph launch per batch"


def run_gpu_batch(args, rank, world, local_rank, emit=True):
    """Batched solve: every instance in one vie_solve_batch call (one graph
    launch).  value = instances / batch time (mixed precision); the FP64 batch
    of the same instances gives the speed-up and the accuracy figures."""
    import numpy as np
    import torch

    import vie_fft_b200 as V
    from vie_fft_b200 import post

    torch.cuda.set_device(local_rank)
    from vie_fft_b200.replicas import shard, throughput
    ws_all, desc = batch_workloads(args.workload)
    ws = shard(ws_all, rank, world)  # replicas: each rank solves its share of the instances
    t0 = time.perf_counter()
    ctxs = []
    for w in ws:
        c = V.Context(*w.shape, *w.d, w.k0, device=local_rank)
        c.set_flags(w.flags)
        c.set_material(w.material, w.eps_table)
        c.green()
        c.incident(w.theta, w.phi, w.psi, copy=False)
        ctxs.append(c)
    setup_s = time.perf_counter() - t0
    n = len(ws)
    for _ in range(args.warmup):
        V.solve_batch(ctxs, "bicgstab", tol=TOL, precision=V.PREC_MIXED, copy=False, raise_errors=False)
    torch.cuda.synchronize()
    sampler = ClockSampler(local_rank) if rank == 0 else None
    launches0 = V.launch_count()
    secs, res = [], None
    for _ in range(args.steps):
        res = V.solve_batch(ctxs, "bicgstab", tol=TOL, precision=V.PREC_MIXED, copy=False, raise_errors=False)
        secs.append(res[0].info["seconds"])
    launches = V.launch_count() - launches0
    clocks = sampler.stop() if sampler else None
    t_mixed_local = statistics.median(secs)
    value_all, ms_max = throughput(len(ws), t_mixed_local * 1e3, device="cuda")
    t_mixed = ms_max / 1e3
    x_mixed = [c.solution() for c in ctxs]
    r64 = V.solve_batch(ctxs, "bicgstab", tol=TOL, precision=V.PREC_FP64, copy=True, raise_errors=False)
    t64 = r64[0].info["seconds"]
    # accuracy of the mixed batch against the FP64 batch, per instance
    xerr = {"q_ext": 0.0, "q_abs_metal": 0.0}
    for w, xm, r in zip(ws, x_mixed, r64):
        a, b = post.cross_sections(w, xm), post.cross_sections(w, r.x)
        for k in xerr:
            if b[k] != 0:
                xerr[k] = max(xerr[k], abs(a[k] - b[k]) / abs(b[k]))
    it = [r.info["iterations"] for r in res]
    it64 = [r.info["iterations"] for r in r64]
    # operator bytes moved by the batch (algorithmic bytes of every FP32 and FP64
    # application; the Krylov vector passes are not counted): a lower bound of
    # the batch's HBM throughput
    op_bytes = sum(r.info["matvecs_fp32"] * bytes_per_matvec(w.shape, 8) +
                   r.info["matvecs_fp64"] * bytes_per_matvec(w.shape, 16) for w, r in zip(ws, res))
    op_bytes64 = sum(r.info["matvecs_fp64"] * bytes_per_matvec(w.shape, 16) for w, r in zip(ws, r64))
    line = {
        "metric": "batched instances/s to rel-res 1e-8 (FP32 inner / FP64 refine, one graph launch per batch)",
        "value": value_all, "unit": "instances/s", "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": t_mixed * 1e3, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "c64 inner + c128 refine", "data": "synthetic",
        "config": {"workload": desc, "instances": len(ws_all), "instances_per_rank": n, "solver": "bicgstab",
                   "tol": TOL, "parallelism": f"replicas x{world}" if world > 1 else "single",
                   "voxels_total": int(sum(w.a for w in ws))},
        "fp64": {"instances_per_s": n / t64, "s_per_batch": t64, "iterations_min_max": [min(it64), max(it64)]},
        "speedup_mixed_vs_fp64": t64 / t_mixed,
        "mixed": {"iterations_min_max": [min(it), max(it)], "failed": sum(1 for r in res if r.status),
                  "graph_loops": res[0].info["graph_loops"]},
        "xsec_max_rel_err_mixed_vs_fp64": xerr,
        "operator_GBps": {"mixed": op_bytes / t_mixed / 1e9, "fp64": op_bytes64 / t64 / 1e9,
                          "note": "operator applications x algorithmic bytes / batch time (vector passes not counted)"},
        "gpu_launches": launches, "clocks": clocks, "setup_s": setup_s,
        "device_bytes": torch.cuda.mem_get_info()[1] - torch.cuda.mem_get_info()[0],
    }
    if rank == 0 and emit:
        print(json.dumps(line), flush=True)
    for c in ctxs:
        c.close()
    return line


def run_gpu_gradient(args, rank, world, local_rank, emit=True, fd_check=True):
    """Adjoint gradient of the active-layer absorption summed over 450, 550 and
    650 nm (x-polarised) on the 128x128x64 design stack (64x64x32 design
    region, seed 5).  value = gradient evaluations/s with mixed-precision forward
    and adjoint solves; also FP64, the agreement of the two, and FP64 central
    differences (h = 1e-6 on Re and Im) at 32 seeded design voxels (seed 6)."""
    import numpy as np
    import torch

    import vie_fft_b200 as V
    from vie_fft_b200 import geometry as G
    from vie_fft_b200 import post

    torch.cuda.set_device(local_rank)
    lams = (450.0, 550.0, 650.0)
    ws = [G.design_stack(wavelength_nm=lam) for lam in lams]
    mask = post.edge_mask(ws[0].material, 3)
    ctxs = []
    for w in ws:
        c = V.Context(*w.shape, *w.d, w.k0, device=local_rank)
        c.set_flags(w.flags)
        c.set_eps(w.eps_voxel)
        c.green()
        c.incident(w.theta, w.phi, w.psi, copy=False)
        ctxs.append(c)

    def evaluate(precision, tol, grad=True):
        p, g, its = 0.0, 0.0, []
        for c in ctxs:
            pi, gi, fi, ai = c.power_grad(mask, tol=tol, precision=precision, grad=grad)
            p += pi
            if grad:
                g = g + gi
            its.append((fi["iterations"], ai["iterations"]))
        return p, g, its

    for _ in range(args.warmup):
        evaluate(V.PREC_MIXED, TOL)
    torch.cuda.synchronize()
    sampler = ClockSampler(local_rank) if rank == 0 else None
    launches0 = V.launch_count()
    t0 = time.perf_counter()
    for _ in range(args.steps):
        pm, gm, itm = evaluate(V.PREC_MIXED, TOL)
    torch.cuda.synchronize()
    t_mixed = (time.perf_counter() - t0) / args.steps
    launches = (V.launch_count() - launches0) // args.steps
    clocks = sampler.stop() if sampler else None
    t0 = time.perf_counter()
    p64, g64, it64 = evaluate(V.PREC_FP64, TOL)
    torch.cuda.synchronize()
    t64 = time.perf_counter() - t0
    fd = None
    if fd_check:
        fd = fd_check_c5(ws, ctxs, mask, evaluate)
    line = {
        "metric": "adjoint gradient evaluations/s (absorbed power in the active layer, 3 wavelengths, "
                  "forward + adjoint solves to rel-res 1e-8)",
        "value": 1.0 / t_mixed, "unit": "gradients/s", "n_gpus": 1, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": t_mixed * 1e3, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "c64 inner + c128 refine", "data": "synthetic",
        "config": {"workload": "128x128x64 solar-cell stack, 64x64x32 design region (eps Re[1,4] Im[0,0.5], "
                               "seed 5), 450/550/650 nm x-pol, objective = NearField Ene_Active sum",
                   "design_voxels": int(ws[0].meta["region"].sum())},
        "fp64": {"gradients_per_s": 1.0 / t64, "iterations_fwd_adj": it64},
        "mixed": {"iterations_fwd_adj": itm},
        "speedup_mixed_vs_fp64": t64 / t_mixed,
        "power": {"mixed": pm, "fp64": p64, "rel_diff": abs(pm - p64) / abs(p64)},
        "grad_rel_diff_mixed_vs_fp64": float(np.abs(gm - g64).max() / np.abs(g64).max()),
        "fd_check": fd,
        "gpu_launches": launches, "clocks": clocks,
    }
    if rank == 0 and emit:
        print(json.dumps(line), flush=True)
    for c in ctxs:
        c.close()
    return line


def fd_check_c5(ws, ctxs, mask, evaluate):
    """Central differences of the FP64 objective at 32 seeded design voxels
    (the same check as tests/test_c5_fd_gpu.py, over the three wavelengths)."""
    import numpy as np

    import vie_fft_b200 as V
    region = np.argwhere(ws[0].meta["region"])
    rng = np.random.default_rng(6)
    picks = [tuple(region[i]) for i in rng.choice(len(region), 32, replace=False)]
    # the FP64 solves of the differences go to 1e-13 (capped at 5000 iterations):
    # with h = 1e-6 the difference quotient carries the solve error / h
    h, fd_tol = 1e-6, 1e-13
    _, gref, _ = evaluate(V.PREC_FP64, fd_tol)
    scale = float(np.abs(gref[ws[0].meta["region"]]).max())
    errs = []
    for v in picks:
        fd = []
        for dz in (h, 1j * h):
            vals = []
            for sgn in (1.0, -1.0):
                tot = 0.0
                for w, c in zip(ws, ctxs):
                    eps = w.eps_voxel.copy()
                    eps[v] += sgn * dz
                    c.set_eps(eps)
                    tot += c.power_grad(mask, tol=fd_tol, grad=False, max_iter=5000)[0]
                vals.append(tot)
            fd.append((vals[0] - vals[1]) / (2 * h))
        errs.append(abs(gref[v] - (fd[0] + 1j * fd[1])) / scale)
    worst = max(errs)
    for w, c in zip(ws, ctxs):
        c.set_eps(w.eps_voxel)
    return {"voxels": 32, "h": h, "solve_tol": fd_tol, "max_abs_err_over_max_grad": worst,
            "median_abs_err_over_max_grad": float(np.median(errs)), "max_grad": scale}


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="vie", choices=["vie", "reference"])
    ap.add_argument("--workload", default="c3",
                    help="c1 | c2 | c3 | c4 (batched: c4i sweep, c4ii spheres) | c5 (adjoint gradient), "
                         "or grid:NX,NY,NZ "
                         "(synthetic operator, --only-matvec)")
    ap.add_argument("--e2e-steps", type=int, default=2)
    ap.add_argument("--no-cpu", action="store_true")
    ap.add_argument("--fp64-iters", type=int, default=0)
    ap.add_argument("--no-autotune", action="store_true", help="keep the default FFT schedule")
    ap.add_argument("--no-extras", action="store_true",
                    help="c3: skip the C4 / C5 summaries appended to the line")
    ap.add_argument("--only-matvec", action="store_true",
                    help="time operator applications only (FP32 and FP64), no solve")
    args = ap.parse_args()
    if args.warmup < 3:
        args.warmup = 3
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local_rank = int(os.environ.get("LOCAL_RANK", "0"))
    if args.impl == "reference":
        run_reference(args, rank, world)
        return
    if world > 1:
        import datetime

        import torch
        import torch.distributed as dist
        torch.cuda.set_device(local_rank)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=600))
    try:
        if args.workload.startswith("c4"):
            run_gpu_batch(args, rank, world, local_rank)
        elif args.workload == "c5":
            run_gpu_gradient(args, rank, world, local_rank)
        else:
            run_gpu(args, rank, world, local_rank)
    finally:
        if world > 1:
            import torch.distributed as dist
            dist.destroy_process_group()


if __name__ == "__main__":
    main()
