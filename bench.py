#!/usr/bin/env python
"""Benchmark: 3D-RISM solute solves per second to ||F(t)||_inf < 1e-10.

Workload (one "step" = one complete solve from t = 0):
  3D-RISM/KH, a 24-site synthetic neutral solute (seeded PCG64, sites in a
  6 A ball, 1.2 A minimum separation, q ~ U[-0.8, 0.8] shifted to zero,
  sigma ~ U[2.5, 4], eps ~ U[0.05, 0.3]) in PR-SPC/E water, chi from 1D
  DRISM/KH (rmax 160 A, nrad 4096, eps_r 78.4), rho 0.0333295, beta 1.6889;
  grid 256^3 with half edge L = 24 A (48 A box, h = 0.1875 A).
  Synthetic data stand in for the reference's molecule inputs.

  python bench.py [--gpus N --steps K --warmup W] [--impl reference]

Our arm: mixed precision (FP32 bulk Newton, FP64 residual + FP32 Jacobian
refinement) with the two-grid preconditioner and flexible GMRES.  Timed
beside it: the plain FP64 form -- the reference's algorithm on the GPU,
FP64 throughout, GMRES(30) without preconditioner at a fixed rtol of 1e-3
(the metric's comparison point) -- and the FP64 form with our Krylov
solver.  The reference arm (--impl reference) times the CPU restatement of
the reference's algorithm (the reference itself cannot be built here) on a
bounded sample of residual and Jacobian evaluations, scaled by the number
of evaluations the plain FP64 solve takes.

Beside the timed line (unless --no-extras): "batch", 64 solutes of 3-40
sites on grids 64^3..192^3 solved by rism3d_solve_batch in mixed and FP64
precision (aggregate solves/s, per-solute |dmu|); "gradient", the adjoint
dmu/d(q, sigma, eps, x) of the workload's solute (time against one
solve, central-difference checks); "pes", an 8-point scan of the solute
rebound on one context with warm starts, against fresh solves;
"cufft_yardstick", the Jacobian product against a cuFFT (torch.fft) form of
it, speed and max difference; "large", the 512^3 / 150-site single solve
below, timed once.

  python bench.py --large           the 512^3 / 150-site single solve
                                    (mixed against plain FP64)

  python bench.py --profile-solve   one warm mixed solve between
                                    cudaProfilerStart/Stop (for ncu
                                    --profile-from-start off)
"""
import argparse
import json
import os
import statistics
import subprocess
import sys
import tempfile
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "solves/s to ‖r‖<1e-10 @256³ 3D-RISM: mixed+batched vs plain FP64, 1 B200"
GRID = 256
N_SITES = 24
SETTINGS = {"L": 24.0, "rho": 0.0333295, "beta": 1.6889, "closure": "KH", "rmax": 160.0, "nrad": 4096,
            "norm-tol": 1e-10, "dielectric": 78.4, "max-iter": 200}
# Residual (iterate_t1) and Jacobian (jacobian_t1) evaluations of one plain
# FP64 Newton-GMRES solve of this workload -- the reference's algorithm
# (SNES NEWTONLS, GMRES(30), rtol 1e-3), counted on the GPU form -- used to
# scale the CPU samples.
FP64_SOLVE_EVALS = {"f": 9, "jv": 464}
PLAIN_FP64 = {"precision": "fp64", "coarse-h": 0, "ew-forcing": 0, "krylov-restart": 30}
# DRAM bytes (read + write) of the five FP32 passes of one Jacobian product at
# 256^3 (x-forward 576.0, y 352.9, z 351.7, y-inverse 352.8, x-inverse
# 574.1 MB), measured by ncu dram__bytes_read.sum + dram__bytes_write.sum on
# the shape-specialised kernels.
JV_TRAFFIC = 2207.5e6


def workload(grid=GRID):
    from bgy3d_b200 import find_molecule, rism_solvent, synthetic_solute
    solvent = find_molecule("water, PR-SPC/E")
    solute = synthetic_solute(N_SITES, radius=6.0, seed=20261203)
    s = dict(SETTINGS, N=grid)
    chi = rism_solvent(solvent, dict(s, **{"norm-tol": 1e-12}))["susceptibility"]
    return solute, solvent, s, chi


BATCH_GRIDS = [64, 72, 96, 108, 128, 144, 162, 192]


def batch_workload(count=64, s=None):
    """Many-solute batch: solute i has n ~ U{3..40} sites drawn as the main
    workload's (seed 20261203 + i, 6 A ball), half edge L = extent + 16 A
    (extent = largest site distance from the centroid) and a grid drawn
    from the even 2^a 3^b set 64..192 (seeded PCG64)."""
    from bgy3d_b200 import synthetic_solute
    rng = np.random.Generator(np.random.PCG64(20261203))
    solutes, sets = [], []
    for i in range(count):
        n = int(rng.integers(3, 41))
        sol = synthetic_solute(n, radius=6.0, seed=20261203 + i)
        x = np.array([a["x"] for a in sol])
        ext = float(np.max(np.linalg.norm(x - x.mean(axis=0), axis=1)))
        solutes.append(sol)
        sets.append(dict(s, N=int(rng.choice(BATCH_GRIDS)), L=ext + 16.0))
    return solutes, sets


def run_batch_report(solvent, s, chi, count=64, workers=8):
    """Config of many solutes: aggregate solves/s of the mixed batch and of
    the FP64 batch, per-solute |dmu| mixed vs FP64."""
    import torch
    from bgy3d_b200 import hnc3d_run_batch
    solutes, sets = batch_workload(count, s)
    out = {}
    mus = {}
    # warm: one solute of every grid (the pass-schedule autotuner times each
    # new grid shape once per process, like an FFT plan)
    first = {}
    for i, x in enumerate(sets):
        first.setdefault(x["N"], i)
    warm = sorted(first.values())
    for prec in ("mixed", "fp64"):
        st = [dict(x, precision=prec) for x in sets]
        hnc3d_run_batch([solutes[i] for i in warm], solvent, [st[i] for i in warm], chi, workers=workers)
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        res = hnc3d_run_batch(solutes, solvent, st, chi, workers=workers)
        torch.cuda.synchronize()
        dt = time.perf_counter() - t0
        ok = sum(r["status"] == 0 for r in res)
        mus[prec] = np.array([r["free-energy"] for r in res])
        out[prec] = {"solves_per_s": count / dt, "seconds": dt, "converged": ok,
                     "launches": int(sum(r["launches"] for r in res))}
    dmu = np.abs(mus["mixed"] - mus["fp64"])
    out.update({"solutes": count, "workers": workers, "grids": BATCH_GRIDS,
                "sites": [len(x) for x in solutes][:8] + ["..."],
                "dmu_max": float(dmu.max()), "dmu_median": float(np.median(dmu)),
                "timing": "host clock around rism3d_solve_batch, setup and teardown of every solve included"})
    return out


def run_gradient_report(solute, solvent, s, chi, ms_solve):
    """Adjoint gradient of the main workload: time per gradient against the
    forward solve, and central differences (h = 1e-4, FP64 solves) for four
    parameters."""
    from bgy3d_b200 import RismContext, hnc3d_run_solute
    ctx = RismContext(solute, solvent, dict(s, precision="mixed"), chi)
    T, res = ctx.solve()
    ctx.gradient(T)  # warm
    g = ctx.gradient(T)
    ctx.close()
    h = 1e-4
    s64 = dict(s, precision="fp64", **{"norm-tol": 1e-12})
    t_host = T.cpu().numpy()
    checks = []
    for u, key, val in ((0, "charge", g["charge"][0]), (1, "sigma", g["sigma"][1]),
                        (2, "epsilon", g["epsilon"][2]), (3, "x", g["x"][3][0])):
        mu = []
        for sgn in (1, -1):
            sol = [dict(a) for a in solute]
            if key == "x":
                x = list(sol[u]["x"])
                x[0] += sgn * h
                sol[u]["x"] = tuple(x)
            else:
                sol[u][key] += sgn * h
            mu.append(hnc3d_run_solute(sol, solvent, s64, chi, restart=t_host, want_g=False)["free-energy"])
        fd = (mu[0] - mu[1]) / (2 * h)
        checks.append({"site": u, "param": key, "adjoint": val, "central_difference": fd,
                       "rel_err": abs(val - fd) / max(abs(fd), 1e-12)})
    return {"seconds_per_gradient": g["seconds"], "seconds_per_solve": ms_solve * 1e-3,
            "gradient_over_solve": g["seconds"] / (ms_solve * 1e-3), "adjoint_jv": g["adjoint-jv"],
            "adjoint_resid": g["adjoint-resid"], "fd_checks": checks,
            "params": "dmu/d{q, sigma, eps, x} of all %d sites" % len(solute)}


def run_pes_report(solute, solvent, s, chi, points=8, step=0.05):
    """A PES scan of the workload's solute (site 0 moved along x in steps of
    0.05 A): one context rebound per point with the solve warm-started from
    the previous t, against a fresh rism3d_solute_solve per point."""
    import torch
    from bgy3d_b200 import RismContext, hnc3d_run_solute
    st = dict(s, precision="mixed")

    def moved(k):
        out = [dict(a) for a in solute]
        x = list(out[0]["x"])
        x[0] += step * k
        out[0]["x"] = tuple(x)
        return out

    geoms = [moved(k) for k in range(points)]
    ctx = RismContext(solute, solvent, st, chi)
    T, _ = ctx.solve()
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    iters = []
    for g in geoms:
        ctx.set_solute(g)
        T, r = ctx.solve(T)
        iters.append(r["newton-iters"])
    torch.cuda.synchronize()
    warm = time.perf_counter() - t0
    ctx.close()
    t0 = time.perf_counter()
    for g in geoms:
        hnc3d_run_solute(g, solvent, st, chi, want_g=False, want_restart=False)
    torch.cuda.synchronize()
    fresh = time.perf_counter() - t0
    return {"points": points, "step_A": step, "rebind_warm_solves_per_s": points / warm,
            "fresh_solves_per_s": points / fresh, "newton_per_point": iters,
            "timing": "host clock around the scan"}


def run_cufft_yardstick(solute, solvent, s, chi, reps=5):
    """cuFFT as a speed and accuracy yardstick for the Jacobian product (the
    evaluation a plain FP64 solve makes 464 of): J dT = (chi-1) * (c'(T) dT)
    - dT written with torch.fft (cuFFT) and dense k-grid chi tables, against
    rism3d_jacobian_t1 on the same T (the workload's field at t = 0) and a
    seeded dT.  Device time per product (CUDA events) and the max |difference|."""
    import torch
    from bgy3d_b200 import RismContext
    ctx = RismContext(solute, solvent, s, chi)
    N, Lf = s["N"], 2 * s["L"]
    m = len(solvent)
    T = ctx.zeros()
    v = ctx.field(0)
    beta = s["beta"]
    x = -beta * v + T
    d = torch.where(x <= 0, torch.expm1(torch.clamp(x, max=0.0)), torch.zeros_like(x))  # KH slope
    g = torch.Generator(device="cuda").manual_seed(7)
    dT = torch.randn(T.shape, generator=g, device="cuda", dtype=torch.float64) * 1e-2
    # chi - 1 on the r2c grid by the reference's radial rule (bgy3d-vec.c:22-46)
    dk = 2 * np.pi / Lf
    kx = torch.arange(N // 2 + 1, device="cuda", dtype=torch.float64)
    ky = torch.fft.fftfreq(N, 1.0 / N, device="cuda", dtype=torch.float64)
    kk = torch.sqrt((kx[None, None, :] * dk) ** 2 + (ky[None, :, None] * dk) ** 2 + (ky[:, None, None] * dk) ** 2)
    nrad, dkr = chi.shape[-1], np.pi / s["rmax"]
    ix = kk / dkr - 0.5
    i = torch.clamp(torch.floor(ix + 0.5).long(), 0, nrad - 1)
    ip = torch.where(i < nrad - 2, i + 1, i)
    im = torch.where(i > 1, i - 1, i)
    tabs = torch.tensor(chi, device="cuda", dtype=torch.float64) - torch.eye(m, device="cuda", dtype=torch.float64)[
        :, :, None]
    K = torch.empty((m, m) + kk.shape, device="cuda", dtype=torch.float64)
    for a in range(m):
        for b in range(m):
            t = tabs[a, b]
            K[a, b] = t[i] + (t[ip] - t[im]) / (ip - im).to(torch.float64) * (ix - i)

    def jv_cufft(dt, dd, KK):
        c = torch.fft.rfftn(dd * dt, dim=(-3, -2, -1))
        re = torch.einsum("abxyz,bxyz->axyz", KK, c.real)
        im = torch.einsum("abxyz,bxyz->axyz", KK, c.imag)
        return torch.fft.irfftn(torch.complex(re, im), s=(N, N, N), dim=(-3, -2, -1)) - dt

    out = {}
    for name, dt_ in (("f64", torch.float64), ("f32", torch.float32)):
        Tq, dTq, dq, Kq = T.to(dt_), dT.to(dt_), d.to(dt_), K.to(dt_)
        ours = ctx.jacobian_t1(Tq, dTq)
        ref = jv_cufft(dTq, dq, Kq)
        torch.cuda.synchronize()
        times = {}
        for label, fn in (("ours", lambda: ctx.jacobian_t1(Tq, dTq, out=ours)), ("cufft", lambda: jv_cufft(dTq, dq, Kq))):
            fn()
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            torch.cuda.synchronize()
            e0.record()
            for _ in range(reps):
                fn()
            e1.record()
            torch.cuda.synchronize()
            times[label] = e0.elapsed_time(e1) / reps
        diff = float((ours.double() - ref.double()).abs().max())
        scale = float(ref.double().abs().max())
        out[name] = {"ms_ours": times["ours"], "ms_cufft": times["cufft"], "ours_over_cufft_speed":
                     times["cufft"] / times["ours"], "max_abs_diff": diff, "max_rel_diff": diff / scale}
        del Tq, dTq, dq, Kq, ours, ref
    ctx.close()
    out["note"] = ("J.v at 256^3 on the workload's T = 0: ours = rism3d_jacobian_t1 (5 fused passes); cufft = "
                   "torch.fft rfftn/irfftn + einsum with dense k-grid chi tables (yardstick only, not a product path)")
    return out


def run_large(args):
    """The large single solve: a 150-site synthetic neutral solute (seed
    20261203, sites in a 14 A ball) in PR-SPC/E water on a 512^3 grid with
    half edge 48 A (96 A box, h = 0.1875 A), mixed precision to |F|inf <
    1e-10 against the plain FP64 form; device time, peak device memory of
    the library's pool and per-pass HBM rates of one mixed solve."""
    print(json.dumps(large_report()))


def large_report():
    """run_large's measurement as a dict (also the "large" key of the default
    line, timed once after the timed steps)."""
    import torch
    from bgy3d_b200 import RismContext, find_molecule, lib, rism_solvent, synthetic_solute
    lib().rism3d_cache_clear()
    torch.cuda.empty_cache()
    solvent = find_molecule("water, PR-SPC/E")
    solute = synthetic_solute(150, radius=14.0, seed=20261203)
    s = dict(SETTINGS, N=512, L=48.0)
    chi = rism_solvent(solvent, dict(s, **{"norm-tol": 1e-12}))["susceptibility"]
    torch.cuda.synchronize()
    free0, _ = torch.cuda.mem_get_info()
    out = {"workload": "150-site synthetic neutral solute (14 A ball) in PR-SPC/E water, 512^3 grid, 96 A box, KH, "
                       "|F|inf < 1e-10", "grid": 512, "solute_sites": 150}
    for label, st in (("mixed", {"precision": "mixed"}), ("fp64_plain", PLAIN_FP64)):
        ctx = RismContext(solute, solvent, dict(s, **st), chi)
        T = ctx.zeros()
        if label == "mixed":  # one untimed solve (graph capture, Krylov buffers)
            ctx.solve(T)
            T.zero_()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        torch.cuda.synchronize()
        e0.record()
        _, res = ctx.solve(T)
        e1.record()
        torch.cuda.synchronize()
        obs = ctx.observables(T)
        free1, _ = torch.cuda.mem_get_info()
        out[label] = {"seconds": e0.elapsed_time(e1) * 1e-3, "mu": obs["free-energy"], "status": res["status"],
                      "resid_inf": res["resid-inf"], "newton": res["newton-iters"],
                      "jv_evals": res["jv-evals"] + res["jv-evals-fp32"], "jv_evals_coarse": res["jv-evals-coarse"],
                      "device_memory_gb": (free0 - free1) / 1e9}
        if label == "mixed":
            ctx.profile(True)  # a third solve with per-pass event timing
            T.zero_()
            ctx.solve(T)
            prof = ctx.profile(False)
            lau = {k: prof[(k, "f32")][1] for k in ("xfwd", "y", "z", "xinv")}
            byt = pass_bytes(512, 3, 4, lau, res["f-evals-fp32"])
            out[label]["pass_gbs_f32"] = {k: byt[k] / (prof[(k, "f32")][0] * 1e-3) / 1e9
                                          for k in lau if prof[(k, "f32")][0] > 0}
            out[label]["passes_ms"] = {f"{a}/{p}": round(v[0], 1) for (a, p), v in prof.items() if v[1]}
            out[label]["tile_shapes"] = ctx.tile_shapes()
        ctx.close()
        del T
        torch.cuda.synchronize()
    out["speedup_vs_plain_fp64"] = out["fp64_plain"]["seconds"] / out["mixed"]["seconds"]
    out["dmu_vs_fp64_plain"] = out["mixed"]["mu"] - out["fp64_plain"]["mu"]
    out["device_memory_note"] = "free device memory before the first context minus after each solve (the pool " \
                                "keeps its high-water mark)"
    return out


def config(grid=GRID, precision="mixed"):
    return {"workload": f"3D-RISM/KH solute solve to |F|inf<1e-10: {N_SITES}-site synthetic neutral solute "
                        f"in PR-SPC/E water (3 sites), {grid}^3 grid, 48 A box, chi from 1D DRISM "
                        f"(rmax 160, nrad 4096)", "grid": grid, "solute_sites": N_SITES, "solvent_sites": 3,
            "closure": "KH", "tolerance": 1e-10, "precision": precision,
            "l2": "fields of 67-201 MB per vector exceed the 126 MB L2; no flush needed"}


def clocks_start():
    f = tempfile.NamedTemporaryFile("w+", suffix=".csv", delete=False)
    q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")
    try:
        p = subprocess.Popen(["nvidia-smi", f"--query-gpu={q}", "--format=csv,noheader,nounits", "-lms", "200"],
                             stdout=f, stderr=subprocess.DEVNULL)
    except OSError:
        p = None
    return p, f.name


def clocks_stop(p, path, dev=0):
    if p is None:
        return None
    p.terminate()
    try:
        p.wait(timeout=5)
    except subprocess.TimeoutExpired:
        p.kill()
    sm, smax, reasons = [], None, set()
    names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
    for line in open(path):
        f = [x.strip() for x in line.split(",")]
        if len(f) < 9 or not f[0].isdigit() or int(f[0]) != dev:
            continue
        try:
            sm.append(float(f[1]))
            smax = float(f[2])
        except ValueError:
            continue
        for k, v in zip(names, f[5:9]):
            if v.lower().startswith("active"):
                reasons.add(k)
    os.unlink(path)
    if not sm:
        return None
    return {"sm_mhz": statistics.median(sm), "sm_max_mhz": smax, "reasons": sorted(reasons), "samples": len(sm)}


def hbm_peak():
    path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    try:
        return float(json.load(open(path))["hbm_gbs"]), "measured"
    except (OSError, KeyError, ValueError):
        return 6650.0, "fallback"


def pass_bytes(grid, m, b, launches, f_evals):
    """Algorithmic HBM bytes of each pass over all its launches (b = bytes per real)."""
    nr = grid ** 3
    nc = (grid // 2 + 1) * grid * grid  # complex half-spectrum points per site
    per = {
        "xfwd": m * (2 * nr * b + nc * 2 * b),        # read t (or dt) and v (or d), write W
        "y": m * 2 * nc * 2 * b,                      # read + write W
        "z": m * 2 * nc * 2 * b,                      # read + write W (+ long-range field in F)
        "xinv": m * (nc * 2 * b + 2 * nr * b),        # read W and t (or dt), write F
    }
    out = {k: per[k] * launches.get(k, 0) for k in per}
    out["z"] += f_evals * nc * 2 * b
    return out


def run_ours(args, rank, world):
    import torch
    import torch.distributed as dist
    from bgy3d_b200 import RismContext, hnc3d_run_solute, lib

    dev = int(os.environ.get("LOCAL_RANK", 0))
    torch.cuda.set_device(dev)
    solute, solvent, s, chi = workload(args.grid)
    ctx = RismContext(solute, solvent, dict(s, precision="mixed"), chi)
    T = ctx.zeros()

    def one(c):
        T.zero_()
        _, res = c.solve(T)
        obs = c.observables(T)
        return res, obs

    for _ in range(args.warmup):
        res, obs = one(ctx)
    if res["status"] != 0:
        raise RuntimeError(f"solve failed: {res}")
    if world > 1:
        dist.barrier()
    torch.cuda.synchronize()
    ctx.profile(False)  # reset launch counters
    clk, clk_path = clocks_start() if rank == 0 else (None, None)
    start, stop = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    start.record()
    for _ in range(args.steps):
        res, obs = one(ctx)
    stop.record()
    torch.cuda.synchronize()
    ms = start.elapsed_time(stop)
    clocks = clocks_stop(clk, clk_path, dev) if rank == 0 else None
    launches = sum(v[1] for v in ctx.profile(False).values())
    if world > 1:
        t = torch.tensor([ms], device="cuda", dtype=torch.float64)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        ms = float(t.item())
        dist.barrier()
    mixed = {"res": res, "obs": obs}

    def timed(settings, k):
        c = RismContext(solute, solvent, dict(s, **settings), chi)
        r, o = one(c)
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        for _ in range(k):
            r, o = one(c)
        e1.record()
        torch.cuda.synchronize()
        c.close()
        return r, o, e0.elapsed_time(e1) / k

    # plain FP64 form (the metric's comparison point) and FP64 with our solver
    resp, obsp, msp = timed(PLAIN_FP64, 1)
    res64, obs64, ms64 = timed({"precision": "fp64"}, max(1, min(args.steps, 2)))

    # per-pass device time of one mixed solve, for the roofline
    ctx.profile(True)
    one(ctx)
    prof = ctx.profile(False)

    # end to end through the host-buffer C-ABI call (hnc3d_run_solute): one
    # untimed call (it builds the device context the later calls reuse),
    # then k timed calls, each with its host arrays, solute upload, solve,
    # observables and the copy of g into host memory
    torch.cuda.synchronize()
    hnc3d_run_solute(solute, solvent, dict(s, precision="mixed"), chi, want_g=True, want_restart=False)
    k_e2e = max(1, min(args.steps, 3))
    t0 = time.perf_counter()
    for _ in range(k_e2e):
        out = hnc3d_run_solute(solute, solvent, dict(s, precision="mixed"), chi, want_g=True,
                               want_restart=False)
    e2e_s = (time.perf_counter() - t0) / k_e2e
    lib().rism3d_cache_clear()
    ctx.close()
    if rank != 0:
        return None

    m = 3
    bw, src = hbm_peak()
    # roofline of the FFT passes of F and J.v (FP32): the five fused passes
    # that evaluate the path's residual and Jacobian products
    prec = "f32"
    passes = ("xfwd", "y", "z", "xinv")
    lau = {kk: prof[(kk, prec)][1] for kk in passes}
    byt_all = pass_bytes(args.grid, m, 4, lau, res["f-evals-fp32"])
    pms = {kk: prof[(kk, prec)][0] for kk in passes}
    achieved = sum(byt_all.values()) / (sum(pms.values()) * 1e-3) / 1e9
    evals = res["f-evals-fp32"] + res["jv-evals-fp32"]
    pass_gbs = {kk: byt_all[kk] / (pms[kk] * 1e-3) / 1e9 for kk in passes if pms[kk] > 0}
    total_ms = sum(v[0] for v in prof.values())
    value = world * args.steps / (ms * 1e-3)
    line = {
        "metric": METRIC, "value": value, "unit": "solves/s", "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": ms / args.steps, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f32+f64 (mixed)", "data": "synthetic (seeded solute, 1D-DRISM chi)",
        "config": dict(config(args.grid), parallelism=f"replicas x{world} (independent solutes)"),
        "fp64_plain": {"value": 1e3 / msp, "unit": "solves/s", "ms_per_step": msp,
                       "solver": "GMRES(30), no preconditioner, fixed rtol 1e-3 (the reference's)",
                       "newton": resp["newton-iters"], "f_evals": resp["f-evals"], "jv_evals": resp["jv-evals"],
                       "resid_inf": resp["resid-inf"], "mu": obsp["free-energy"]},
        "speedup_vs_plain_fp64": msp / (ms / args.steps),
        "fp64": {"value": 1e3 / ms64, "unit": "solves/s", "ms_per_step": ms64,
                 "solver": "two-grid FGMRES(30), Eisenstat-Walker forcing",
                 "newton": res64["newton-iters"], "f_evals": res64["f-evals"], "jv_evals": res64["jv-evals"],
                 "jv_evals_coarse": res64["jv-evals-coarse"], "resid_inf": res64["resid-inf"],
                 "mu": obs64["free-energy"]},
        "speedup_vs_fp64": ms64 / (ms / args.steps),
        "solve": {"mu": mixed["obs"]["free-energy"], "mu_fp64_plain": obsp["free-energy"],
                  "dmu_vs_fp64_plain": mixed["obs"]["free-energy"] - obsp["free-energy"],
                  "dmu_vs_fp64": mixed["obs"]["free-energy"] - obs64["free-energy"],
                  "resid_inf": res["resid-inf"], "newton": res["newton-iters"],
                  "f_evals_f64": res["f-evals"], "jv_evals_f64": res["jv-evals"],
                  "f_evals_f32": res["f-evals-fp32"], "jv_evals_f32": res["jv-evals-fp32"],
                  "jv_evals_coarse": res["jv-evals-coarse"]},
        "roofline": {"bound": "hbm", "kernel": "F / J.v FFT passes (FP32: x-forward, y, z, y-inverse, x-inverse)",
                     "achieved": achieved, "peak": bw, "peak_source": src, "unit": "GB/s", "frac": achieved / bw,
                     "traffic": JV_TRAFFIC,
                     "traffic_note": "ncu dram__bytes_read.sum + dram__bytes_write.sum of the five FP32 passes "
                                     "of one J.v at 256^3 (per launch of the pipeline)",
                     "bytes_per_launch": sum(byt_all.values()) / max(evals, 1),
                     "share_of_solve": sum(pms.values()) / total_ms, "pass_gbs": pass_gbs,
                     "passes_ms": {f"{a}/{p}": round(v[0], 3) for (a, p), v in prof.items() if v[1]}},
        "e2e": {"value": 1.0 / e2e_s, "unit": "solves/s",
                "h2d_bytes_per_step": int(48 * N_SITES),
                "d2h_bytes_per_step": int(out["GUV"].nbytes), "calls": k_e2e,
                "timing": "host clock around hnc3d_run_solute (rism3d_solute_solve with host buffers): solute "
                          "upload, solve from t = 0, observables, g copied into a fresh host array; the device "
                          "context of the untimed first call is reused (the solute rebound)"},
        "gpu_launches": int(launches),
    }
    if clocks:
        line["clocks"] = clocks
    if world == 1 and not args.no_cpu_baseline:
        line["cpu_baseline"] = cpu_baseline(args)
    if world == 1 and not args.no_extras:
        extras = (("batch", lambda: run_batch_report(solvent, s, chi)),
                  ("gradient", lambda: run_gradient_report(solute, solvent, s, chi, ms / args.steps)),
                  ("pes", lambda: run_pes_report(solute, solvent, s, chi)),
                  ("cufft_yardstick", lambda: run_cufft_yardstick(solute, solvent, dict(s, precision="mixed"), chi)),
                  ("large", large_report))
        for key, fn in extras:
            try:
                line[key] = fn()
            except Exception as e:  # an extra report never costs the timed line
                line[key] = {"error": f"{type(e).__name__}: {e}"}
    return line


def host_threads():
    """Host threads this process may run on (all of them are used)."""
    try:
        return len(os.sched_getaffinity(0))
    except AttributeError:
        return os.cpu_count() or 1


def cpu_problem(grid, threads):
    """The workload as the CPU restatement's Problem (built once); returns it
    with its set-up time (field, chi and long-range tables)."""
    from oracle import closures as cl
    from oracle import hnc3d
    solute, solvent, s, chi = workload(grid)
    t0 = time.perf_counter()
    P = hnc3d.Problem((grid,) * 3, (2 * s["L"],) * 3, s["beta"], s["rho"], cl.KH, solvent, solute, chi,
                      s["rmax"], threads=threads)
    return P, time.perf_counter() - t0


def cpu_evals(P):
    """One bounded sample: one iterate_t1 and one jacobian_t1 of the CPU
    restatement at the workload's size; returns their seconds."""
    T = np.zeros((P.m, P.N[2], P.N[1], P.N[0]))
    t0 = time.perf_counter()
    F = P.iterate_t1(T)
    tf = time.perf_counter() - t0
    t0 = time.perf_counter()
    P.jacobian_t1(T, F)
    return tf, time.perf_counter() - t0


def per_solve_model(setup_s, tf, tj):
    """Seconds of one plain FP64 solve: set-up plus the residual and Jacobian
    evaluations of the reference's Newton-GMRES at this workload."""
    return setup_s + FP64_SOLVE_EVALS["f"] * tf + FP64_SOLVE_EVALS["jv"] * tj


def cpu_scaling_check(threads, grid=64):
    """A complete plain FP64 Newton-GMRES solve (GMRES(30), rtol 1e-3,
    backtracking) of the workload's solute at a small grid on the CPU
    restatement, timed, against the evaluation-count model: the model holds
    when the solve's time is its set-up plus its F and J.v evaluations."""
    from oracle import newton
    P, setup_s = cpu_problem(grid, threads)
    cnt = {"f": 0, "jv": 0, "tf": 0.0, "tj": 0.0}

    def F(x):
        t0 = time.perf_counter()
        r = P.iterate_t1(x)
        cnt["tf"] += time.perf_counter() - t0
        cnt["f"] += 1
        return r

    def J(x, v):
        t0 = time.perf_counter()
        r = P.jacobian_t1(x, v)
        cnt["tj"] += time.perf_counter() - t0
        cnt["jv"] += 1
        return r

    t0 = time.perf_counter()
    newton.solve(F, np.zeros((P.m, grid, grid, grid)), jv=J, tol=SETTINGS["norm-tol"])
    solve_s = time.perf_counter() - t0
    tf, tj = cnt["tf"] / max(cnt["f"], 1), cnt["tj"] / max(cnt["jv"], 1)
    model = setup_s + cnt["f"] * tf + cnt["jv"] * tj
    return {"grid": grid, "f_evals": cnt["f"], "jv_evals": cnt["jv"], "measured_s": setup_s + solve_s,
            "model_s": model, "measured_over_model": (setup_s + solve_s) / model}


def cpu_baseline(args):
    threads = host_threads()
    P, setup_s = cpu_problem(args.grid, threads)
    tf, tj = cpu_evals(P)
    per_solve = per_solve_model(setup_s, tf, tj)
    return {"value": 1.0 / per_solve, "unit": "solves/s", "cores": threads, "kind": "port",
            "sample": f"NumPy/SciPy restatement of hnc3d.c on {threads} host threads at {args.grid}^3: set-up "
                      f"{setup_s:.2f} s + {FP64_SOLVE_EVALS['f']} x iterate_t1 ({tf:.2f} s) + "
                      f"{FP64_SOLVE_EVALS['jv']} x jacobian_t1 ({tj:.2f} s), the evaluations of one plain FP64 "
                      f"Newton-GMRES solve; one F and one J.v timed"}


def run_reference(args):
    """The reference arm: the CPU restatement of the reference's algorithm
    (the reference itself needs PETSc/FFTW/MPI/Guile, absent here) on all
    host threads.  Built once; each step is one bounded sample (one F and
    one J.v at the full size) scaled to a solve by the evaluation counts."""
    threads = host_threads()
    P, setup_s = cpu_problem(args.grid, threads)
    times = []
    for _ in range(args.warmup + args.steps):
        tf, tj = cpu_evals(P)
        times.append((tf, tj))
    t = times[args.warmup:]
    tf = sum(a for a, _ in t) / len(t)
    tj = sum(b for _, b in t) / len(t)
    per_solve = per_solve_model(setup_s, tf, tj)
    value = 1.0 / per_solve
    del P
    check = cpu_scaling_check(threads)
    sample = (f"per step one iterate_t1 + one jacobian_t1 of the NumPy/SciPy restatement of hnc3d.c at "
              f"{args.grid}^3 on {threads} host threads (mean {tf:.3f} s + {tj:.3f} s over {len(t)} steps); a solve "
              f"= set-up ({setup_s:.2f} s, once) + {FP64_SOLVE_EVALS['f']} F + {FP64_SOLVE_EVALS['jv']} J.v, the "
              f"evaluations of the plain FP64 Newton-GMRES solve; model checked by a complete CPU solve at "
              f"{check['grid']}^3 (measured / model = {check['measured_over_model']:.3f})")
    return {"metric": METRIC, "value": value, "unit": "solves/s", "n_gpus": 1, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": 1e3 * per_solve, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64", "impl": "reference",
            "data": "synthetic (seeded solute, 1D-DRISM chi)", "config": config(args.grid, "fp64"),
            "cpu_baseline": {"value": value, "unit": "solves/s", "cores": threads, "kind": "port",
                             "sample": sample},
            "scaling_check": check,
            "e2e": {"value": value, "unit": "solves/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}


def run_profile_solve(args):
    """Profiling mode: one mixed solve between cudaProfilerStart/Stop (after
    two warm solves), then its per-pass totals from rism3d_profile."""
    import torch
    from bgy3d_b200 import RismContext
    solute, solvent, s, chi = workload(args.grid)
    ctx = RismContext(solute, solvent, dict(s, precision="mixed"), chi)
    T = ctx.zeros()
    for _ in range(2):
        T.zero_()
        ctx.solve(T)
    torch.cuda.synchronize()
    ctx.profile(False)
    torch.cuda.profiler.start()
    T.zero_()
    _, res = ctx.solve(T)
    torch.cuda.synchronize()
    torch.cuda.profiler.stop()
    launches = sum(v[1] for v in ctx.profile(True).values())
    T.zero_()
    ctx.solve(T)
    prof = ctx.profile(False)
    ctx.close()
    print(json.dumps({"grid": args.grid, "launches": launches, "result": {k: v for k, v in res.items()},
                      "passes_ms": {f"{a}/{p}": round(v[0], 3) for (a, p), v in prof.items() if v[1]}}))


def run_evals(args):
    """Profiling mode: args.evals residual and Jacobian evaluations in each
    precision on the workload (no Newton solve); prints per-evaluation times."""
    import torch
    from bgy3d_b200 import RismContext
    solute, solvent, s, chi = workload(args.grid)
    ctx = RismContext(solute, solvent, s, chi)
    out = {"grid": args.grid}
    for dt in (torch.float32, torch.float64):
        T = ctx.zeros(dt)
        F, _ = ctx.iterate_t1(T)
        ctx.jacobian_t1(T, F)
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        for _ in range(args.evals):
            ctx.iterate_t1(T, out=F)
        e1.record()
        torch.cuda.synchronize()
        tf = e0.elapsed_time(e1) / args.evals
        J = torch.empty_like(F)
        e0.record()
        for _ in range(args.evals):
            ctx.jacobian_t1(T, F, out=J)
        e1.record()
        torch.cuda.synchronize()
        out[str(dt).split(".")[-1]] = {"F_ms": tf, "Jv_ms": e0.elapsed_time(e1) / args.evals}
    ctx.close()
    print(json.dumps(out))


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="b200", choices=["b200", "reference"])
    ap.add_argument("--grid", type=int, default=GRID)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-extras", action="store_true",
                    help="skip the many-solute batch and gradient reports")
    ap.add_argument("--evals", type=int, default=0,
                    help="profiling mode: time this many F and J.v evaluations instead of solves")
    ap.add_argument("--large", action="store_true",
                    help="the 512^3 / 150-site single solve against plain FP64 (prints its own line)")
    ap.add_argument("--profile-solve", action="store_true",
                    help="profiling mode: one warm mixed solve between cudaProfilerStart/Stop")
    args = ap.parse_args()
    if args.evals:
        run_evals(args)
        return
    if args.profile_solve:
        run_profile_solve(args)
        return
    if args.large:
        run_large(args)
        return
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    if args.impl == "reference":
        if rank == 0:
            print(json.dumps(run_reference(args)))
        return
    if world > 1:
        import datetime

        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=600))
    line = run_ours(args, rank, world)
    if world > 1:
        import torch.distributed as dist
        dist.barrier()
        dist.destroy_process_group()
    if rank == 0:
        print(json.dumps(line))


if __name__ == "__main__":
    main()
