#!/usr/bin/env python
"""Benchmark of the linear PMCHWT solve on B200: solves/s (assemble + LU + solve).

Workload (N=1): the mixed-precision solve at scale -- an icosphere of radius
50 nm subdivided 4 times (5120 triangles, 7680 RWG edges, 15360 PMCHWT
unknowns, complex128), interior eps = -9 + 1.3i, vacuum outside, vacuum
wavelength 600 nm, x-polarised plane wave along +z.  One step = one solve:
system-matrix assembly + right-hand side + LU factorisation + solve with FP64
iterative refinement to a relative residual <= 1e-12.  The FP64 path is timed
beside it ("fp64"), and sigma_ext of the mixed solve is compared with the FP64
solve (which matches the CPU oracle to 1e-9 in the test suite).

Data are synthetic (a seeded icosphere; no dataset exists for this path).  The
3.8 GB FP64 matrix exceeds the 126 MB L2, so no L2 flush is needed between steps.

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl reference]

For N > 1 (torchrun) every rank solves its own replica (the path has no data
exchange: "replicas only"); the step time is the max over ranks.
"""
from __future__ import annotations

import argparse
import csv
import io
import json
import os
import statistics
import subprocess
import sys
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
PKG = os.path.join(ROOT, "for90-mom2_b200")
sys.path.insert(0, PKG)

METRIC = "solves/s (assemble+LU+solve), mixed vs FP64 on 1 B200 at sigma_ext rel err <=1e-6"
WL = 600e-9
EPS_IN = complex(-9.0, 1.3)
SUBDIV = 4
RADIUS_NM = 50.0
TOL = 1e-12
MAXIT = 60


def workload_name(subdiv):
    F = 20 * 4 ** subdiv
    return "icosphere r=50nm s=%d (%d triangles, %d unknowns), eps=-9+1.3i, 600 nm, x-pol pw +z" % (
        subdiv, F, 3 * F)


def dist_env():
    return int(os.environ.get("RANK", 0)), int(os.environ.get("LOCAL_RANK", 0)), int(os.environ.get("WORLD_SIZE", 1))


def load_peaks():
    path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(path):
        with open(path) as fh:
            d = json.load(fh)
        return d.get("hbm_gbs", 6650.0), d.get("bf16_tflops", 1590.0), "measured"
    return 6650.0, 1590.0, "fallback"


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled during the timed region."""

    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,clocks_event_reasons.hw_slowdown,"
         "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
         "clocks_event_reasons.sw_power_cap")

    def __init__(self, dev):
        self.dev = dev
        self.p = None

    def start(self):
        try:
            self.p = subprocess.Popen(["nvidia-smi", "-i", str(self.dev), "--query-gpu=" + self.Q,
                                       "--format=csv,noheader,nounits", "-lms", "200"],
                                      stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
        except OSError:
            self.p = None

    def stop(self):
        if self.p is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.p.terminate()
        out, _ = self.p.communicate(timeout=10)
        rows = [r for r in csv.reader(io.StringIO(out)) if len(r) >= 9]
        sm, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for r in rows:
            try:
                sm.append(float(r[1]))
                mx = float(r[2])
            except ValueError:
                continue
            for nm, v in zip(names, r[5:9]):
                if v.strip().lower() == "active":
                    reasons.add(nm)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": mx, "reasons": sorted(reasons),
                "samples": len(sm)}


def make_problem(M, subdiv):
    import numpy as np
    from mom_b200 import meshgen
    nodes, faces = meshgen.icosphere(subdiv, RADIUS_NM)
    ids = np.ones(len(faces), dtype=np.int32)
    return nodes, faces, ids, [[1], [-1]]


def cpu_sample(subdiv, threads, budget_s=20.0):
    """Time the CPU oracle (C restatement of the reference + OpenBLAS LAPACK) on a
    bounded sample of the workload and extrapolate to one full solve."""
    import numpy as np
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    os.environ.setdefault("OMP_NUM_THREADS", str(threads))
    import oracle as O
    from mom_b200 import meshgen
    nodes, faces = meshgen.icosphere(subdiv, RADIUS_NM)
    ids = np.ones(len(faces), int)
    P = O.OracleProblem(nodes, faces, ids, 1e-9, [[1], [-1]])
    F = len(faces)
    n = 2 * P.N
    om = O.omega_of(WL)
    ri = [1.0, np.sqrt(EPS_IN)]
    src = dict(type="pw", theta=0.0, phi=90 * O.DEGTORAD, psi=0.0)
    # assembly: rows of m_s test faces per domain, extrapolated by F / m_s
    m_s = max(2, min(F, 64))
    t0 = time.perf_counter()
    P.sysmat_sample(om, ri, 0, m_s, threads)
    t_asm = (time.perf_counter() - t0) * F / m_s
    # RHS and sigma: full
    t0 = time.perf_counter()
    q = P.srcvec(om, ri[0], src)
    t_rhs = time.perf_counter() - t0
    # LU + getrs: scipy zgetrf/zgetrs on an n_s x n_s matrix, scaled by n^3 and n^2
    from scipy.linalg import lapack
    n_s = min(n, 4096)
    rng = np.random.default_rng(0)
    As = rng.standard_normal((n_s, n_s)) + 1j * rng.standard_normal((n_s, n_s)) + n_s * np.eye(n_s)
    As = np.asfortranarray(As)
    t0 = time.perf_counter()
    lu, piv, info = lapack.zgetrf(As, overwrite_a=True)
    t_lu = (time.perf_counter() - t0) * (n / n_s) ** 3
    b = rng.standard_normal(n_s) + 0j
    t0 = time.perf_counter()
    lapack.zgetrs(lu, piv, b)
    t_rs = (time.perf_counter() - t0) * (n / n_s) ** 2
    total = t_asm + t_rhs + t_lu + t_rs
    sample = ("sysmat rows of %d/%d test faces per domain (x%d), srcvec full, zgetrf/zgetrs on n=%d (x(n/%d)^3, "
              "x(n/%d)^2); OpenMP + OpenBLAS" % (m_s, F, F // m_s, n_s, n_s, n_s))
    return dict(total_s=total, phases_s=dict(assembly=t_asm, rhs=t_rhs, lu=t_lu, getrs=t_rs), sample=sample)


def reduce_max(x, world, device):
    """Max of a per-rank scalar over the process group (step times are taken as the max over ranks)."""
    if world == 1:
        return x
    import torch
    import torch.distributed as dist
    t = torch.tensor([x], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def replica_value(ms_per_step_max, world):
    """Whole-job solves/s of N independent replicas: every rank completes one solve per step."""
    return world * 1000.0 / ms_per_step_max


def host_cores():
    try:
        return len(os.sched_getaffinity(0))
    except AttributeError:
        return os.cpu_count() or 1


def run_reference(args, rank, world):
    """Reference arm: the CPU restatement of the reference's path (the Fortran
    reference cannot be compiled here: no Fortran compiler), all host threads."""
    if rank != 0:
        return 0
    cores = host_cores()
    vals = []
    info = None
    for _ in range(args.steps):
        info = cpu_sample(args.subdiv, cores)
        vals.append(1.0 / info["total_s"])
    v = statistics.median(vals)
    line = {"impl": "reference", "metric": METRIC, "value": v, "unit": "solves/s", "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1e3 / v, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "complex128", "data": "synthetic",
            "config": {"workload": workload_name(args.subdiv), "precision": "FP64 (CPU)"},
            "cpu_baseline": {"value": v, "unit": "solves/s", "cores": cores, "kind": "port", "sample": info["sample"],
                             "phases_s": info["phases_s"]},
            "e2e": {"value": v, "unit": "solves/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)
    return 0


def run_ours(args, rank, local_rank, world):
    import numpy as np
    import torch
    import mom_b200 as M
    torch.cuda.set_device(local_rank)
    if world > 1:
        import torch.distributed as dist
        from datetime import timedelta
        dist.init_process_group("nccl", timeout=timedelta(seconds=600))
    nodes, faces, ids, doms = make_problem(M, args.subdiv)
    S = M.Solver(local_rank)
    S.set_problem(M.Problem.from_arrays(nodes, faces, ids, 1e-9, doms))
    om = M.omega_of(WL)
    ri = [1.0, np.sqrt(EPS_IN)]
    src = [M.src_pw(0, 90, 0)]
    stream = torch.cuda.ExternalStream(S.stream)

    def step(prec):
        S.sysmat(om, ri, prec)
        S.srcvec(om, ri[0], src)
        S.solve(prec, tol=TOL, maxit=MAXIT, want_host=False)

    def barrier():
        torch.cuda.synchronize()
        if world > 1:
            torch.distributed.barrier()
        torch.cuda.synchronize()

    def max_over_ranks(x):
        return reduce_max(x, world, "cuda")

    def timed(prec, steps, warm):
        # timers on during warm-up too, so the LU graph captured there (timing
        # nodes included) is the one replayed in the timed steps
        S.profile(True)
        for _ in range(warm):
            step(prec)
        barrier()
        l0, b0, f0 = S.launch_count, S.library_calls, S.tensor_flops
        S.profile(True)
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        iters = []
        for _ in range(steps):
            step(prec)
            iters.append(S.iters)
        e1.record(stream)
        e1.synchronize()
        prof = S.profile_read()
        S.profile(False)
        barrier()
        ms = e0.elapsed_time(e1) / steps
        return max_over_ranks(ms), prof, S.launch_count - l0, S.library_calls - b0, iters, S.tensor_flops - f0

    # ---- mixed precision (the headline) ----
    sampler = ClockSampler(local_rank)
    sampler.start()
    ms_mixed, prof, launches, libcalls, iters, tc_flops = timed(M.MIXED, args.steps, args.warmup)
    clocks = sampler.stop()
    csca, cabs = S.cross_sections(om, ri[0], src)
    ext_mixed = float(csca[0] + cabs[0])
    # ---- FP64 path, same workload ----
    ms_fp64, prof64, ext_fp64, sig_err = None, {}, None, None
    if args.fp64_steps > 0:
        ms_fp64, prof64, _, _, _, _ = timed(M.FP64, args.fp64_steps, 1)
        csca64, cabs64 = S.cross_sections(om, ri[0], src)
        ext_fp64 = float(csca64[0] + cabs64[0])
        sig_err = abs(ext_mixed - ext_fp64) / abs(ext_fp64)

    # ---- end to end through the C ABI with pinned host buffers ----
    e2e_ms = None
    if not args.no_e2e:
        pin_x = torch.empty((1, 2 * S.N * 2), dtype=torch.float64, pin_memory=True).numpy()
        xh = pin_x.view(np.complex128).reshape(2 * S.N, 1, order="F")
        S.solve_wavelength(om, ri, src, M.MIXED, TOL, MAXIT, want_host=True)
        barrier()
        t0 = time.perf_counter()
        for _ in range(args.steps):
            x = S.solve_wavelength(om, ri, src, M.MIXED, TOL, MAXIT, want_host=True)
            xh[:, 0] = x[:, 0]
            S.cross_sections(om, ri[0], src)
        torch.cuda.synchronize()
        e2e_ms = max_over_ranks((time.perf_counter() - t0) * 1e3 / args.steps)
    h2d = 48 * len(src) + 16 * len(ri)  # mom_src structs + refractive indices
    d2h = 16 * 2 * S.N * len(src) + 16 * len(src)  # solution + (csca, cabs)

    # ---- rooflines of the timed kernels (device time from events around each launch) ----
    hbm_gbs, bf16_tf, peak_src = load_peaks()
    F = len(faces)
    n = 2 * S.N
    nb = 64
    sm_mhz = clocks.get("sm_mhz") or 1965.0
    roofs = {}
    ms, cnt = prof["tc_gemm"]
    if cnt:
        ach = tc_flops / (ms * 1e-3) / 1e12
        roofs["tc_gemm"] = {"kernel": "tc_gemm_kernel (tcgen05 kind::tf32, 3 passes, LU trailing update)",
                            "bound": "tensor", "achieved": ach, "unit": "TFLOP/s", "peak": bf16_tf / 2.0,
                            "frac": ach / (bf16_tf / 2.0), "traffic": None,
                            "peak_note": "dense TF32 = half of the %s bf16 burst peak; FLOP = 3 passes executed" % peak_src}
    ms, cnt = prof["panel"]
    if cnt:
        bytes_ = sum(2.0 * 8 * (n - k * nb) * nb for k in range(n // nb)) * args.steps  # FP32 panel read + write
        ach = bytes_ / (ms * 1e-3) / 1e9
        # DRAM bytes of one panel launch at m = 3520 rows (ncu, profiles/panel_kernel_s3.md),
        # scaled by rows to the average panel height of this order
        traffic = 1.841e6 * (n / 2.0) / 3520.0
        roofs["panel"] = {"kernel": "panel_kernel<float2> (pivoted panel, one device-wide exchange per column)",
                          "bound": "hbm", "achieved": ach, "unit": "GB/s", "peak": hbm_gbs, "frac": ach / hbm_gbs,
                          "traffic": traffic, "traffic_note": "bytes per launch, ncu at 3520 rows scaled by rows",
                          "peak_note": "%s; latency-bound: one device-wide pivot exchange per column" % peak_src}
    ms, cnt = prof["pair"]
    if cnt:
        flop = 17914.0 * F * F * cnt  # 17,914 FLOP per face pair, F^2 pairs per launch (one domain)
        ach = flop / (ms * 1e-3) / 1e12
        peak = 148 * 128 * 2 * sm_mhz * 1e6 / 1e12
        roofs["pair"] = {"kernel": "pair_kernel<float,13> (far-pair assembly, FP32 pipe)", "bound": "fp32",
                         "achieved": ach, "unit": "TFLOP/s", "peak": peak, "frac": ach / peak,
                         "traffic": 430.4e6 * (F / 1280.0) ** 2,
                         "traffic_note": "bytes per launch, ncu at 1280 faces scaled by face pairs",
                         "peak_note": "nominal FP32 SIMT at the sampled SM clock %.0f MHz" % sm_mhz}
    ms, cnt = prof["trsv"]
    if cnt:
        bytes_ = 8.0 * n * n * cnt  # FP32 L and U factors read once per solve
        ach = bytes_ / (ms * 1e-3) / 1e9
        roofs["trsv"] = {"kernel": "trsv_flow_kernel<float2> (forward+backward substitution, published solved blocks)",
                         "bound": "hbm", "achieved": ach, "unit": "GB/s", "peak": hbm_gbs, "frac": ach / hbm_gbs,
                         "traffic": 125.4e6 * (n / 3840.0) ** 2,
                         "traffic_note": "bytes per launch, ncu at 3840 unknowns scaled by n^2",
                         "peak_note": peak_src}
    ms, cnt = prof["residual"]
    if cnt:
        bytes_ = 16.0 * n * n * cnt  # FP64 matrix read once per residual
        ach = bytes_ / (ms * 1e-3) / 1e9
        roofs["residual"] = {"kernel": "gemv_partial_kernel (FP64 refinement residual)", "bound": "hbm",
                             "achieved": ach, "unit": "GB/s", "peak": hbm_gbs, "frac": ach / hbm_gbs,
                             "traffic": None, "peak_note": peak_src}
    top = max(roofs, key=lambda k: prof[k][0])  # the kernel with the most device time per step
    roof = dict(roofs[top])

    phases = {k: {"ms_per_step": v[0] / args.steps, "launches_per_step": v[1] / args.steps} for k, v in prof.items()}
    phases64 = {k: {"ms_per_step": v[0] / args.fp64_steps} for k, v in prof64.items()}

    value = replica_value(ms_mixed, world)
    line = {"metric": METRIC, "value": value, "unit": "solves/s", "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": ms_mixed, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "fp32/tf32 far pairs + LU, fp64 near pairs + refinement (complex)",
            "data": "synthetic",
            "config": {"workload": workload_name(args.subdiv), "precision": "mixed", "refine_tol": TOL,
                       "l2": "matrix 3.8 GB > 126 MB L2, no flush", "parallelism": "replicas x%d" % world},
            "fp64": ({"value": world * 1000.0 / ms_fp64, "unit": "solves/s", "ms_per_step": ms_fp64,
                      "phases": phases64} if ms_fp64 else None),
            "mixed_over_fp64": (ms_fp64 / ms_mixed) if ms_fp64 else None,
            "sigma_ext": {"mixed": ext_mixed, "fp64": ext_fp64, "rel_err": sig_err},
            "refine_iters": iters,
            "phases": phases,
            "clocks": clocks,
            "e2e": ({"value": world * 1000.0 / e2e_ms, "unit": "solves/s", "h2d_bytes_per_step": h2d,
                     "d2h_bytes_per_step": d2h} if e2e_ms else None),
            "autotune_panel": {"mixed": tune_or_none(M, S, M.MIXED),
                               "fp64": tune_or_none(M, S, M.FP64) if ms_fp64 else None},
            "gpu_launches": int(launches),
            "library_gemm_calls": libcalls,
            "roofline": roof,
            "rooflines": roofs}
    if not args.no_extras and world == 1:
        line["sweep"] = bench_sweep(M, args.sweep_workers, local_rank)
        line["adjoint"] = bench_adjoint(M, local_rank)
        line["core_shell"] = bench_core_shell(M, local_rank)
        try:
            line["near_field"] = bench_nearfield(M, local_rank, with_cpu=not args.no_cpu)
        except Exception as exc:  # a side measurement must not cost the bench line
            line["near_field"] = {"error": repr(exc)[:300]}
    if rank == 0 and world == 1 and not args.no_cpu:
        cores = host_cores()
        info = cpu_sample(args.subdiv, cores)
        line["cpu_baseline"] = {"value": 1.0 / info["total_s"], "unit": "solves/s", "cores": cores, "kind": "port",
                                "sample": info["sample"], "phases_s": info["phases_s"]}
    if rank == 0:
        print(json.dumps(line), flush=True)
    S.close()
    if world > 1:
        torch.distributed.destroy_process_group()
    return 0


def bench_nearfield(M, dev, n=101, with_cpu=True):
    """Near fields (scat_fields + incident, the nfpl plane) of the cfg1 sphere
    (s=3, FP64 solution at 600 nm): an n x n grid 200 nm wide in the xz plane
    through the particle, exterior domain.  GPU time per plane through the C ABI
    (host points in, host fields out); with with_cpu, the CPU baseline of this
    row: the oracle on a sample of points on one host core, and the largest
    relative difference on that sample."""
    import numpy as np
    from mom_b200 import workloads as W
    nodes, faces, ids, doms = W.sphere(3)
    S = M.Solver(dev)
    S.set_problem(M.Problem.from_arrays(nodes, faces, ids, 1e-9, doms))
    om = M.omega_of(WL)
    src = [M.src_pw(0, 90, 0)]
    x = S.solve_wavelength(om, [1.0, np.sqrt(EPS_IN)], src, M.FP64, 1e-12, 30)
    a, b = np.meshgrid(np.linspace(-100e-9, 100e-9, n), np.linspace(-100e-9, 100e-9, n), indexing="ij")
    pts = np.stack([a.ravel(), np.zeros(n * n), b.ravel()], axis=1)
    S.scat_fields(om, 1.0, pts, x=x, srcs=src, dom=0)  # warm-up
    reps = 3
    t0 = time.perf_counter()
    for _ in range(reps):
        e, h = S.scat_fields(om, 1.0, pts, x=x, srcs=src, dom=0)
    gpu_s = (time.perf_counter() - t0) / reps
    S.close()
    F = len(faces)
    flop = 1300.0 * n * n * F  # ~13 x 70 FLOP of quadrature + ~400 of contraction per point-face pair
    out = {"workload": "nfpl plane %d x %d points (200 nm, xz) on the s=3 sphere, exterior domain, + incident" % (n, n),
           "gpu_ms_per_plane": gpu_s * 1e3, "points_per_s": n * n / gpu_s,
           "point_face_pairs_per_s": n * n * F / gpu_s,
           "fp64_tflops_est": flop / gpu_s / 1e12,
           "fp64_peak_note": "nominal FP64 SIMT 148 SM x 64 FMA x 2 x 1.965 GHz = 37 TFLOP/s; FLOP per pair estimated"}
    if with_cpu:
        sys.path.insert(0, os.path.join(ROOT, "oracle"))
        import oracle as O
        P = O.OracleProblem(nodes, faces, ids, 1e-9, doms)
        idx = np.linspace(0, n * n - 1, 16).astype(int)
        t0 = time.perf_counter()
        eo, ho = P.scat_fields(om, 1.0, x, pts[idx], srcs=src, d=0)
        cpu_s = time.perf_counter() - t0
        err = max(float(np.abs(e[0, idx] - eo[0]).max() / np.abs(eo[0]).max()),
                  float(np.abs(h[0, idx] - ho[0]).max() / np.abs(ho[0]).max()))
        out["cpu_baseline"] = {"value": len(idx) / cpu_s, "unit": "points/s", "cores": 1, "kind": "port",
                               "sample": "16 of the plane's points"}
        out["max_rel_diff_vs_oracle"] = err
    return out


def bench_sweep(M, workers, dev):
    """Uneven wavelength sweep: the s=3 sphere and three seeded ellipsoids, 64 wavelengths
    on 400-900 nm with a Drude permittivity, mixed precision refined to 1e-12; every mesh's
    wavelengths split over `workers` contexts that run concurrently (mom_gpu_sweep_many)."""
    import numpy as np
    from mom_b200 import workloads as W
    meshes = W.sweep_meshes()
    wls = W.sweep_wavelengths(64)
    oms = np.array([M.omega_of(w) for w in wls])
    ri = np.stack([np.ones(len(wls)), np.sqrt(W.drude_eps(wls))], axis=1)
    src = [M.src_pw(0, 90, 0)]
    solvers, parts = [], []
    for _, (nodes, faces, ids, doms) in meshes:
        prob = M.Problem.from_arrays(nodes, faces, ids, 1e-9, doms)
        for w in range(workers):
            s = M.Solver(dev)
            s.set_problem(prob)
            solvers.append(s)
            parts.append(np.arange(w, len(wls), workers))
    out = {"workload": "sweep: sphere s=3 + 3 ellipsoids (%s unknowns), 64 wavelengths 400-900 nm, Drude eps"
                       % "/".join(str(2 * solvers[i * workers].N) for i in range(len(meshes))),
           "contexts": len(solvers)}
    for prec, name in ((M.MIXED, "mixed"), (M.FP64, "fp64")):
        # warm-up: autotuning and graph capture of every context
        M.sweep_many(solvers, [oms[p[:1]] for p in parts], [ri[p[:1]] for p in parts], src, prec)
        t0 = time.perf_counter()
        res = M.sweep_many(solvers, [oms[p] for p in parts], [ri[p] for p in parts], src, prec)
        dt = time.perf_counter() - t0
        out[name] = {"solves_per_s": len(meshes) * len(wls) / dt, "seconds": dt,
                     "panel_ctas_by_height": [
                         (lambda t: dict(zip(t["heights"], t["ctas"])) if t else None)(
                             tune_or_none(M, solvers[i * workers], prec)) for i in range(len(meshes))]}
        out[name + "_sigma_ext_first"] = float(res[0][0][0, 0] + res[0][1][0, 0])
    for s in solvers:
        s.close()
    return out


def tune_or_none(M, S, prec):
    """The LU autotuner's table, or None when tuning is off (MOM_AUTOTUNE=0 / MOM_PANEL_CTAS)."""
    try:
        return S.autotune_result(prec)
    except M.MomError:
        return None


def bench_core_shell(M, dev, nsrc=512):
    """Core-shell (30,720 unknowns, 3 domains) with 512 incidences: one factorisation reused
    for all right-hand sides (GEMM-based blocked solves, FP64 ZGEMM residuals), cross
    sections, and d(mean sigma_ext, sigma_abs)/d(shell eps) by the adjoint; mixed and FP64."""
    import numpy as np
    from mom_b200 import workloads as W
    nodes, faces, ids, doms = W.core_shell(4)
    srcs = W.incidences(nsrc)
    S = M.Solver(dev)
    S.set_problem(M.Problem.from_arrays(nodes, faces, ids, 1e-9, doms))
    om = M.omega_of(WL)
    ri = [1.0, np.sqrt(W.EPS_AU), np.sqrt(W.EPS_SILICA)]
    out = {"workload": "core-shell s=4 (r 40/60 nm, %d unknowns), %d pw_elliptic incidences" % (2 * S.N, nsrc)}
    ext = {}
    for prec, name in ((M.MIXED, "mixed"), (M.FP64, "fp64")):
        S.solve_wavelength(om, ri, srcs[:1], prec, TOL, MAXIT, want_host=False)  # autotune + graph capture
        S.synchronize()
        t0 = time.perf_counter()
        S.solve_wavelength(om, ri, srcs, prec, TOL, MAXIT, want_host=False)
        a, b = S.cross_sections(om, ri[0], srcs)
        t1 = time.perf_counter()
        g = S.adjoint_mean_eps(om, ri, srcs, prec, eps_dom=1, tol=TOL, maxit=MAXIT)
        t2 = time.perf_counter()
        ext[name] = a + b
        out[name] = {"solve_s": t1 - t0, "rhs_per_s": nsrc / (t1 - t0), "adjoint_mean_eps_s": t2 - t1,
                     "refine_iters": S.iters, "dmean_ext_deps": [g[0, 0], g[0, 1]]}
    out["sigma_ext_max_rel_mixed_vs_fp64"] = float(np.max(np.abs(ext["mixed"] - ext["fp64"]) / np.abs(ext["fp64"])))
    S.close()
    return out


def bench_adjoint(M, dev):
    """Adjoint gradients on the perturbed s=3 sphere (3840 unknowns, 642 vertices):
    time of d sigma / d eps and of d sigma / d(all vertex coordinates), and the eps
    gradient against central differences (step 1e-6) of the FP64 cross sections."""
    import numpy as np
    from mom_b200 import workloads as W
    nodes, faces, ids, doms = W.perturbed(3)
    S = M.Solver(dev)
    S.set_problem(M.Problem.from_arrays(nodes, faces, ids, 1e-9, doms))
    om = M.omega_of(WL)
    src = [M.src_pw(0, 90, 0)]

    def sig(eps, prec=M.FP64):
        ri = [1.0, np.sqrt(eps)]
        S.solve_wavelength(om, ri, src, prec, 1e-12, 30)
        a, b = S.cross_sections(om, ri[0], src)
        return np.array([a[0] + b[0], b[0]])

    out = {"workload": "perturbed sphere s=3 (3840 unknowns, %d vertices)" % len(nodes)}
    fd = []
    for dz in (1e-6, 1e-6j):
        fd.append((sig(EPS_IN + dz) - sig(EPS_IN - dz)) / 2e-6)
    fd = np.array(fd)
    for prec, name in ((M.FP64, "fp64"), (M.MIXED, "mixed")):
        ri = [1.0, np.sqrt(EPS_IN)]
        sig(EPS_IN, prec)
        S.adjoint(om, ri, src, prec, eps_dom=1)  # untimed: first-call set-up
        t0 = time.perf_counter()
        g = S.adjoint(om, ri, src, prec, eps_dom=1)["deps"][0]
        t1 = time.perf_counter()
        sig(EPS_IN, prec)
        t2 = time.perf_counter()
        S.adjoint(om, ri, src, prec, nodes=True)
        t3 = time.perf_counter()
        out[name] = {"eps_grad_ms": (t1 - t0) * 1e3, "vertex_grad_ms": (t3 - t2) * 1e3,
                     "eps_grad_vs_fd_max_rel": float(np.max(np.abs(g.T - fd) / np.abs(fd)))}
    S.close()
    return out


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--fp64-steps", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--subdiv", type=int, default=SUBDIV)
    ap.add_argument("--no-cpu", action="store_true", help="skip the CPU baseline sample")
    ap.add_argument("--no-e2e", action="store_true", help="skip the end-to-end (host buffer) measurement")
    ap.add_argument("--no-extras", action="store_true", help="skip the sweep and adjoint side measurements")
    ap.add_argument("--sweep-workers", type=int, default=6, help="concurrent contexts per sweep mesh")
    args = ap.parse_args()
    rank, local_rank, world = dist_env()
    if args.impl == "reference":
        return run_reference(args, rank, world)
    return run_ours(args, rank, local_rank, world)


if __name__ == "__main__":
    sys.exit(main())
