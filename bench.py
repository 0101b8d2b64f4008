#!/usr/bin/env python3
"""Benchmark of the dense PMCHWT solve (the metric of this repository).

Workload: icosphere refinement 5 (20480 triangles, 30720 RWG, 61440
unknowns), ka = 15, m = 1.3116 + 1e-4 i, 7-point quadrature, 45 x 31 x 1
orientations x 2 polarisations = 2790 right-hand sides.

A step is one solve: FP32 factorisation of the FP64-assembled Z (tensor-core
updates with FP32 operands split into three FP16 products after power-of-two
row / column scaling; --tensor-split 0: three TF32 products), the
2790-column triangular solves, and FP64
iterative refinement (int8 digit-pair residuals of iterates kept to two
digits) until every column's estimated relative error is below 2e-10 (the
metric asks for 1e-9; the measured error against the FP64 LU solution is
reported as max_rel_err_vs_fp64).
value = seconds per solve: the device time of the K timed steps (one region
bracketed by barrier + synchronize, CUDA events) divided by K, max over
ranks; step_times_s lists the steps.  The
plain FP64 LU + solve of the same Z is timed once beside it and is the
oracle of the 1e-9 error check.  e2e = the whole pipeline through the C ABI
call bem_dense_run (host mesh in, host Mueller matrix out).

--impl reference: the reference's CPU dense path (python/bem_core.py,
restated by the oracle: assembly, LAPACK zgetrf / zgetrs as bem_core.py:1637,
1713 call them, far field) on bounded samples scaled to the workload; value
is the solve, e2e the whole path.

--config c1 | c2 | c4 | c5: the other workloads of the path (run_config);
the default, c3, is the metric's.

--impl cusolver: the reference's GPU call for the solve, cuSOLVER getrf +
getrs in FP64 (solver.cu:87-142; 64-bit API, baseline/cusolver_lu.cpp), on
the same device-assembled Z and right-hand sides, with this library's FP64
LU and FP32 + refinement solves timed beside it under the same clocks and
the solutions compared.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import tempfile
import time

REPO = os.path.dirname(os.path.abspath(__file__))
for _p in (REPO, os.path.join(REPO, "bem-cpp_b200")):
    if _p not in sys.path:
        sys.path.insert(0, _p)

METRIC = "s/solve at 2N=61440: FP32+refine vs FP64 LU on one B200 at 1e-9 rel err"
FP64_PEAK_TFS = 37.0
# DRAM traffic of a kernel class from ncu captures of the full-size launches
# (one-pass dram__bytes_read/write): per algorithmic byte for the trailing
# update, per int8 digit-pair GEMM for the residual
TRAFFIC_MODEL = {
    "lu_update": ("per_byte", 1.52, "ncu dram__bytes_read+write of the first 2N=61440 lower-triangle update "
                                    "(45.75 GB) / its algorithmic bytes (30.1 GB), times the average launch's "
                                    "algorithmic bytes"),
    "residual": ("per_pair", 75.6e9, "ncu dram__bytes_read+write of the two 2N=61440 residuals (2.105 TB for 28 "
                                     "digit pairs, 1.142 TB for 15) = 75.6 GB per digit-pair GEMM, times the "
                                     "average launch's pairs"),
}


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=3)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="bem", choices=["bem", "reference", "cusolver"])
    ap.add_argument("--ref", type=int, default=5, help="icosphere refinement (5: 2N=61440)")
    ap.add_argument("--ka", type=float, default=15.0)
    ap.add_argument("--m", type=complex, default=complex(1.3116, 1e-4))
    ap.add_argument("--orient", type=int, nargs=3, default=[45, 31, 1])
    ap.add_argument("--tol", type=float, default=2e-10,
                    help="refinement target: estimated max-column relative error")
    ap.add_argument("--residual-digits", type=int, default=7,
                    help="int8 digits of the refinement residual (0: FP64 DMMA GEMM)")
    ap.add_argument("--factor-superblock", type=int, default=4, choices=[1, 2, 3, 4],
                    help="256-column blocks per L D L^T trailing update")
    ap.add_argument("--solve-superblock", type=int, default=4, choices=[1, 2, 3, 4],
                    help="256-row blocks per L D L^T solve update")
    ap.add_argument("--gemm-group-m", type=int, default=16,
                    help="row tiles per raster group of the tensor-core GEMM")
    ap.add_argument("--tensor-split", type=int, default=1, choices=[0, 1],
                    help="FP32 operand split of the tensor-core GEMMs: 0 = 3xTF32, 1 = 3xFP16 with "
                         "power-of-two row / column scales")
    ap.add_argument("--gemm-pairs", type=int, default=1, choices=[0, 1],
                    help="FP16-part tensor-core GEMM on CTA pairs (1, cta_group::2, 256-row tiles) or one CTA "
                         "per 128-row tile (0)")
    ap.add_argument("--option", action="append", default=[], metavar="NAME=VALUE",
                    help="any other bem_ctx_set_option switch (repeatable), e.g. residual_pace_epoch=16")
    ap.add_argument("--no-factor-cache", action="store_true",
                    help="free the FP32 factors and digit planes after every step instead of reusing them")
    ap.add_argument("--no-fp64", action="store_true")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-cpu", action="store_true")
    ap.add_argument("--config", default="c3", choices=["c1", "c2", "c3", "c4", "c5", "gemm"],
                    help="c3: the metric's workload; c1, c2, c4, c5: the other configurations; gemm: the FP32 "
                         "tensor-core GEMM alone at the L D L^T trailing-update shape")
    ap.add_argument("--gemm-n", type=int, default=12288, help="--config gemm: rows of C (complex)")
    ap.add_argument("--gemm-ncol", type=int, default=2790, help="--config gemm --gemm-shape solve: columns of C")
    ap.add_argument("--gemm-k", type=int, default=512,
                    help="--config gemm: K (complex), 256 per diagonal block of a super-block")
    ap.add_argument("--gemm-shape", default="factor", choices=["factor", "solve"],
                    help="--config gemm: factor: square row-major C -= A B (B row-major); solve: C (n x 2790, "
                         "column-major, --gemm-ncol) -= A B with B column-major, the multi-RHS solve's update")
    return ap.parse_args()


def extra_options(a):
    out = {}
    for kv in a.option:
        name, _, value = kv.partition("=")
        out[name.strip()] = int(value)
    return out


def workload(a, n):
    return {"workload": f"icosphere ref {a.ref} (2N={n}), ka={a.ka:g}, m={a.m.real:g}+{a.m.imag:g}i, "
                        f"quad 7, {a.orient[0]}x{a.orient[1]}x{a.orient[2]} orientations x 2 pol",
            "unknowns": n, "rhs": 2 * a.orient[0] * a.orient[1] * a.orient[2],
            "l2_policy": "inputs larger than L2 (Z is 16 n^2 bytes)"}


# ---------------------------------------------------------------- CPU baseline
# The reference's CPU dense path (python/bem_core.py: assemble_pmchwt :1032,
# lu_factor / lu_solve :1637 / :1713, the far field of
# orientation_average_mueller_batched :1606) restated by the oracle and timed
# on samples scaled by operation counts (oracle/cpu_dense_path.py).  At
# 2N = 61440 one sample is ~5 s of CPU work; the full path would take hours.
def c3_sample_kw(ref):
    import bem_b200 as bb
    vs, ts = bb.icosphere(1.0, min(ref, 3))
    return dict(rows=2, n_lu=4096, n_ff=1, ff_dirs=19, sing_mesh=(vs, ts))


def cpu_dense_path(verts, tris, ka, m, n_orient, ntheta=181, reps=1, **sample):
    """Median over `reps` of the sampled CPU reference path; returns the dict of
    oracle.cpu_dense_path.time_dense_path with the medians."""
    from oracle.cpu_dense_path import time_dense_path
    runs = [time_dense_path(verts, tris, ka, m, n_orient, ntheta, seed=i, **sample) for i in range(reps)]
    out = dict(runs[-1])
    for k in ("assembly", "lu", "solve", "farfield", "total", "solve_only"):
        if k in out:
            out[k] = statistics.median(r[k] for r in runs)
    out["description"] += f" (median of {reps})" if reps > 1 else ""
    return out


# ---------------------------------------------------------------- clocks
class ClockSampler:
    def __init__(self, index):
        self.f = tempfile.NamedTemporaryFile("w+", suffix=".csv", delete=False)
        q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")
        try:
            self.p = subprocess.Popen(["nvidia-smi", f"--id={index}", f"--query-gpu={q}",
                                       "--format=csv,noheader,nounits", "-lms", "200"],
                                      stdout=self.f, stderr=subprocess.DEVNULL)
        except Exception:
            self.p = None

    def stop(self):
        if self.p is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.p.terminate()
        try:
            self.p.wait(timeout=5)
        except Exception:
            self.p.kill()
        self.f.flush()
        self.f.seek(0)
        rows = [r.split(",") for r in self.f.read().strip().splitlines() if r.strip()]
        sm, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for r in rows:
            r = [x.strip() for x in r]
            try:
                sm.append(float(r[1]))
                mx = float(r[2])
                pw = float(r[3])
            except (ValueError, IndexError):
                continue
            for nm, v in zip(names, r[5:9]):
                if v.lower().startswith("active"):
                    reasons.add(nm)
        load = [s for s in sm if mx and s > 0.3 * mx] or sm
        return {"sm_mhz": statistics.median(load) if load else None, "sm_max_mhz": mx,
                "reasons": sorted(reasons), "samples": len(sm)}


def peaks():
    p = os.path.join(REPO, "MEASURED_PEAKS.json")
    try:
        with open(p) as f:
            d = json.load(f)
        return d, "measured"
    except Exception:
        return {"hbm_gbs": 6650.0, "bf16_tflops": 1590.0, "bf16_tflops_sustained": 1400.0}, "fallback"


# ---------------------------------------------------------------- reference arm
def run_reference(a):
    """The reference's CPU dense path on this host's cores: each step one
    bounded sample of the workload (oracle/cpu_dense_path.py), scaled to the
    full size.  value: the solve (LU + the 2790-column solves), the metric's
    scope; e2e: assembly + solve + far field, the scope of this library's e2e
    line."""
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    import bem_b200 as bb
    verts, tris = bb.icosphere(1.0, a.ref)
    no = a.orient[0] * a.orient[1] * a.orient[2]
    n = 2 * _n_rwg_ico(a.ref)
    kw = c3_sample_kw(a.ref)
    vals, tots, last = [], [], None
    for i in range(a.warmup + a.steps):
        from oracle.cpu_dense_path import time_dense_path
        r = time_dense_path(verts, tris, a.ka, a.m, no, 181, seed=i, **kw)
        if i >= a.warmup:
            vals.append(r["solve_only"])
            tots.append(r["total"])
            last = r
    val, tot = statistics.median(vals), statistics.median(tots)
    line = {"impl": "reference", "metric": METRIC, "value": val, "unit": "s/solve",
            "n_gpus": a.gpus, "steps": a.steps, "warmup": a.warmup, "ms_per_step": val * 1e3,
            "higher_is_better": False, "scaling": "strong", "vs_baseline": None,
            "dtype": "complex128", "data": "synthetic (generated icosphere mesh and plane waves)",
            "config": workload(a, n),
            "extrapolated": "each step times a sample of every phase and scales it by operation counts",
            "phases_s": {k: last[k] for k in ("assembly", "lu", "solve", "farfield")},
            "cpu_baseline": {"value": val, "unit": "s/solve", "cores": last["cores"], "kind": "port",
                             "sample": last["description"]},
            "e2e": {"value": tot, "unit": "s/solve", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0,
                    "scope": "assembly + LU + solves + far field / Mueller (sampled, scaled)"}}
    print(json.dumps(line), flush=True)


# ---------------------------------------------------------------- cuSOLVER arm
def run_cusolver(a):
    import ctypes as C

    import torch

    import bem_b200 as bb

    if int(os.environ.get("RANK", "0")) != 0:
        return
    lib = C.CDLL(os.path.join(REPO, "baseline", "lib", "libcs_lu.so"))
    lib.cs_lu_solve.restype = C.c_int
    lib.cs_lu_solve.argtypes = [C.c_void_p, C.c_void_p, C.c_int64, C.c_void_p, C.c_int64, C.c_int64]
    torch.cuda.set_device(0)
    ctx = bb.Context(0)
    stream = torch.cuda.current_stream(0)

    def cs_solve(Z, X):
        # X: (nrhs, n) row-major = column-major n x nrhs, ldb = n
        rc = lib.cs_lu_solve(C.c_void_p(stream.cuda_stream), C.c_void_p(Z.data_ptr()), Z.shape[0],
                             C.c_void_p(X.data_ptr()), X.shape[1], X.shape[0])
        if rc != 0:
            raise RuntimeError(f"cs_lu_solve returned {rc}")

    verts, tris = bb.icosphere(1.0, a.ref)
    kx, ki, ee, ei = bb.physics(a.ka, a.m)
    g = bb.Geometry(ctx, verts, tris, 7)
    n = g.n
    RT, _ = bb.generate_orientations(*a.orient, sort_nearest=True)
    B = bb.rhs_planewave_dev(g, kx, ee, RT)
    nrhs = B.shape[0]
    # warm-up: library load and handles on a small well-conditioned system
    gen = torch.Generator(device="cuda:0").manual_seed(0)
    Zs = None
    for _ in range(a.warmup):
        Zs = torch.randn((2048, 2048), dtype=torch.complex128, device="cuda:0", generator=gen)
        Zs += 2048 * torch.eye(2048, dtype=torch.complex128, device="cuda:0")
        cs_solve(Zs, torch.randn((8, 2048), dtype=torch.complex128, device="cuda:0", generator=gen))
    del Zs
    Z = torch.empty((n, n), dtype=torch.complex128, device="cuda:0")
    X = torch.empty_like(B)
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)

    def timed(fn):
        torch.cuda.synchronize(0)
        ev0.record(stream)
        out = fn()
        ev1.record(stream)
        torch.cuda.synchronize(0)
        return ev0.elapsed_time(ev1) / 1e3, out

    sampler = ClockSampler(0)
    t_cs = []
    for _ in range(a.steps):
        bb.assemble_pmchwt_dev(g, kx, ki, ee, ei, Z=Z)          # getrf overwrites Z
        X.copy_(B)
        t_cs.append(timed(lambda: cs_solve(Z, X))[0])
    # this library on the same Z and right-hand sides, under the same clocks
    bb.assemble_pmchwt_dev(g, kx, ki, ee, ei, Z=Z)
    bb.set_residual_digits(ctx, a.residual_digits)
    X32 = torch.empty_like(B)

    def fp32_step():
        lu = bb.LU(ctx, Z, bb.PREC_FP32_REFINE)
        lu.solve(B, X=X32, tol=a.tol, max_iter=12, raise_noconv=False)
        lu.close()

    fp32_step()
    t32, _ = timed(fp32_step)

    def fp64_step():
        lu = bb.LU(ctx, Z, bb.PREC_FP64)                          # factors Z in place
        X64, _ = lu.solve(B)
        lu.close()
        return X64

    ctx.profile(True)
    t64, X64 = timed(fp64_step)
    fp64_classes = {k: {"launches": v[0], "s": v[1] / 1e3, "tflops": v[2] / max(v[1], 1e-9) / 1e9}
                    for k, v in ctx.profile_read().items() if v[0] > 0}
    ctx.profile(False)
    clocks = sampler.stop()

    def rel(U, V):
        return float(((U - V).abs().pow(2).sum(dim=1).sqrt() / V.abs().pow(2).sum(dim=1).sqrt()).max().item())

    val = statistics.median(t_cs)
    flops = 8.0 * n ** 3 / 3.0 + 8.0 * n * n * nrhs
    line = {"impl": "cusolver", "metric": METRIC, "value": val, "unit": "s/solve", "n_gpus": 1,
            "steps": a.steps, "warmup": a.warmup, "ms_per_step": val * 1e3, "higher_is_better": False,
            "scaling": "strong", "vs_baseline": None, "dtype": "complex128",
            "data": "synthetic (generated icosphere mesh and plane waves)", "config": workload(a, n),
            "library": "cuSOLVER (CUDA toolkit) cusolverDnXgetrf + cusolverDnXgetrs(OP_T), FP64",
            "step_times_s": t_cs,
            "fp64_tflops": flops / val / 1e12, "fp64_frac_of_37tfs": flops / val / 1e12 / FP64_PEAK_TFS,
            "bem_fp64_s_per_solve": t64, "bem_fp64_classes": fp64_classes, "bem_fp32_refine_s_per_solve": t32,
            "speedup_fp32_refine_vs_cusolver": val / t32, "speedup_bem_fp64_vs_cusolver": val / t64,
            "max_rel_err_cusolver_vs_bem_fp64": rel(X, X64),
            "max_rel_err_fp32_refine_vs_cusolver": rel(X32, X), "clocks": clocks}
    print(json.dumps(line), flush=True)
    del Z, X, X32, X64, B
    g.close()
    ctx.close()


def _n_rwg_ico(ref):
    # closed icosphere: E = 30 * 4^ref interior edges
    return 30 * 4 ** ref


# ---------------------------------------------------------------- our arm
def run_bem(a):
    import numpy as np
    import torch
    import torch.distributed as dist

    import bem_b200 as bb

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if world > 1:
        dist.init_process_group("nccl", timeout=__import__("datetime").timedelta(seconds=600))
    torch.cuda.set_device(local)
    ctx = bb.Context(local)
    stream = torch.cuda.current_stream(local)

    def barrier():
        torch.cuda.synchronize(local)
        if world > 1:
            dist.barrier()

    verts, tris = bb.icosphere(1.0, a.ref)
    kx, ki, ee, ei = bb.physics(a.ka, a.m)
    g = bb.Geometry(ctx, verts, tris, 7)
    n = g.n
    RT, w = bb.generate_orientations(*a.orient, sort_nearest=True)
    no_all = len(w)
    # strong scaling over right-hand sides: every rank factors its own copy,
    # rank r solves its contiguous slice of the orientations
    o0, o1 = rank * no_all // world, (rank + 1) * no_all // world
    RTr, wr = RT[o0:o1], w[o0:o1]
    nrhs = 2 * len(wr)

    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    ctx.profile(True)
    ev0.record(stream)
    Z = bb.assemble_pmchwt_dev(g, kx, ki, ee, ei)
    ev1.record(stream)
    torch.cuda.synchronize(local)
    t_asm = ev0.elapsed_time(ev1) / 1e3
    prof_asm = ctx.profile_read()["assembly"]
    ctx.profile(False)
    B = bb.rhs_planewave_dev(g, kx, ee, RTr)

    # FP64 comparator (also the oracle of the error check)
    t64, X64, st64 = None, None, None
    if not a.no_fp64:
        Zc = Z.clone()
        barrier()
        ev0.record(stream)
        lu64 = bb.LU(ctx, Zc, bb.PREC_FP64)
        X64, st64 = lu64.solve(B)
        ev1.record(stream)
        torch.cuda.synchronize(local)
        t64 = ev0.elapsed_time(ev1) / 1e3
        lu64.close()
        del lu64, Zc
        torch.cuda.empty_cache()

    bb.set_residual_digits(ctx, a.residual_digits)
    bb.set_option(ctx, "factor_superblock", a.factor_superblock)
    bb.set_option(ctx, "solve_superblock", a.solve_superblock)
    bb.set_option(ctx, "gemm_group_m", a.gemm_group_m)
    bb.set_option(ctx, "tensor_split", a.tensor_split)
    bb.set_option(ctx, "gemm_pairs", a.gemm_pairs)
    for name, value in extra_options(a).items():
        bb.set_option(ctx, name, value)
    # a loop of solves of one size keeps its factor / digit-plane memory
    bb.set_option(ctx, "cache_factor_memory", 0 if a.no_factor_cache else 1)
    X = torch.empty_like(B)
    def step():
        lu = bb.LU(ctx, Z, bb.PREC_FP32_REFINE)
        Xs, st = lu.solve(B, X=X, tol=a.tol, max_iter=12, raise_noconv=False)
        lu.close()
        return st

    for _ in range(a.warmup):
        step()
    # the K timed steps: one region bracketed by barrier + synchronize, with
    # per-step events inside for the spread
    sampler = ClockSampler(local)
    ctx.profile(True)
    launches0 = ctx.launches
    times, stats = [], []
    evs = [torch.cuda.Event(enable_timing=True) for _ in range(a.steps + 1)]
    barrier()
    evs[0].record(stream)
    for i in range(a.steps):
        stats.append(step())
        evs[i + 1].record(stream)
    barrier()
    prof = ctx.profile_read()
    ctx.profile(False)
    clocks = sampler.stop()
    bb.set_option(ctx, "cache_factor_memory", 0)
    launches = ctx.launches - launches0
    times = [evs[i].elapsed_time(evs[i + 1]) / 1e3 for i in range(a.steps)]
    t_total = evs[0].elapsed_time(evs[-1]) / 1e3
    tt = torch.tensor([t_total / a.steps, t64 or 0.0, t_asm, max(times)], device=f"cuda:{local}",
                      dtype=torch.float64)
    if world > 1:
        dist.all_reduce(tt, op=dist.ReduceOp.MAX)
    t_step, t64m, t_asm, t_max = tt.tolist()

    err = None
    if X64 is not None:
        d = (X - X64).abs().pow(2).sum(dim=1).sqrt() / X64.abs().pow(2).sum(dim=1).sqrt()
        err = float(d.max().item())
        if world > 1:
            e = torch.tensor([err], device=f"cuda:{local}", dtype=torch.float64)
            dist.all_reduce(e, op=dist.ReduceOp.MAX)
            err = float(e.item())

    # the metric's second bar: the orientation-averaged Mueller matrix of the
    # FP32 + refinement solution against that of the FP64 solution
    merr = None
    if X64 is not None:
        from bem_b200.parallel import allreduce_sum
        M32 = bb.mueller_from_solutions_dev(g, X, RTr, wr, kx, ee, ntheta=181)
        M64 = bb.mueller_from_solutions_dev(g, X64, RTr, wr, kx, ee, ntheta=181)
        if world > 1:
            M32 = allreduce_sum(M32, device=f"cuda:{local}").reshape(M32.shape)
            M64 = allreduce_sum(M64, device=f"cuda:{local}").reshape(M64.shape)
        merr = {"rel_fro": float(np.linalg.norm(M32 - M64) / np.linalg.norm(M64)),
                "max_abs_over_max_M11": float(np.abs(M32 - M64).max() / np.abs(M64[0, 0]).max()),
                "M11_max_rel": float((np.abs(M32[0, 0] - M64[0, 0]) / np.abs(M64[0, 0])).max())}

    # dominant kernel of the timed steps -> roofline
    pk, basis = peaks()
    dom = max(prof.items(), key=lambda kv: kv[1][1])
    name, (nl, ms, fl, by) = dom
    ms_launch = ms / max(nl, 1)
    achieved = fl / max(nl, 1) / (ms_launch / 1e3) / 1e12
    # the kernels run inside a seconds-long step under the power cap: the
    # sustained bf16 figure is the denominator
    bf16 = pk.get("bf16_tflops_sustained", pk["bf16_tflops"])
    if name in ("lu_update", "solve_update") and a.tensor_split == 1:
        peak = bf16 / 3.0
        pbasis = (f"complex flops at 3xFP16: {basis} sustained bf16 {bf16} TF/s (fp16 rate = bf16 rate) "
                  f"/ 3 (split terms)")
    elif name in ("lu_update", "solve_update"):
        peak = bf16 / 2.0 / 3.0
        pbasis = (f"complex flops at 3xTF32: {basis} sustained bf16 {bf16} TF/s / 2 (tf32 rate) "
                  f"/ 3 (split terms)")
    elif name == "residual" and a.residual_digits > 0:
        peak = 2.0 * bf16
        pbasis = (f"int8 tensor ops (digit-pair GEMMs): 2 x {basis} sustained bf16 {bf16} TF/s "
                  f"(B200 dense int8 rate = 2 x bf16)")
    else:
        peak = FP64_PEAK_TFS
        pbasis = ("FP64: 37.0 TF/s measured on B200 (cuBLAS ZGEMM 8192^3; DFMA and m8n8k4 DMMA "
                  "throughput probes 36-37 TF/s); MEASURED_PEAKS.json has no FP64 figure")
    traffic, tbasis = None, None
    if name in TRAFFIC_MODEL and (name != "residual" or a.residual_digits > 0):
        kind, f, tbasis = TRAFFIC_MODEL[name]
        if kind == "per_byte":
            traffic = f * by / max(nl, 1)
        else:
            pair_ops = 2.0 * n * (2.0 * nrhs) * (2.0 * n)
            traffic = f * (fl / max(nl, 1)) / pair_ops
    roof = {"bound": "tensor", "kernel": name, "achieved": achieved, "peak": peak, "unit": "TFLOP/s",
            "frac": achieved / peak, "traffic": traffic, "traffic_unit": "bytes per launch",
            "traffic_basis": tbasis, "algorithmic_bytes_per_launch": by / max(nl, 1),
            "launches": nl, "ms_per_launch": ms_launch, "peak_basis": pbasis,
            "share": {k: v[1] / max(1e-9, sum(x[1] for x in prof.values())) for k, v in prof.items()}}

    # free the step buffers before the end-to-end pipeline
    del Z, B, X, X64
    torch.cuda.empty_cache()
    e2e = None
    if not a.no_e2e:
        from bem_b200.parallel import allreduce_max, allreduce_sum
        # N > 1: every rank runs the pipeline on its orientation range
        # (--orient-range, main.cpp:118-121) and one all-reduce sums the
        # partial Mueller matrices (the cluster_bem.py JSON sum).  Every rank
        # takes the same collectives whether or not its pipeline failed.
        dev = f"cuda:{local}"
        # two calls: the first allocates the pipeline's device buffers (kept
        # by cache_factor_memory, as for the timed steps), the second is the
        # timed one; the first call's time is reported as cold_value
        bb.set_option(ctx, "cache_factor_memory", 1)
        walls = []
        err_e2e, info = None, None
        M = np.zeros((4, 4, 181))
        for call in range(2):
            barrier()
            t0 = time.perf_counter()
            try:
                M, info = bb.dense_run(ctx, verts, tris, a.ka, a.m, orient=tuple(a.orient), ntheta=181,
                                       precision=bb.PREC_FP32_REFINE, refine_tol=a.tol, max_refine=12,
                                       orient_range=(o0, o1) if world > 1 else None)
            except bb.BemError as ex:
                err_e2e = str(ex)
                M = np.zeros((4, 4, 181))
            if world > 1:
                M = allreduce_sum(M, device=dev).reshape(M.shape)
            walls.append(allreduce_max(time.perf_counter() - t0, device=dev))
        bb.set_option(ctx, "cache_factor_memory", 0)
        t_e2e = walls[-1]
        failed = allreduce_max(1.0 if err_e2e else 0.0, device=dev) > 0
        if failed:
            e2e = {"value": None, "unit": "s/solve", "error": err_e2e or "the pipeline failed on another rank"}
        else:
            h2d = verts.nbytes + tris.astype(np.int32).nbytes + 9 * 8 * no_all + 8 * no_all
            e2e = {"value": t_e2e, "unit": "s/solve", "h2d_bytes_per_step": int(h2d),
                   "d2h_bytes_per_step": int(M.nbytes), "cold_value": walls[0],
                   "scope": "bem_dense_run: host mesh -> assembly, FP32 LU + refinement, far field -> host Mueller"
                            + (f"; orientations split over {world} ranks, Mueller all-reduced" if world > 1 else ""),
                   "t_assembly_s": info["t_assembly_s"], "t_solve_s": info["t_solve_s"],
                   "t_farfield_s": info["t_farfield_s"], "t_setup_s": info["t_setup_s"],
                   "t_release_s": info["t_release_s"], "t_total_s": info["t_total_s"],
                   "refine": info["stats"]["iterations"]}

    cpu = None
    if rank == 0 and world == 1 and not a.no_cpu:
        r = cpu_dense_path(verts, tris, a.ka, a.m, no_all, 181, reps=3, **c3_sample_kw(a.ref))
        cpu = {"value": r["solve_only"], "unit": "s/solve", "cores": r["cores"], "kind": "port",
               "sample": r["description"], "e2e_value": r["total"],
               "phases_s": {k: r[k] for k in ("assembly", "lu", "solve", "farfield")}}

    if rank == 0:
        its = [s["iterations"] for s in stats]
        line = {"metric": METRIC, "value": t_step, "unit": "s/solve", "n_gpus": world,
                "steps": a.steps, "warmup": a.warmup, "ms_per_step": t_step * 1e3,
                "higher_is_better": False, "scaling": "strong", "vs_baseline": None,
                "dtype": ("complex64 factors (3xFP16, scaled) + complex128 refinement" if a.tensor_split == 1 else
                          "complex64 factors (3xTF32) + complex128 refinement") +
                         (f" (int8 Ozaki residual, {a.residual_digits} digits)" if a.residual_digits else
                          " (FP64 DMMA residual)"),
                "data": "synthetic (generated icosphere mesh and plane waves)",
                "config": {**workload(a, n), "parallelism": f"rhs-split x{world}" if world > 1 else "single",
                           "operand_split": ("3xFP16 with power-of-two row / column scales (tensor_split 1)"
                                             if a.tensor_split == 1 else "3xTF32"),
                           "fp32_gemm_tiles": ("256-row CTA-pair tiles (cta_group::2)" if a.gemm_pairs else
                                               "128-row one-CTA tiles"),
                           **({"options": extra_options(a)} if a.option else {}),
                           "factor_memory": ("allocated and freed by every step" if a.no_factor_cache else
                                             "FP32 factors and digit planes allocated once, reused by every step "
                                             "(cache_factor_memory)")},
                "step_times_s": times, "max_step_s": t_max,
                "fp64_s_per_solve": t64m or None,
                "speedup_vs_fp64": (t64m / t_step) if t64m else None,
                "max_rel_err_vs_fp64": err, "refine_iterations": its,
                "refine_update_hist": stats[-1].get("update_hist"),
                "est_rel_err": stats[-1].get("est_rel_error"),
                "verified_rel_err": stats[-1].get("verified_rel_error"),
                "verified_columns": stats[-1].get("verified_columns"),
                "exact_residual_sweeps": stats[-1].get("exact_residual_sweeps"),
                "mueller_err_vs_fp64": merr,
                "t_factor_s": stats[-1]["t_factor_ms"] / 1e3, "t_first_solve_s": stats[-1]["t_solve_ms"] / 1e3,
                "t_refine_s": stats[-1]["t_refine_ms"] / 1e3,
                "converged": all(s["converged"] for s in stats),
                "assembly_s": t_asm,
                "assembly_roofline": {"unit_evals_per_s": prof_asm[2] / 64.0 / max(prof_asm[1], 1e-9) * 1e3},
                "roofline": roof, "cpu_baseline": cpu, "e2e": e2e, "gpu_launches": int(launches),
                "clocks": clocks}
        print(json.dumps(line), flush=True)
    ctx.close()
    if world > 1:
        dist.destroy_process_group()


# ---------------------------------------------------------------- other configurations
CONFIGS = {
    "c1": {"metric": "s per C1 run: icosphere r2 (2N=960), ka=1, m=1.3116, single orientation, 181 angles, FP64",
           "workload": "icosphere ref 2 (2N=960), ka=1, m=1.3116, quad 7, --single (k=z, E=x/y), 181 angles"},
    "c2": {"metric": "s per C2 run: hex prism AR 1.4286 r3 (2N=4608), ka=5, 128 RHS: assembly + FP64 LU + solves + "
                     "far field / Mueller",
           "workload": "hex prism AR=1.4286 ref 3 (2N=4608), ka=5, m=1.3116, quad 7, 8x8x1 orientations x 2 pol"},
    "c4": {"metric": "s per batch of 64 seeded hex prisms (2N 1152 / 4608): assembly + LU + solves + Mueller",
           "workload": "64 hex prisms from seed 0: AR U[0.5,2], ref 2 or 3, ka U[1,5], Re m U[1.3,1.6], "
                       "Im m logU[1e-6,1e-2], 4x4x1 orientations x 2 pol, 181 angles"},
    "c5": {"metric": "s per adjoint gradient at C5: 1926 vertex coordinates + Re/Im m",
           "workload": "icosphere ref 3 (642 vertices, 2N=3840) displaced by a seeded degree<=6 field (RMS 0.05), "
                       "ka=5, m=1.5+0.01i, 8x8x1 orientations, loss sum (M11 - M11_sphere)^2 over 181 angles"},
}


def _ref_gpu_run(args):
    """The reference's own GPU dense path (its sources built by
    oracle/Makefile into oracle/_ref/ref_dense_branch, driven by the same
    consumer program the tests build against this library), and the same
    program built against this library's compat surface: wall times and the
    phase times each reports through write_json."""
    import shutil
    import tempfile
    exe_ref = os.path.join(REPO, "oracle", "_ref", "ref_dense_branch")
    if not os.path.exists(exe_ref):
        return {"unavailable": "oracle/_ref/ref_dense_branch not built (needs the reference sources)"}
    tmp = tempfile.mkdtemp(prefix="bem_refgpu_")
    lib = os.path.join(REPO, "bem-cpp_b200", "lib")
    exe_ours = os.path.join(tmp, "dense_branch")
    r = subprocess.run(["g++", "-O2", "-std=c++17", "-I" + os.path.join(REPO, "include", "bem"),
                        "-I" + os.path.join(REPO, "include"), "-o", exe_ours,
                        os.path.join(REPO, "tests", "compat", "dense_branch.cpp"), "-L" + lib,
                        "-Wl,-rpath," + lib, "-lbem_compat", "-lbemdense"], capture_output=True, text=True)
    if r.returncode != 0:
        return {"unavailable": "compat consumer did not build: " + r.stderr[-200:]}
    out = {}
    for tag, exe in (("reference", exe_ref), ("bem", exe_ours)):
        d = os.path.join(tmp, tag)
        os.makedirs(d)
        t0 = time.perf_counter()
        p = subprocess.run([exe, d] + args, capture_output=True, text=True, timeout=1200)
        wall = time.perf_counter() - t0
        if p.returncode != 0:
            out[tag] = {"rc": p.returncode, "stderr": p.stderr[-300:]}
            continue
        ph = [ln for ln in p.stdout.splitlines() if ln.startswith("phase seconds:")]
        words = ph[-1].split()[2:] if ph else []
        out[tag] = {"wall_s": wall}
        out[tag].update({words[i].replace("+", "_") + "_s": float(words[i + 1]) for i in range(0, len(words) - 1, 2)})
    if all("wall_s" in out.get(k, {}) for k in ("reference", "bem")):
        import numpy as np
        with open(os.path.join(tmp, "reference", "orient.json")) as f:
            mr = np.array(json.load(f)["mueller"])
        with open(os.path.join(tmp, "bem", "orient.json")) as f:
            mb = np.array(json.load(f)["mueller"])
        out["mueller_rel_diff"] = float(np.linalg.norm(mb - mr) / np.linalg.norm(mr))
    shutil.rmtree(tmp, ignore_errors=True)
    out["program"] = ("tests/compat/dense_branch.cpp (the dense branch's calls: assemble_pmchwt, lu_factorize_cuda + "
                      "lu_solve_cuda, lu_solve_full, far field, write_json) with arguments " + " ".join(args))
    return out


def _clocked(fn, steps, warmup, stream, local=0):
    """Runs fn warmup + steps times; returns (per-step device seconds over the
    timed steps, results of the timed steps, clocks)."""
    import torch
    for _ in range(warmup):
        fn()
    sampler = ClockSampler(local)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    torch.cuda.synchronize(local)
    e0.record(stream)
    res = [fn() for _ in range(steps)]
    e1.record(stream)
    torch.cuda.synchronize(local)
    clocks = sampler.stop()
    return e0.elapsed_time(e1) / 1e3 / steps, res, clocks


def _roofline_from_profile(prof, bf16):
    """Dominant kernel class of a profiled region: achieved algorithmic rate
    against its peak (FP64 classes 37 TF/s, tensor-core FP32 updates 3xFP16 of
    the sustained bf16 figure, the int8 residual 2 x bf16, assembly / far field
    in counted units per second with no peak)."""
    if not prof:
        return None
    name, (nl, ms, fl, by) = max(prof.items(), key=lambda kv: kv[1][1])
    if nl == 0 or ms <= 0:
        return None
    rate = fl / (ms / 1e3)
    share = {k: v[1] / max(1e-9, sum(x[1] for x in prof.values())) for k, v in prof.items()}
    if name in ("assembly", "farfield"):
        unit = 64.0 if name == "assembly" else 110.0
        return {"bound": "fp64-simt", "kernel": name, "achieved": rate / unit, "peak": None,
                "unit": "quadrature-pair evaluations/s" if name == "assembly" else "far-field point terms/s",
                "frac": None, "traffic": None, "launches": nl, "ms_per_launch": ms / nl, "share": share}
    return {"bound": "tensor", "kernel": name, "achieved": rate / 1e12, "peak": None, "unit": "TFLOP/s",
            "frac": None, "traffic": None, "launches": nl, "ms_per_launch": ms / nl, "share": share,
            "peak_basis": f"FP64 37 TF/s; 3xFP16 {bf16 / 3:.0f} TF/s; int8 {2 * bf16:.0f} TOPS"}


def run_gemm(a):
    """The FP32 tensor-core GEMM of the factorisation alone: C -= A B with
    complex64 A (n x K), B (K x n) and a square row-major C (n x n), the
    shape of an L D L^T super-block trailing update (K = 256 per diagonal
    block: --gemm-k 1024 for the default four-block super-block, 512 by
    default here), timed with CUDA events over the steps (C larger than L2
    for n >= 4096)."""
    import torch

    import bem_b200 as bb

    if int(os.environ.get("RANK", "0")) != 0:
        return
    torch.cuda.set_device(0)
    stream = torch.cuda.current_stream(0)
    ctx = bb.Context(0)
    bb.set_option(ctx, "tensor_split", a.tensor_split)
    bb.set_option(ctx, "gemm_pairs", a.gemm_pairs)
    bb.set_option(ctx, "gemm_group_m", a.gemm_group_m)
    for name, value in extra_options(a).items():
        bb.set_option(ctx, name, value)
    n, K = a.gemm_n, a.gemm_k
    solve = a.gemm_shape == "solve"
    ncol = a.gemm_ncol if solve else n
    g = torch.Generator(device="cuda:0").manual_seed(0)
    A = torch.randn((n, K), dtype=torch.complex64, device="cuda:0", generator=g)
    # solve: B given as its transpose (ncol x K row-major), C stored as (ncol x n) row-major
    B = torch.randn((ncol, K) if solve else (K, ncol), dtype=torch.complex64, device="cuda:0", generator=g)
    C = torch.zeros((ncol, n) if solve else (n, ncol), dtype=torch.complex64, device="cuda:0")
    launches0 = ctx.launches
    t, _, clocks = _clocked(lambda: bb.cgemm_tf32x3(ctx, A, B, C, b_rowmajor=not solve, c_colmajor=solve),
                            a.steps, a.warmup, stream)
    pk, basis = peaks()
    bf16 = pk.get("bf16_tflops_sustained", pk["bf16_tflops"])
    flops = 8.0 * n * ncol * K
    peak = bf16 / 3.0 if a.tensor_split == 1 else bf16 / 6.0
    line = {"metric": f"TFLOP/s of the FP32 tensor-core GEMM, C -= A B, {n} x {ncol} x {K} complex64",
            "value": flops / t / 1e12, "unit": "TFLOP/s", "n_gpus": 1, "steps": a.steps, "warmup": a.warmup,
            "ms_per_step": t * 1e3, "higher_is_better": True, "scaling": "strong", "vs_baseline": None,
            "dtype": "complex64 (3xFP16 parts)" if a.tensor_split == 1 else "complex64 (3xTF32 parts)",
            "data": "synthetic (seeded normal operands)",
            "config": {"workload": (f"C {n} x {ncol} column-major, A {n} x {K} row-major, B {K} x {ncol} column-major "
                                    "(the multi-RHS solve's update)" if solve else
                                    f"C {n} x {n} row-major, A {n} x {K}, B {K} x {n} row-major (the factorisation's "
                                    "trailing update)"),
                       "tiles": "256-row CTA pairs" if a.gemm_pairs else "128-row one-CTA tiles",
                       "l2_policy": "C larger than L2" if 8 * n * ncol > 126e6 else "C within L2"},
            "roofline": {"bound": "tensor", "achieved": flops / t / 1e12, "peak": peak, "unit": "TFLOP/s",
                         "frac": flops / t / 1e12 / peak, "traffic": None,
                         "peak_basis": f"{basis} sustained bf16 {bf16} TF/s / 3 split terms"
                                       + ("" if a.tensor_split == 1 else " / 2 (tf32)")},
            "gpu_launches": int(ctx.launches - launches0), "clocks": clocks}
    print(json.dumps(line), flush=True)
    ctx.close()


def run_config(a):
    import numpy as np
    import torch

    import bem_b200 as bb

    if a.config == "gemm":
        return run_gemm(a)
    if int(os.environ.get("RANK", "0")) != 0:
        return
    c = CONFIGS[a.config]
    torch.cuda.set_device(0)
    stream = torch.cuda.current_stream(0)
    pk, basis = peaks()
    bf16 = pk.get("bf16_tflops_sustained", pk["bf16_tflops"])
    line = {"metric": c["metric"], "unit": "s", "n_gpus": 1, "steps": a.steps, "warmup": a.warmup,
            "higher_is_better": False, "scaling": "strong", "vs_baseline": None,
            "data": "synthetic (generated meshes and plane waves)", "config": {"workload": c["workload"]}}
    if a.impl == "reference":
        line["impl"] = "reference"
    ctx = None if a.impl == "reference" else bb.Context(0)

    def cpu_leg(reps):
        if a.config == "c1":
            v, t = bb.icosphere(1.0, 2)
            r = cpu_dense_path(v, t, 1.0, 1.3116, 1, 181, reps=reps)
            return r, r["total"]
        if a.config == "c2":
            # the whole path at full size (every assembly row, in blocks; the
            # full LU, solves and far field): a few minutes of CPU
            v, t = bb.hex_prism(1.4286, 3)
            r = cpu_dense_path(v, t, 5.0, 1.3116, 64, 181, reps=reps, rows="blocks")
            return r, r["total"]
        if a.config == "c4":
            parts = bb.c4_particles(0, 64)
            tot, descs, cores = 0.0, [], 1
            for ref in (2, 3):
                sel = [p for p in parts if p["meta"]["refinements"] == ref]
                p0 = sel[0]
                r = cpu_dense_path(p0["verts"], p0["tris"], p0["ka"], p0["m"], 16, 181, reps=reps,
                                   rows=None if ref == 2 else 48, n_ff=None if ref == 2 else 4)
                tot += r["total"] * len(sel)
                cores = r["cores"]
                descs.append(f"{len(sel)} x (2N={r['n']}: {r['description']})")
            return {"total": tot, "description": "; ".join(descs), "cores": cores}, tot
        # c5: the reference has no gradient code; a CPU user would difference
        # the forward path, two forward runs per coordinate and per Re/Im m
        v, t = bb.c5_mesh(11, refinements=3, rms=0.05)
        r = cpu_dense_path(v, t, 5.0, complex(1.5, 0.01), 64, 181, reps=reps, rows=24, n_ff=4)
        ncoord = 3 * len(v) + 2
        r = dict(r)
        r["description"] = (f"central differences of the forward path: 2 x {ncoord} forward runs of "
                            + r["description"])
        return r, 2 * ncoord * r["total"]

    if a.impl == "reference":
        vals = []
        for i in range(a.warmup + a.steps):
            r, v = cpu_leg(1)
            if i >= a.warmup:
                vals.append(v)
        val = statistics.median(vals)
        line.update({"value": val, "ms_per_step": val * 1e3, "dtype": "complex128",
                     "cpu_baseline": {"value": val, "unit": "s", "cores": r["cores"], "kind": "port",
                                      "sample": r["description"]},
                     "e2e": {"value": r.get("total", val), "unit": "s", "h2d_bytes_per_step": 0,
                             "d2h_bytes_per_step": 0}})
        if a.config in ("c1", "c2"):
            args = (["2", "1.0", "1.3116", "0", "1", "1", "1", "181"] if a.config == "c1" else
                    ["3", "5.0", "1.3116", "0", "8", "8", "1", "181", "1.4286"])
            line["reference_gpu"] = _ref_gpu_run(args)
        print(json.dumps(line), flush=True)
        return

    launches0 = ctx.launches
    if a.config in ("c1", "c2"):
        if a.config == "c1":
            v, t = bb.icosphere(1.0, 2)
            ka, m, RT, w = 1.0, 1.3116, np.eye(3)[None], np.array([1.0])
        else:
            v, t = bb.hex_prism(1.4286, 3)
            ka, m = 5.0, 1.3116
            RT, w = bb.generate_orientations(8, 8, 1)
        g = bb.Geometry(ctx, v, t, 7)
        kx, ki, ee, ei = bb.physics(ka, m)
        Z = torch.empty((g.n, g.n), dtype=torch.complex128, device="cuda:0")
        B = bb.rhs_planewave_dev(g, kx, ee, RT)
        X = torch.empty_like(B)

        def step64():
            bb.assemble_pmchwt_dev(g, kx, ki, ee, ei, Z=Z)
            lu = bb.LU(ctx, Z, bb.PREC_FP64)
            lu.solve(B, X=X)
            lu.close()
            return bb.mueller_from_solutions_dev(g, X, RT, w, kx, ee, ntheta=181)

        # timed without the per-class events (thousands of small launches at
        # these sizes, where recording them costs time); one more step with
        # them gives the class shares
        t64, Ms, clocks = _clocked(step64, a.steps, a.warmup, stream)
        ctx.profile(True)
        step64()
        prof = ctx.profile_read()
        ctx.profile(False)
        bb.set_option(ctx, "cache_factor_memory", 1)

        def step32():
            bb.assemble_pmchwt_dev(g, kx, ki, ee, ei, Z=Z)
            lu = bb.LU(ctx, Z, bb.PREC_FP32_REFINE)
            _, st = lu.solve(B, X=X, tol=2e-10, max_iter=12, raise_noconv=False)
            lu.close()
            return bb.mueller_from_solutions_dev(g, X, RT, w, kx, ee, ntheta=181), st

        t32, res32, _ = _clocked(step32, a.steps, a.warmup, stream)
        M64, (M32, st32) = Ms[-1], res32[-1]
        # e2e through bem_dense_run (host mesh -> host Mueller), the device
        # buffers kept between calls as in the full-size line (without the
        # cache each call's allocations and frees cost 10-130 ms here)
        walls = []
        for i in range(a.warmup + a.steps):
            t0 = time.perf_counter()
            Mp, info = bb.dense_run(ctx, v, t, ka, m, single=a.config == "c1",
                                    orient=(8, 8, 1), ntheta=181, precision=bb.PREC_FP64)
            if i >= a.warmup:
                walls.append(time.perf_counter() - t0)
        bb.set_option(ctx, "cache_factor_memory", 0)
        h2d = v.nbytes + t.astype(np.int32).nbytes
        line.update({"value": t64, "ms_per_step": t64 * 1e3, "dtype": "complex128",
                     "step": "assembly + FP64 LU + solves + far field / Mueller, device-resident",
                     "fp32_refine_s": t32, "fp32_refine_vs_fp64": t64 / t32,
                     "fp32_refine_mueller_rel_err": float(np.linalg.norm(M32 - M64) / np.linalg.norm(M64)),
                     "fp32_refine_est_rel_err": st32["est_rel_error"],
                     "e2e": {"value": statistics.median(walls), "unit": "s", "h2d_bytes_per_step": int(h2d),
                             "d2h_bytes_per_step": int(Mp.nbytes),
                             "scope": "bem_dense_run FP64, device buffers kept between calls"},
                     "e2e_mueller_rel_diff": float(np.linalg.norm(Mp - M64) / np.linalg.norm(M64)),
                     "roofline": _roofline_from_profile(prof, bf16), "clocks": clocks})
    elif a.config == "c4":
        p32 = bb.c4_particles(0, 64, precision=bb.PREC_FP32_REFINE)
        p64 = bb.c4_particles(0, 64, precision=bb.PREC_FP64)
        bb.batch_run(ctx, p64[:2])  # library load and first allocations
        walls, clocks = {}, None
        res = {}
        for tag, parts in (("fp64", p64), ("fp32", p32)):
            ws = []
            for i in range(a.warmup + a.steps):
                sampler = ClockSampler(0) if (tag == "fp64" and i == a.warmup) else None
                t0 = time.perf_counter()
                out = bb.batch_run(ctx, parts)
                if i >= a.warmup:
                    ws.append(time.perf_counter() - t0)
                if sampler is not None:
                    clocks = sampler.stop()
            walls[tag] = statistics.median(ws)
            res[tag] = out
        errs = [float(np.linalg.norm(r32[0] - r64[0]) / np.linalg.norm(r64[0]))
                for r32, r64 in zip(res["fp32"], res["fp64"])]
        sizes = sorted({r[1]["N"] * 2 for r in res["fp64"]})
        # the value: the FP64 buckets (batched assembly, LU and solves per
        # system size), the faster path at these sizes; FP32 + refinement
        # (one particle at a time) beside it
        line.update({"value": walls["fp64"], "ms_per_step": walls["fp64"] * 1e3,
                     "dtype": "complex128 (FP64 buckets); FP32 + refinement beside it",
                     "fp64_s": walls["fp64"], "fp32_refine_s": walls["fp32"],
                     "fp32_refine_vs_fp64": walls["fp64"] / walls["fp32"],
                     "max_particle_mueller_rel_err_fp32_vs_fp64": max(errs), "sizes_2N": sizes,
                     "counts": {str(n): sum(1 for r in res["fp64"] if 2 * r[1]["N"] == n) for n in sizes},
                     "e2e": {"value": walls["fp64"], "unit": "s",
                             "h2d_bytes_per_step": int(sum(p["verts"].nbytes + p["tris"].nbytes for p in p64)),
                             "d2h_bytes_per_step": int(64 * 16 * 181 * 8),
                             "scope": "bem_batch_run: host meshes -> host Mueller matrices"},
                     "clocks": clocks})
    else:  # c5
        v, t = bb.c5_mesh(11, refinements=3, rms=0.05)
        vs, ts = bb.icosphere(1.0, 3)
        ka, m = 5.0, complex(1.5, 0.01)
        Ms, _ = bb.dense_run(ctx, vs, ts, ka, m, orient=(8, 8, 1), ntheta=181)
        target = Ms[0, 0].copy()
        walls, clocks = [], None
        for i in range(a.warmup + a.steps):
            sampler = ClockSampler(0) if i == a.warmup else None
            t0 = time.perf_counter()
            lv, gv, _ = bb.adjoint_grad_vertices(ctx, v, t, ka, m, target, orient=(8, 8, 1))
            lm, gm, _ = bb.adjoint_grad(ctx, v, t, ka, m, target, orient=(8, 8, 1))
            if i >= a.warmup:
                walls.append(time.perf_counter() - t0)
            if sampler is not None:
                clocks = sampler.stop()
        val = statistics.median(walls)
        line.update({"value": val, "ms_per_step": val * 1e3, "dtype": "complex128",
                     "step": "bem_adjoint_grad_vertices + bem_adjoint_grad: each one FP64 forward solve, one "
                             "adjoint solve and the contraction kernels",
                     "loss": lv, "grad_m": gm.tolist(), "grad_v_max": float(np.abs(gv).max()),
                     "e2e": {"value": val, "unit": "s", "h2d_bytes_per_step": int(v.nbytes + t.nbytes),
                             "d2h_bytes_per_step": int(gv.nbytes + gm.nbytes),
                             "scope": "host mesh -> host gradients"},
                     "clocks": clocks})
    line["gpu_launches"] = int(ctx.launches - launches0)
    if not a.no_cpu:
        r, v = cpu_leg(3 if a.config == "c1" else 1)
        line["cpu_baseline"] = {"value": v, "unit": "s", "cores": r["cores"], "kind": "port",
                                "sample": r["description"]}
    print(json.dumps(line), flush=True)
    ctx.close()


def main():
    a = parse()
    if a.config != "c3":
        run_config(a)
    elif a.impl == "reference":
        run_reference(a)
    elif a.impl == "cusolver":
        run_cusolver(a)
    else:
        run_bem(a)


if __name__ == "__main__":
    main()
