"""Timing of the reference's CPU dense path on samples (TEST / BASELINE
INFRASTRUCTURE ONLY: used by bench.py's CPU-baseline legs, never by the
product).

The reference's CPU implementation of the dense PMCHWT path is
``python/bem_core.py``: ``assemble_pmchwt`` (bem_core.py:1032, with
``assemble_L_K`` :787 for each medium), ``scipy.linalg.lu_factor`` /
``lu_solve`` (:1637, :1713) and the far field of
``orientation_average_mueller_batched`` (:1606, ``_compute_far_field_vec``
:1265).  That file cannot be shipped with this repository, so the timings
here run the oracle's restatement of it (``bem_oracle``), in the same
arrangement: the assembly in the oracle's ``distance="expanded"`` mode, which
replays bem_core's three half-pair passes with matrix-product distances
(measured in the build container at 2N = 960: 9.9 s against bem_core's
~12 s once numba is compiled), the LU and the solves through the same SciPy
LAPACK calls, the far field with the same per-orientation vectorisation.

Full sizes are out of reach of a CPU at 2N = 61440 (about 11 h of assembly),
so each phase is timed on a sample and scaled by its operation count, and the
result says which:
  * assembly: all source columns for a block of test rows, both media, the
    four half pairs; scaled by 3 N / (4 rows) (the reference computes three
    N x N half-pair passes);
  * Graglia corrections: every triangle (linear in the triangle count), or
    every triangle of a smaller mesh of the same kind, scaled by the count;
  * LU: a seeded complex matrix of order n_lu (LAPACK's cost does not depend
    on the values), scaled by (n / n_lu)^3; the solves likewise by
    (n / n_lu)^2 nrhs / nrhs_lu;
  * far field: n_ff orientations of the full mesh at ff_dirs of the ntheta
    scattering angles, scaled by orientations x angles.
"""
from __future__ import annotations

import os
import time

import numpy as np

from . import bem_oracle as bo


def cpu_model():
    try:
        with open("/proc/cpuinfo") as f:
            for line in f:
                if line.startswith("model name"):
                    return line.split(":", 1)[1].strip()
    except OSError:
        pass
    return "CPU model unknown"


def _sub_half(h, rows):
    return bo.Half(qp=h.qp[rows], f=h.f[rows], div=h.div[rows], jw=h.jw[rows], tri=h.tri[rows],
                   sign=h.sign, free=h.free[rows], coeff=h.coeff[rows])


def time_dense_path(verts, tris, ka, m, n_orient, ntheta=181, rows=None, n_lu=None, n_ff=None,
                    ff_dirs=None, sing_mesh=None, phases=("assembly", "lu", "solve", "farfield"), seed=0):
    """Times the reference's CPU dense path on the mesh (verts, tris) with
    n_orient orientations x 2 polarisations, on samples (rows / n_lu / n_ff
    None: the full size; rows "blocks": every test row, in blocks of 256, for
    sizes whose one-call assembly would not fit the host's memory).  Returns a
    dict of seconds per phase (scaled to the full size), their sum, and a
    description of the samples."""
    tris = np.asarray(tris, dtype=np.int64)
    rwg = bo.build_rwg(verts, tris, "cpp")
    N = rwg["N"]
    n = 2 * N
    nrhs = 2 * n_orient
    kx, ki, ee, ei = bo.physics(ka, m)
    out, desc = {}, []
    if "assembly" in phases:
        H = bo.halves(rwg, verts, tris, 7)
        r = N if rows in (None, "blocks") else max(1, min(N, rows))
        sel = np.arange(r)
        t0 = time.perf_counter()
        if rows == "blocks":
            # every test row, in blocks of 256 (bounded memory), the same
            # passes as the sampled rows below
            for r0 in range(0, N, 256):
                Hs = [_sub_half(h, np.arange(r0, min(N, r0 + 256))) for h in H]
                for k in (kx, ki):
                    for a in range(2):
                        for b in range(2):
                            bo._regular_LK(Hs[a], H[b], k, distance="expanded")
            t_rows = time.perf_counter() - t0
            t1 = time.perf_counter()
            for k in (kx, ki):
                bo.singular_corrections(rwg, verts, tris, k, 7)
            t_sing = time.perf_counter() - t1
            t_asm = t_rows * 3.0 / 4.0 + t_sing
            desc.append(f"assembly: all {N} test rows in blocks of 256 x all columns, 2 media, 4 half pairs in "
                        f"{t_rows:.2f} s x 3/4 + Graglia terms {t_sing:.2f} s")
        elif r == N:
            bo.assemble_pmchwt(rwg, verts, tris, kx, ki, ee, ei, 7, distance="expanded")
            t_asm = time.perf_counter() - t0
            desc.append(f"assembly full ({t_asm:.2f} s)")
        else:
            Hs = [_sub_half(h, sel) for h in H]
            for k in (kx, ki):
                for a in range(2):
                    for b in range(2):
                        bo._regular_LK(Hs[a], H[b], k, distance="expanded")
            t_rows = time.perf_counter() - t0
            sv, st = (verts, tris) if sing_mesh is None else (sing_mesh[0], np.asarray(sing_mesh[1], np.int64))
            srwg = rwg if sing_mesh is None else bo.build_rwg(sv, st, "cpp")
            t1 = time.perf_counter()
            for k in (kx, ki):
                bo.singular_corrections(srwg, sv, st, k, 7)
            t_sing = (time.perf_counter() - t1) * len(tris) / len(st)
            t_asm = t_rows * 3.0 * N / (4.0 * r) + t_sing
            desc.append(f"assembly: {r} of {N} test rows x all columns, 2 media, 4 half pairs in "
                        f"{t_rows:.2f} s x 3N/(4 rows) + Graglia terms {t_sing:.2f} s"
                        + ("" if sing_mesh is None else f" (timed on {len(st)} triangles, x triangles)"))
        out["assembly"] = t_asm
    if "lu" in phases or "solve" in phases:
        from scipy.linalg import lu_factor, lu_solve
        m_lu = n if n_lu is None else min(n, n_lu)
        r_lu = max(1, round(nrhs * m_lu / n))
        rng = np.random.default_rng(seed)
        A = rng.standard_normal((m_lu, m_lu)) + 1j * rng.standard_normal((m_lu, m_lu))
        Bs = rng.standard_normal((m_lu, r_lu)) + 1j * rng.standard_normal((m_lu, r_lu))
        t0 = time.perf_counter()
        f = lu_factor(A)
        t1 = time.perf_counter()
        lu_solve(f, Bs)
        t2 = time.perf_counter()
        out["lu"] = (t1 - t0) * (n / m_lu) ** 3
        out["solve"] = (t2 - t1) * (n / m_lu) ** 2 * (nrhs / r_lu)
        desc.append(f"LAPACK zgetrf n={m_lu} {t1 - t0:.2f} s, zgetrs {r_lu} rhs {t2 - t1:.2f} s"
                    + ("" if m_lu == n else f", scaled by (n/{m_lu})^3 and (n/{m_lu})^2 nrhs"))
    if "farfield" in phases:
        cache = bo.FarFieldCache(rwg, verts, tris, 7)
        n_s = n_orient if n_ff is None else max(1, min(n_orient, n_ff))
        orients = bo.generate_orientations(max(1, n_s), 1, 1)[:n_s]
        rng = np.random.default_rng(seed + 1)
        X = rng.standard_normal((n, 2 * n_s)) + 1j * rng.standard_normal((n, 2 * n_s))
        nd = ntheta if ff_dirs is None else max(2, min(ntheta, ff_dirs))
        t0 = time.perf_counter()
        bo.mueller_from_solutions(cache, X, orients, kx, ee, bo.theta_grid(nd))
        t_ff = time.perf_counter() - t0
        out["farfield"] = t_ff * (n_orient / n_s) * (ntheta / nd)
        desc.append(f"far field + Mueller of {n_s} of {n_orient} orientations at {nd} of {ntheta} angles "
                    f"{t_ff:.2f} s" + ("" if n_s == n_orient and nd == ntheta else " x orientations x angles"))
    out["total"] = sum(out[k] for k in ("assembly", "lu", "solve", "farfield") if k in out)
    out["solve_only"] = out.get("lu", 0.0) + out.get("solve", 0.0)
    out["description"] = (f"reference CPU dense path (oracle restatement of python/bem_core.py) on 2N={n}, "
                          f"{nrhs} rhs: " + "; ".join(desc) + f"; {cpu_model()}, {os.cpu_count()} logical cores, "
                          f"OPENBLAS_NUM_THREADS={os.environ.get('OPENBLAS_NUM_THREADS', 'unset')}")
    out["n"] = n
    out["cores"] = os.cpu_count() or 1
    return out
