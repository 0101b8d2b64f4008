"""Generate the golden fixtures in this folder by running the reference itself.

Runs the reference's FP64 CPU implementation, ``python/bem_core.py`` of
KirillSalnikov/BEM-CPP (imported read-only from ``--ref``), and the reference's
own C++ mesher (``oracle/_ref/libref_host.so``, built by ``oracle/Makefile``)
on small seeded cases, and stores inputs and outputs as ``.npz`` files:

  ico0_Z.npz      icosahedron (n=60): full Z, lossless and absorbing media
  ico1_probe.npz  ico ref 1 (n=240), quad orders 4/7/13: Z probes
  c1_single.npz   ico ref 2, ka=1, m=1.3116 (n=960), --single: Z probes, b, X, Mueller
  ico1_orient.npz ico ref 1, ka=2, m=1.3116+0.001i, 3x4x2 orientations: <M>
  hex1_probe.npz  hex prism AR=0.7 ref 1 from the C++ mesher (C++ RWG order): Z probes
  c1_gmres.npz    C1 system solved by the reference's GMRES: solve_gmres_aext (both
                  columns) and solve_gmres with 'block_diag', 'diag' and None
                  (column 0); solutions and the inner iteration counts it prints

"Z probes" are Z @ v for a seeded complex vector v, diag(Z), ||Z||_F and
Z[::s, ::s].  Usage:  python tests/golden/make_golden.py --ref <reference checkout>
[--only gmres]  (--ref defaults to the environment variable BEM_REFERENCE_DIR).
"""
from __future__ import annotations

import argparse
import contextlib
import io
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
REPO = os.path.dirname(os.path.dirname(HERE))


def probes(Z, stride):
    rng = np.random.default_rng(1234)
    v = rng.standard_normal(Z.shape[0]) + 1j * rng.standard_normal(Z.shape[0])
    return {"probe_v": v, "Zv": Z @ v, "diag": np.diag(Z).copy(),
            "fro": np.linalg.norm(Z), "sub": Z[::stride, ::stride].copy(),
            "stride": stride}


def rwg_arrays(rwg):
    return {f"rwg_{k}": np.asarray(v) for k, v in rwg.items() if k != "N"}


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--ref", default=os.environ.get("BEM_REFERENCE_DIR"))
    ap.add_argument("--only", choices=["gmres"], default=None)
    a = ap.parse_args()
    if not a.ref or not os.path.isdir(os.path.join(a.ref, "python")):
        ap.error("give the reference checkout with --ref or BEM_REFERENCE_DIR")
    # bem_core's numba functions cache next to their source unless told
    # otherwise; the reference tree is read-only
    import tempfile
    os.environ.setdefault("NUMBA_CACHE_DIR", tempfile.mkdtemp(prefix="bem_golden_numba_"))
    sys.path.insert(0, os.path.join(a.ref, "python"))
    sys.path.insert(0, REPO)
    import bem_core as bc  # noqa: E402  (the reference, read-only)
    from oracle import ref_host  # noqa: E402

    quiet = contextlib.redirect_stdout(io.StringIO())
    if a.only == "gmres":
        gmres_golden(bc)
        return

    # 1. icosahedron, full Z
    v, t = bc.icosphere(1.0, 0)
    rwg = bc.build_rwg(v, t)
    out = {"verts": v, "tris": t, **rwg_arrays(rwg)}
    for tag, m in (("lossless", 1.3116), ("absorbing", 1.3116 + 0.01j)):
        with quiet:
            Z, _, _ = bc.assemble_pmchwt(rwg, v, t, 1.0, 1.0 * m, 1.0, 1.0 / abs(m),
                                         quad_order=7, parallel=False)
        out[f"Z_{tag}"] = Z
        out[f"m_{tag}"] = m
    out["ka"] = 1.0
    np.savez_compressed(os.path.join(HERE, "ico0_Z.npz"), **out)

    # 2. ico ref 1, three quadrature orders
    v, t = bc.icosphere(1.0, 1)
    rwg = bc.build_rwg(v, t)
    out = {"verts": v, "tris": t, **rwg_arrays(rwg), "ka": 2.0, "m": 1.5 + 0.02j}
    for q in (4, 7, 13):
        with quiet:
            Z, _, _ = bc.assemble_pmchwt(rwg, v, t, 2.0, 2.0 * (1.5 + 0.02j), 1.0,
                                         1.0 / abs(1.5 + 0.02j), quad_order=q, parallel=False)
        for k, val in probes(Z, 7).items():
            out[f"q{q}_{k}"] = val
    np.savez_compressed(os.path.join(HERE, "ico1_probe.npz"), **out)

    # 3. C1: ico ref 2, ka=1, m=1.3116, single orientation (validate.py:9-12)
    v, t = bc.icosphere(1.0, 2)
    rwg = bc.build_rwg(v, t)
    m = 1.3116
    with quiet:
        Z, _, _ = bc.assemble_pmchwt(rwg, v, t, 1.0, 1.0 * m, 1.0, 1.0 / abs(m),
                                     quad_order=7, parallel=False)
    theta = np.linspace(0, np.pi, 181)
    from scipy.linalg import lu_factor, lu_solve
    lu = lu_factor(Z)
    b_par = bc.compute_rhs_planewave(rwg, v, t, 1.0, 1.0, E0=np.array([1.0, 0, 0]),
                                     k_hat=np.array([0, 0, 1.0]), quad_order=7)
    b_perp = bc.compute_rhs_planewave(rwg, v, t, 1.0, 1.0, E0=np.array([0, 1.0, 0]),
                                      k_hat=np.array([0, 0, 1.0]), quad_order=7)
    B = np.stack([b_par, b_perp], 1)
    X = lu_solve(lu, B)
    with quiet:
        M = bc.compute_mueller_matrix(rwg, v, t, 1.0, 1.0, theta, Z_lu=lu,
                                      k_hat=np.array([0, 0, 1.0]), sM=-1, quad_order=7)
    out = {"verts": v, "tris": t, **rwg_arrays(rwg), "ka": 1.0, "m": m, "B": B, "X": X,
           "mueller": M, "theta": theta, **probes(Z, 17)}
    np.savez_compressed(os.path.join(HERE, "c1_single.npz"), **out)

    # 4. orientation average, ico ref 1
    v, t = bc.icosphere(1.0, 1)
    rwg = bc.build_rwg(v, t)
    m = 1.3116 + 0.001j
    with quiet:
        Z, _, _ = bc.assemble_pmchwt(rwg, v, t, 2.0, 2.0 * m, 1.0, 1.0 / abs(m),
                                     quad_order=7, parallel=False)
        theta = np.linspace(0, np.pi, 37)
        Mavg = bc.orientation_average_mueller_batched(rwg, v, t, 2.0, 1.0, theta, Z=Z,
                                                      quad_order=7, n_alpha=3, n_beta=4,
                                                      n_gamma=2)
    out = {"verts": v, "tris": t, **rwg_arrays(rwg), "ka": 2.0, "m": m, "theta": theta,
           "orient": np.array([3, 4, 2]), "mueller": Mavg, **probes(Z, 7)}
    np.savez_compressed(os.path.join(HERE, "ico1_orient.npz"), **out)

    # 5. hex prism from the reference's C++ mesher, C++ RWG order
    if ref_host.available():
        v, t, rwg = ref_host.make_mesh("hex", 0.7, 1)
        m = 1.31 + 0.0001j
        with quiet:
            Z, _, _ = bc.assemble_pmchwt(rwg, v, t, 3.0, 3.0 * m, 1.0, 1.0 / abs(m),
                                         quad_order=7, parallel=False)
        out = {"verts": v, "tris": t, **rwg_arrays(rwg), "ka": 3.0, "m": m, "ar": 0.7,
               "ref": 1, **probes(Z, 5)}
        np.savez_compressed(os.path.join(HERE, "hex1_probe.npz"), **out)
    else:
        print("oracle/_ref/libref_host.so missing: run `make -C oracle` first; hex1 skipped")
    gmres_golden(bc)


def gmres_golden(bc):
    """6. C1 solved by the reference's GMRES paths (bem_core.py:1071-1183)."""
    import re
    v, t = bc.icosphere(1.0, 2)
    rwg = bc.build_rwg(v, t)
    N = len(rwg["length"])
    m = 1.3116
    with contextlib.redirect_stdout(io.StringIO()):
        Z, Lext, Kext = bc.assemble_pmchwt(rwg, v, t, 1.0, 1.0 * m, 1.0, 1.0 / abs(m),
                                           quad_order=7, parallel=False)
        Zext_lu, _ = bc.build_aext_preconditioner(Lext, Kext, 1.0, N)
    B = np.stack([bc.compute_rhs_planewave(rwg, v, t, 1.0, 1.0, E0=np.array(e),
                                           k_hat=np.array([0, 0, 1.0]), quad_order=7)
                  for e in ([1.0, 0, 0], [0, 1.0, 0])], 1)
    out = {"verts": v, "tris": t, **rwg_arrays(rwg), "ka": 1.0, "m": m, "B": B,
           "tol_aext": 1e-5, "maxiter_aext": 200, "tol": 1e-4, "maxiter": 500}
    buf = io.StringIO()
    with contextlib.redirect_stdout(buf):
        xs = [bc.solve_gmres_aext(Z, B[:, c], Zext_lu) for c in range(2)]
    out["x_aext"] = np.stack(xs, 1)
    out["it_aext"] = np.array([int(i) for i in re.findall(r"GMRES\(A_ext\): (\d+) iter", buf.getvalue())])
    assert len(out["it_aext"]) == 2, buf.getvalue()
    for tag, pc in (("block_diag", "block_diag"), ("diag", "diag"), ("none", None)):
        buf = io.StringIO()
        with contextlib.redirect_stdout(buf):
            x = bc.solve_gmres(Z, B[:, 0], precond=pc)
        it = re.findall(r"(\d+) iterations", buf.getvalue())
        assert len(it) == 1, buf.getvalue()
        out[f"x_{tag}"] = x
        out[f"it_{tag}"] = int(it[0])
        out[f"conv_{tag}"] = "did not converge" not in buf.getvalue()
    np.savez_compressed(os.path.join(HERE, "c1_gmres.npz"), **out)


if __name__ == "__main__":
    main()
