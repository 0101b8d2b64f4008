"""Pins the CPU oracle against golden vectors made by the reference itself
(tests/golden/make_golden.py runs python/bem_core.py and the C++ mesher)."""
import numpy as np
import pytest

from conftest import golden_rwg, load_golden, rel
from oracle import bem_oracle as bo


def _Z(g, ka, m, q=7, distance="expanded", smooth="literal"):
    rwg = golden_rwg(g)
    kx, ki, ee, ei = bo.physics(ka, m)
    return bo.assemble_pmchwt(rwg, g["verts"], g["tris"].astype(np.int64), kx, ki, ee, ei, q,
                              distance=distance, smooth=smooth)


@pytest.mark.parametrize("tag", ["lossless", "absorbing"])
def test_full_Z_icosahedron_replays_reference(tag):
    g = load_golden("ico0_Z.npz")
    Z = _Z(g, float(g["ka"]), complex(g[f"m_{tag}"]))
    assert rel(Z, g[f"Z_{tag}"]) < 1e-13


def test_direct_distance_within_reference_noise_lossless():
    # bem_core forms R by |a|^2+|b|^2-2a.b; the direct form differs by the
    # rounding noise of that expansion at (near-)coincident points only.
    g = load_golden("ico0_Z.npz")
    Z = _Z(g, float(g["ka"]), complex(g["m_lossless"]), distance="direct")
    assert rel(Z, g["Z_lossless"]) < 3e-10


def test_absorbing_coincident_point_artifact_is_confined():
    # For absorbing media the reference's literal G_smooth at R=0 is +-1 ulp of
    # 1/(4 pi 1e-15); the direct distance changes which ulp.  Only the L
    # blocks (diagonal blocks of Z) and only same-triangle pairs can move.
    g = load_golden("ico0_Z.npz")
    Z = _Z(g, float(g["ka"]), complex(g["m_absorbing"]), distance="direct")
    D = np.abs(Z - g["Z_absorbing"])
    N = Z.shape[0] // 2
    assert D[:N, N:].max() < 1e-12 and D[N:, :N].max() < 1e-12
    assert rel(Z, g["Z_absorbing"]) < 1e-3


@pytest.mark.parametrize("q", [4, 7, 13])
def test_quadrature_orders_probe(q):
    g = load_golden("ico1_probe.npz")
    Z = _Z(g, float(g["ka"]), complex(g["m"]), q=q)
    # 1e-12: the singular correction sums in a different order than numba
    assert rel(Z @ g[f"q{q}_probe_v"], g[f"q{q}_Zv"]) < 1e-12
    assert rel(np.diag(Z), g[f"q{q}_diag"]) < 1e-12
    s = int(g[f"q{q}_stride"])
    assert rel(Z[::s, ::s], g[f"q{q}_sub"]) < 1e-12


def test_hex_prism_mesh_and_probe():
    g = load_golden("hex1_probe.npz")
    v, t = bo.hex_prism(float(g["ar"]), int(g["ref"]))
    assert np.array_equal(t, g["tris"]) and np.abs(v - g["verts"]).max() == 0.0
    rwg = bo.build_rwg(v, t, order="cpp")
    gr = golden_rwg(g)
    assert np.array_equal(rwg["tri_p"], gr["tri_p"]) and np.array_equal(rwg["tri_m"], gr["tri_m"])
    assert np.abs(rwg["length"] - gr["length"]).max() < 1e-15
    Z = _Z(g, float(g["ka"]), complex(g["m"]))
    assert rel(Z @ g["probe_v"], g["Zv"]) < 1e-13


def test_c1_single_orientation_end_to_end():
    g = load_golden("c1_single.npz")
    rwg = golden_rwg(g)
    v, t = g["verts"], g["tris"].astype(np.int64)
    Z = _Z(g, 1.0, complex(g["m"]))
    assert rel(Z @ g["probe_v"], g["Zv"]) < 1e-13
    M, X, B = bo.single_orientation_mueller(rwg, v, t, Z, 1.0, 1.0, 181, 7)
    assert rel(B, g["B"]) < 1e-14
    assert rel(X, g["X"]) < 1e-12
    assert rel(M, g["mueller"]) < 1e-12


def test_orientation_average():
    g = load_golden("ico1_orient.npz")
    rwg = golden_rwg(g)
    v, t = g["verts"], g["tris"].astype(np.int64)
    Z = _Z(g, float(g["ka"]), complex(g["m"]))
    na, nb, ng = (int(x) for x in g["orient"])
    M, _, _ = bo.orientation_average_mueller(rwg, v, t, Z, float(g["ka"]), 1.0, na, nb, ng,
                                             len(g["theta"]), 7)
    assert rel(M, g["mueller"]) < 1e-11
