"""Reciprocity of the oracle's discretisation (CPU): the plane-wave right-hand
side (rhs.cpp:6-64) and the far field (farfield.cu:100-262) test the same
currents with the same quadrature, so p_s . F(k_s | k_i, p_i) =
p_i . F(-k_i | -k_s, p_s) holds to rounding for any mesh."""
import numpy as np
import pytest

from oracle import bem_oracle as bo


@pytest.mark.parametrize("m", [1.4, complex(1.5, 0.02)])
def test_oracle_reciprocity(m):
    rng = np.random.default_rng(3)
    v, t = bo.icosphere(1.0, 1)
    v = v * (1.0 + 0.1 * rng.standard_normal(len(v)))[:, None]   # no symmetry left
    t = t.astype(np.int64)
    rwg = bo.build_rwg(v, t, "cpp")
    kx, ki, ee, ei = bo.physics(2.0, m)
    Z = bo.assemble_pmchwt(rwg, v, t, kx, ki, ee, ei)
    cache = bo.FarFieldCache(rwg, v, t)
    N = rwg["N"]

    def perp(k):
        p = np.cross(k, rng.standard_normal(3))
        return p / np.linalg.norm(p)

    def amp(k_in, p_in, k_out):
        x = np.linalg.solve(Z, bo.rhs_planewave(rwg, v, t, kx, ee, p_in, k_in))
        return bo.far_field_vec(cache, x[:N], x[N:], kx, ee, k_out[None])[0]

    for _ in range(3):
        a, b = rng.standard_normal(3), rng.standard_normal(3)
        k_i, k_s = a / np.linalg.norm(a), b / np.linalg.norm(b)
        p_i, p_s = perp(k_i), perp(k_s)
        f1, f2 = p_s @ amp(k_i, p_i, k_s), p_i @ amp(-k_s, p_s, -k_i)
        assert abs(f1 - f2) <= 1e-12 * max(abs(f1), abs(f2)), (f1, f2)
