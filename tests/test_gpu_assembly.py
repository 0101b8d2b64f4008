"""Device assembly against the oracle (same inputs, FP64)."""
import numpy as np
import pytest

from conftest import golden_rwg, load_golden, rel
from oracle import bem_oracle as bo

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def ctx():
    import bem_b200 as bb
    c = bb.Context(0)
    yield c
    c.close()


def _oracle_Z(v, t, ka, m, q=7, smooth="literal"):
    rwg = bo.build_rwg(v, t, order="cpp")
    kx, ki, ee, ei = bo.physics(ka, m)
    return bo.assemble_pmchwt(rwg, v, t, kx, ki, ee, ei, q, distance="direct", smooth=smooth)


@pytest.mark.parametrize("ref,ka,m,q", [(1, 2.0, 1.5 + 0.02j, 7), (2, 1.0, 1.3116, 7),
                                        (1, 3.0, 1.31 + 1e-4j, 4), (1, 3.0, 1.6, 13)])
def test_icosphere_Z_matches_oracle(ctx, ref, ka, m, q):
    import bem_b200 as bb
    v, t = bb.icosphere(1.0, ref)
    g = bb.Geometry(ctx, v, t, q)
    kx, ki, ee, ei = bb.physics(ka, m)
    Z = bb.assemble_pmchwt_dev(g, kx, ki, ee, ei).cpu().numpy()
    Zo = _oracle_Z(v, t.astype(np.int64), ka, m, q)
    assert rel(Z, Zo) < 1e-12


def test_exact_gsmooth_matches_oracle(ctx):
    import bem_b200 as bb
    v, t = bb.icosphere(1.0, 1)
    g = bb.Geometry(ctx, v, t, 7)
    kx, ki, ee, ei = bb.physics(2.0, 1.5 + 0.05j)
    Z = bb.assemble_pmchwt_dev(g, kx, ki, ee, ei, exact_gsmooth=True).cpu().numpy()
    Zo = _oracle_Z(v, t.astype(np.int64), 2.0, 1.5 + 0.05j, 7, smooth="exact")
    assert rel(Z, Zo) < 1e-12


def test_hex_prism_against_reference_golden(ctx):
    # golden made by the reference's bem_core on the reference C++ mesher's hex
    import bem_b200 as bb
    g0 = load_golden("hex1_probe.npz")
    v, t = bb.hex_prism(float(g0["ar"]), int(g0["ref"]))
    g = bb.Geometry(ctx, v, t, 7)
    kx, ki, ee, ei = bb.physics(float(g0["ka"]), complex(g0["m"]))
    Z = bb.assemble_pmchwt_dev(g, kx, ki, ee, ei).cpu().numpy()
    Zo = _oracle_Z(v, t.astype(np.int64), float(g0["ka"]), complex(g0["m"]))
    assert rel(Z, Zo) < 1e-12
    # Same RWG order as the reference C++ (rwg.cpp), so probes compare
    # directly.  The medium is absorbing (k_int has Im 3e-4): the reference's
    # literal G_smooth at coincident points is +-1 ulp of 1/(4 pi 1e-15) and
    # depends on its |a|^2+|b|^2-2a.b distance rounding, which moves the L
    # diagonal blocks by ~1e-6 relative (see oracle/bem_oracle.py).
    assert rel(Z @ g0["probe_v"], g0["Zv"]) < 2e-6


def test_L_K_single_medium(ctx):
    import bem_b200 as bb
    v, t = bb.icosphere(1.0, 1)
    g = bb.Geometry(ctx, v, t, 7)
    L, K = bb.assemble_L_K_dev(g, 2.5 + 0.01j)
    rwg = bo.build_rwg(v, t.astype(np.int64), order="cpp")
    Lo, Ko = bo.assemble_L_K(rwg, v, t.astype(np.int64), 2.5 + 0.01j, 7)
    assert rel(L.cpu().numpy(), Lo) < 1e-12
    assert rel(K.cpu().numpy(), Ko) < 1e-12


@pytest.mark.parametrize("case", ["ico2", "hex_absorbing", "ico1_exact", "ico1_q13"])
def test_triangle_pair_kernel_matches_rwg_pair_kernel(ctx, case):
    # the default assembly (triangle-pair moments over Morton-ordered tiles)
    # against the per-RWG-pair kernel: PMCHWT, L/K of one medium and A_ext
    import bem_b200 as bb
    if case == "hex_absorbing":
        v, t = bb.hex_prism(0.7, 1)
        ka, m, q, ex = 3.0, 1.31 + 1e-4j, 7, False
    else:
        v, t = bb.icosphere(1.0, 2 if case == "ico2" else 1)
        ka, m = (1.0, 1.3116) if case == "ico2" else (2.0, 1.5 + 0.05j)
        q, ex = (13 if case == "ico1_q13" else 7), case == "ico1_exact"
    g = bb.Geometry(ctx, v, t, q)
    kx, ki, ee, ei = bb.physics(ka, m)
    out = {}
    for kern in (1, 0):
        bb.set_option(ctx, "assembly_kernel", kern)
        try:
            Z = bb.assemble_pmchwt_dev(g, kx, ki, ee, ei, exact_gsmooth=ex).cpu().numpy()
            L, K = (x.cpu().numpy() for x in bb.assemble_L_K_dev(g, ki, exact_gsmooth=ex))
            A = bb.assemble_aext_dev(g, kx, ee, exact_gsmooth=ex).cpu().numpy()
        finally:
            bb.set_option(ctx, "assembly_kernel", 0)
        out[kern] = (Z, L, K, A)
    for new, old in zip(out[0], out[1]):
        assert rel(new, old) < 1e-13
    Z = out[0][0]
    n = Z.shape[0]
    S = Z.copy()
    S[:, n // 2:] *= -1
    assert np.array_equal(S, S.T)          # still written once per symmetric pair
    g.close()


def test_vertices_moved_in_place_equal_a_new_geometry(ctx):
    # bem_geom_set_vertices: right-hand sides and Mueller matrix of a geometry
    # moved in place are bitwise those of a geometry created from the moved
    # mesh; the operator agrees to rounding (the moved geometry keeps its
    # assembly tiles, which fix the orientation each symmetric pair is
    # computed in) and is bitwise its own again when moved back
    import bem_b200 as bb
    v0, t = bb.c5_mesh(1, refinements=2, rms=0.05)
    v1, _ = bb.c5_mesh(2, refinements=2, rms=0.05)
    kx, ki, ee, ei = bb.physics(2.0, complex(1.4, 0.01))
    RT, w = bb.generate_orientations(2, 3, 1)

    def products(g):
        Z = bb.assemble_pmchwt_dev(g, kx, ki, ee, ei).cpu().numpy()
        B = bb.rhs_planewave_dev(g, kx, ee, RT)
        M = bb.mueller_from_solutions_dev(g, B, RT, w, kx, ee, 19)
        return Z, B.cpu().numpy(), M

    gm = bb.Geometry(ctx, v0, t, 7)
    p0 = products(gm)
    gm.set_vertices(v1)
    moved = products(gm)
    gn = bb.Geometry(ctx, v1, t, 7)
    fresh = products(gn)
    assert rel(moved[0], fresh[0]) < 1e-14
    for a, b in zip(moved[1:], fresh[1:]):
        assert np.array_equal(a, b)
    assert rel(p0[0], fresh[0]) > 1e-3          # the shape did change
    gm.set_vertices(v0)
    for a, b in zip(products(gm), p0):
        assert np.array_equal(a, b)
    with pytest.raises(bb.BemError):
        gr = bb.Geometry.from_rwg(ctx, v0, t, bb.build_rwg(v0, t), 7)
        gr.set_vertices(v1)
    gm.close()
    gn.close()
