"""Physics checks of the device path (assembly, FP64 solve, far field) that
need no reference output: the optical theorem (extinction from the forward
far-field amplitude equals the scattered power integrated over all
directions for a lossless sphere, and exceeds it for an absorbing one), and
the extinction cross section against the Mie series."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def ctx():
    import bem_b200 as bb
    c = bb.Context(0)
    yield c
    c.close()


def _cross_sections(ctx, m, ka=1.0, refinements=2):
    import bem_b200 as bb
    v, t = bb.icosphere(1.0, refinements)
    g = bb.Geometry(ctx, v, t, 7)
    kx, ki, ee, ei = bb.physics(ka, m)
    Z = bb.assemble_pmchwt_dev(g, kx, ki, ee, ei).cpu().numpy()
    b = bb.compute_rhs_planewave(g, kx, ee, E0=(1.0, 0.0, 0.0), k_hat=(0.0, 0.0, 1.0))
    x = np.linalg.solve(Z, b)
    N = g.N
    # Gauss-Legendre in cos(theta) x uniform phi, then the forward direction
    nt, nph = 40, 80
    mu, wmu = np.polynomial.legendre.leggauss(nt)
    ph = 2 * np.pi * np.arange(nph) / nph
    st = np.sqrt(1 - mu ** 2)
    rh = np.stack([np.outer(st, np.cos(ph)), np.outer(st, np.sin(ph)), np.outer(mu, np.ones(nph))], -1)
    rh = np.concatenate([rh.reshape(-1, 3), [[0.0, 0.0, 1.0]]])
    # one orientation carries two calls (par, perp): the same solution twice
    X2 = np.stack([x, x])
    F = bb.compute_farfield_batch(g, X2[:, :N], X2[:, N:], rh[None], kx, ee)[0]
    w = np.outer(wmu, np.full(nph, 2 * np.pi / nph)).ravel()
    c_sca = float(np.sum(w * np.sum(np.abs(F[:-1]) ** 2, axis=1)))
    # E_s = F exp(ikr)/r with exp(-i omega t): C_ext = (4 pi / k) Im(x . F(z))
    c_ext = float(4 * np.pi / ka * F[-1, 0].imag)
    g.close()
    return c_ext, c_sca


_CACHE = {}


def _cs(ctx, m, refinements):
    key = (complex(m), refinements)
    if key not in _CACHE:
        _CACHE[key] = _cross_sections(ctx, m, 1.0, refinements)
    return _CACHE[key]


def _mie_cross_sections(m, x=1.0):
    """C_ext = (4 pi / k^2) Re S(0); C_sca = (pi / k^2) int (|S1|^2 + |S2|^2) sin(theta)
    (Bohren & Huffman eqs. 4.61, 3.24) for a unit sphere, k = x."""
    from oracle.mie import mie_S12
    mu, w = np.polynomial.legendre.leggauss(200)
    S1, S2 = mie_S12(x, m, np.arccos(mu))
    S0, _ = mie_S12(x, m, np.array([0.0]))
    return 4 * np.pi / x ** 2 * S0[0].real, np.pi / x ** 2 * float(np.sum(w * (abs(S1) ** 2 + abs(S2) ** 2)))


@pytest.mark.parametrize("refinements,tol", [(2, 5e-4), (3, 2e-4)])
def test_optical_theorem_lossless_sphere(ctx, refinements, tol):
    # measured: 6.6e-5 (320 triangles), 1.7e-5 (1280 triangles)
    c_ext, c_sca = _cs(ctx, 1.33, refinements)
    assert c_ext > 0 and abs(c_ext - c_sca) <= tol * c_ext, (c_ext, c_sca)


def test_lossless_sphere_converges_to_mie(ctx):
    e_mie, s_mie = _mie_cross_sections(1.33)
    assert abs(e_mie - s_mie) < 1e-12 * e_mie
    err = [abs(_cs(ctx, 1.33, r)[0] - e_mie) / e_mie for r in (2, 3)]
    # polyhedral sphere: 5.5 % at 320 triangles, 1.25 % at 1280 (h^2)
    assert err[1] < 0.03 and err[1] < err[0] / 3, err


def test_absorbing_sphere_against_mie(ctx):
    m = complex(1.5, 0.05)
    e_mie, s_mie = _mie_cross_sections(m)
    c_ext, c_sca = _cs(ctx, m, 3)
    assert c_ext > c_sca > 0
    # at 1280 triangles, measured against Mie: extinction 2.1 %, scattering
    # 0.5 %, absorption C_ext - C_sca 4.6 % (the polyhedron's volume deficit)
    assert abs(c_ext - e_mie) <= 0.04 * e_mie, (c_ext, e_mie)
    assert abs(c_sca - s_mie) <= 0.02 * s_mie, (c_sca, s_mie)
    assert abs((c_ext - c_sca) - (e_mie - s_mie)) <= 0.08 * (e_mie - s_mie)


def _unit_perp(rng, k):
    p = np.cross(k, rng.standard_normal(3))
    return p / np.linalg.norm(p)


@pytest.mark.parametrize("m", [1.4, complex(1.5, 0.02)])
def test_reciprocity_on_an_irregular_particle(ctx, m):
    """p_s . F(k_s | k_i, p_i) = p_i . F(-k_i | -k_s, p_s) for any scatterer
    (Saxon's reciprocity of the amplitude matrix); checked on a randomly
    perturbed sphere with no symmetry, several direction pairs.  The Galerkin
    discretisation keeps it exactly (the right-hand side and the far field
    share one quadrature), so the bound is rounding, not discretisation."""
    import bem_b200 as bb
    v, t = bb.c5_mesh(11, refinements=2, rms=0.08)
    g = bb.Geometry(ctx, v, t, 7)
    kx, ki, ee, ei = bb.physics(2.0, m)
    Z = bb.assemble_pmchwt_dev(g, kx, ki, ee, ei).cpu().numpy()
    N = g.N
    rng = np.random.default_rng(5)
    worst = 0.0
    for _ in range(4):
        a, b = rng.standard_normal(3), rng.standard_normal(3)
        k_i, k_s = a / np.linalg.norm(a), b / np.linalg.norm(b)
        p_i, p_s = _unit_perp(rng, k_i), _unit_perp(rng, k_s)

        def amp(k_in, p_in, k_out):
            x = np.linalg.solve(Z, bb.compute_rhs_planewave(g, kx, ee, E0=p_in, k_hat=k_in))
            X2 = np.stack([x, x])
            return bb.compute_farfield_batch(g, X2[:, :N], X2[:, N:], k_out[None, None], kx, ee)[0, 0]

        f1 = p_s @ amp(k_i, p_i, k_s)
        f2 = p_i @ amp(-k_s, p_s, -k_i)
        worst = max(worst, abs(f1 - f2) / max(abs(f1), abs(f2)))
    g.close()
    assert worst < 1e-10, worst
