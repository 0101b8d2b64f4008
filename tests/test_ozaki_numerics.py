"""The arithmetic of the int8 Ozaki refinement residual, restated in NumPy
(CPU): the row / column exponent e = ilogb(max|v|) + 2 (every scaled entry
below 1/2), digits q_s = rint(128 t) of the running remainder (q in
[-64, 64], remainder at most 2^(-7S-1)), the digit pairs kept (s + t <= S + 1),
the int32 headroom of an accumulator shared by up to four pairs, and the
digit count of the update-form residual r1 = r0 - Z d0.  The products are
taken exactly in int64 here; what is measured is the slicing and the pair
truncation, the two approximations of the device kernel."""
import math

import numpy as np
import pytest


def _exp(m):
    """ilogb(m) + 2, or 0 for m = 0."""
    return np.where(m > 0, np.frexp(np.where(m > 0, m, 1.0))[1] - 1 + 2, 0)


def _digits(v, S):
    q = np.zeros((S,) + v.shape, dtype=np.int64)
    for s in range(S):
        t = v * 128.0
        r = np.rint(t)
        q[s] = r.astype(np.int64)
        v = t - r
    return q, v


def _ozaki_product(A, B, S):
    """A (m x K), B (K x n) real -> the S-digit, s + t <= S + 1 approximation of A B."""
    ea = _exp(np.abs(A).max(axis=1))
    eb = _exp(np.abs(B).max(axis=0))
    qa, _ = _digits(A * np.ldexp(1.0, -ea)[:, None], S)
    qb, _ = _digits(B * np.ldexp(1.0, -eb)[None, :], S)
    out = np.zeros((A.shape[0], B.shape[1]))
    for s in range(1, S + 1):
        for t in range(1, S + 2 - s):
            P = qa[s - 1] @ qb[t - 1]                       # exact in int64
            out += np.ldexp(P.astype(np.float64), -7 * (s + t))
    return out * np.ldexp(1.0, ea)[:, None] * np.ldexp(1.0, eb)[None, :], ea, eb


def test_digits_reconstruct_to_the_stated_remainder():
    rng = np.random.default_rng(0)
    v = rng.uniform(-0.5, 0.5, 100000) * 10.0 ** rng.uniform(-20, 0, 100000)
    v = np.clip(v, -0.4999999999, 0.4999999999)
    for S in (5, 7, 8):
        q, r = _digits(v, S)
        assert np.abs(q).max() <= 64
        recon = sum(np.ldexp(q[s].astype(np.float64), -7 * (s + 1)) for s in range(S))
        assert np.abs(v - recon).max() <= 2.0 ** (-7 * S - 1)
        assert np.abs(r).max() <= 0.5


def test_scaled_entries_stay_below_one_half():
    rng = np.random.default_rng(1)
    m = np.abs(rng.standard_normal(10000)) * 10.0 ** rng.uniform(-300, 300, 10000)
    e = _exp(m)
    s = m * np.ldexp(1.0, -e)
    assert (s < 0.5).all() and (s >= 0.25).all()
    assert _exp(np.array([0.0]))[0] == 0


@pytest.mark.parametrize("S", [5, 7])
def test_pair_truncation_bound(S):
    # per term 2^(4-7S) of max|row| max|column|: summed over K terms
    rng = np.random.default_rng(2)
    K = 384
    A = rng.standard_normal((64, K)) * 10.0 ** rng.uniform(-3, 3, (64, 1))
    B = rng.standard_normal((K, 48)) * 10.0 ** rng.uniform(-3, 3, (1, 48))
    P, ea, eb = _ozaki_product(A, B, S)
    # FP64's own rounding of A B is far below the bound at S = 5 and near it
    # at S = 7, so a few ulps of the scale are allowed on top
    exact = A @ B
    scale = np.abs(A).max(axis=1)[:, None] * np.abs(B).max(axis=0)[None, :]
    err = np.abs(P - exact) / (K * scale)
    assert err.max() <= 2.0 ** (4 - 7 * S) + 4 * 2.0 ** -53, (S, err.max())


def test_shared_accumulator_stays_in_int32():
    # four pairs of |q| <= 64 digits over K' = 2n terms, n = 61440
    K2 = 2 * 61440
    assert 4 * 64 * 64 * K2 < 2 ** 31
    # the host's group size for the padded K' (a multiple of 128 bytes)
    ldk = ((K2 + 127) // 128) * 128
    maxp = min(4, (2 ** 31) // (4096 * ldk + 1))
    assert maxp == 4
    # one digit pair of the largest order that fits the 2^31 bound alone
    assert 64 * 64 * ((2 ** 31 - 1) // 4096) < 2 ** 31


def _update_digits(prev_upd, S=7):
    """The device rule: S - floor((-log2(prev_upd) + 1) / 7), clamped to [2, S]."""
    lg = -math.log2(prev_upd) + 1.0
    return min(S, max(2, S - int(min(64.0, math.floor(lg / 7.0)))))


@pytest.mark.parametrize("prev_upd", [0.4, 1.1e-4, 5.6e-5, 1e-6, 2.2e-9, 1e-14])
def test_update_form_digits_keep_the_absolute_accuracy(prev_upd):
    # the update form truncates 2^(4 - 7d) of max|Z| max|d| with
    # max|d| ~ prev_upd max|x|; it must stay within twice the full product's
    # 2^(4 - 7S) of max|Z| max|x| (one bit of slack)
    S = 7
    d = _update_digits(prev_upd, S)
    assert 2 <= d <= S
    assert 2.0 ** (4 - 7 * d) * prev_upd <= 2.0 * 2.0 ** (4 - 7 * S) or d == 2
    # and it is the fewest digits that do
    if d > 2:
        assert not (2.0 ** (4 - 7 * (d - 1)) * prev_upd <= 2.0 * 2.0 ** (4 - 7 * S))
    assert {1.1e-4: 5, 5.6e-5: 5}.get(prev_upd, d) == d


def _ozaki_product_sx(A, B, S, Sx):
    """The product with B's columns kept to Sx digits: pairs s <= S, t <= Sx,
    s + t <= S + 1 (1-based), and the value B~ those Sx digits represent."""
    ea = _exp(np.abs(A).max(axis=1))
    eb = _exp(np.abs(B).max(axis=0))
    qa, _ = _digits(A * np.ldexp(1.0, -ea)[:, None], S)
    qb, _ = _digits(B * np.ldexp(1.0, -eb)[None, :], Sx)
    # the rounded B, rebuilt from its digits by Horner in base 128 (exact)
    Bt = np.zeros_like(B)
    for t in range(Sx - 1, -1, -1):
        Bt = (Bt + qb[t]) / 128.0
    Bt = Bt * np.ldexp(1.0, eb)[None, :]
    out = np.zeros((A.shape[0], B.shape[1]))
    for s in range(1, S + 1):
        for t in range(1, min(Sx, S + 1 - s) + 1):
            out += np.ldexp((qa[s - 1] @ qb[t - 1]).astype(np.float64), -7 * (s + t))
    return out * np.ldexp(1.0, ea)[:, None] * np.ldexp(1.0, eb)[None, :], Bt


@pytest.mark.parametrize("Sx", [2, 3])
def test_rounded_iterate_is_exact_and_needs_fewer_pairs(Sx):
    # the refinement's iterate kept to Sx digits: the rebuilt value equals the
    # sum of its digits exactly, lies within 2^(-7 Sx - 1) of its column's
    # scale from the original, and the product over the pairs t <= Sx is the
    # product with the rounded iterate to the same bound as with every digit
    rng = np.random.default_rng(3 + Sx)
    K, S = 256, 7
    A = rng.standard_normal((40, K)) * 10.0 ** rng.uniform(-2, 2, (40, 1))
    X = rng.standard_normal((K, 6)) * 10.0 ** rng.uniform(-5, 5, (1, 6))
    P, Xt = _ozaki_product_sx(A, X, S, Sx)
    eb = _exp(np.abs(X).max(axis=0))
    assert np.all(np.abs(Xt - X) <= np.ldexp(2.0 ** (-7 * Sx - 1), eb)[None, :])
    qb, _ = _digits(Xt * np.ldexp(1.0, -eb)[None, :], S)
    assert not qb[Sx:].any()  # the rounded iterate has no digits beyond Sx
    exact = A.astype(np.longdouble) @ Xt.astype(np.longdouble)
    scale = np.abs(A).max(axis=1)[:, None] * np.abs(Xt).max(axis=0)[None, :]
    err = np.abs(P - exact.astype(np.float64)) / (K * scale)
    assert err.max() <= 2.0 ** (4 - 7 * S) + 4 * 2.0 ** -53
    # 13 pairs instead of 28 for Sx = 2 (18 for 3)
    pairs = sum(1 for s in range(1, S + 1) for t in range(1, min(Sx, S + 1 - s) + 1))
    assert pairs == {2: 13, 3: 18}[Sx]
