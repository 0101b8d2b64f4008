"""The arithmetic of the tensor-core GEMM's FP16 operand split, restated in
NumPy (CPU): a power-of-two scale per row of A and per column of B that
brings the largest |Re|, |Im| into [2^14, 2^15) (the device code's
f16_scale_kernel: frexp, exponent clamped at -100), the split
x s = hi + lo with hi, lo rounded to FP16, and the three products
hi*hi + hi*lo + lo*hi.  The products are summed here in FP64, so what is
measured is the split alone, not the tensor core's FP32 accumulation."""
import numpy as np


def _scale(m):
    """(s, 1/s) with m s in [2^14, 2^15); (1, 1) for m = 0."""
    m = np.asarray(m, dtype=np.float32)
    _, e = np.frexp(m)
    e = np.maximum(e, -100)
    s = np.where(m > 0, np.ldexp(np.float32(1), 15 - e), np.float32(1)).astype(np.float32)
    return s, (np.float32(1) / s).astype(np.float32)


def _split(x):
    hi = x.astype(np.float16)
    lo = (x - hi.astype(np.float32)).astype(np.float16)
    return hi, lo


def _split_product(A, B):
    """A (M x K), B (K x N) float32 -> the three-product approximation of A B."""
    sa, ia = _scale(np.abs(A).max(axis=1))
    sb, ib = _scale(np.abs(B).max(axis=0))
    ah, al = _split((A * sa[:, None]).astype(np.float32))
    bh, bl = _split((B * sb[None, :]).astype(np.float32))
    f = lambda x: x.astype(np.float64)
    acc = f(ah) @ f(bh) + f(ah) @ f(bl) + f(al) @ f(bh)
    return acc * f(ia)[:, None] * f(ib)[None, :], (ah, al, bh, bl)


def _rand(rng, m, n, spread=0.0):
    x = rng.standard_normal((m, n))
    if spread:
        x *= 10.0 ** (spread * (2 * rng.random(m) - 1))[:, None]
        x *= 10.0 ** (spread * (2 * rng.random(n) - 1))[None, :]
    return x.astype(np.float32)


def test_scale_brings_the_largest_entry_into_range():
    for m in (1e-30, 3e-8, 0.7, 1.0, 2.0, 65504.0, 1e30, np.float32(2.0 ** -140)):
        s, inv = _scale(m)
        v = np.float32(m) * s
        assert np.float32(v * inv) == np.float32(m)
        if m >= 2.0 ** -100:
            assert 2.0 ** 14 <= v < 2.0 ** 15, (m, v)
        else:
            assert v < 2.0 ** 15
    assert _scale(0.0) == (1.0, 1.0)


def test_split_error_is_fp32_class():
    rng = np.random.default_rng(0)
    A, B = _rand(rng, 200, 256), _rand(rng, 256, 150)
    P, _ = _split_product(A, B)
    ref = A.astype(np.float64) @ B.astype(np.float64)
    bound = np.abs(A).astype(np.float64) @ np.abs(B).astype(np.float64)
    err = (np.abs(P - ref) / bound).max()
    # two 11-bit parts per operand: about 2^-22 of |A| |B| at most, well under
    # the FP32 accumulation error of a K = 256 sum
    assert err < 2.0 ** -20, err


def test_spread_rows_and_columns_stay_finite_and_accurate():
    rng = np.random.default_rng(1)
    A, B = _rand(rng, 120, 200, spread=12.0), _rand(rng, 200, 90, spread=12.0)
    P, parts = _split_product(A, B)
    for p in parts:
        assert np.isfinite(p.astype(np.float32)).all()
        assert np.abs(p.astype(np.float32)).max() < 2.0 ** 15
    ref = A.astype(np.float64) @ B.astype(np.float64)
    bound = np.abs(A).astype(np.float64) @ np.abs(B).astype(np.float64)
    assert (np.abs(P - ref) / bound).max() < 2.0 ** -20


def test_entries_far_below_their_row_lose_bits_but_not_the_sum():
    # a row of one large and many tiny entries: the tiny ones keep fewer bits
    # (their lo parts are FP16-subnormal), bounded by 2^-39 of the row's largest
    A = np.full((1, 64), 1e-7, dtype=np.float32)
    A[0, 0] = 1.0
    B = np.ones((64, 1), dtype=np.float32)
    P, _ = _split_product(A, B)
    ref = A.astype(np.float64) @ B.astype(np.float64)
    assert abs(P[0, 0] - ref[0, 0]) <= 64 * 2.0 ** -39 + 2.0 ** -22 * ref[0, 0]
