"""The FP64 complex GEMM's three-real-product form (Gauss; Higham, SIMAX 13,
1992), restated in NumPy (CPU) as the device kernel evaluates it:
T1 = Ar Br, T2 = Ai Bi, T3 = (Ar + Ai)(Br + Bi), Re = T1 - T2,
Im = T3 - T1 - T2, against the four-product form and an extended-precision
reference.  Its error is normwise at the unit roundoff: the imaginary part's
bound is (|Ar| + |Ai|)(|Br| + |Bi|) instead of |Ar||Bi| + |Ai||Br|."""
import numpy as np
import pytest


def _gauss(A, B):
    Ar, Ai, Br, Bi = A.real, A.imag, B.real, B.imag
    T1, T2 = Ar @ Br, Ai @ Bi
    T3 = (Ar + Ai) @ (Br + Bi)
    return (T1 - T2) + 1j * (T3 - T1 - T2)


def _four(A, B):
    Ar, Ai, Br, Bi = A.real, A.imag, B.real, B.imag
    return (Ar @ Br - Ai @ Bi) + 1j * (Ar @ Bi + Ai @ Br)


@pytest.mark.parametrize("case", ["random", "imag_small", "cancelling"])
def test_three_products_stay_at_fp64_accuracy(case):
    rng = np.random.default_rng({"random": 0, "imag_small": 1, "cancelling": 2}[case])
    m, K, n = 96, 256, 80
    A = rng.standard_normal((m, K)) + 1j * rng.standard_normal((m, K))
    B = rng.standard_normal((K, n)) + 1j * rng.standard_normal((K, n))
    if case == "imag_small":
        A = A.real + 1e-6j * A.imag
    if case == "cancelling":
        A = A.real - 1j * A.real + 1e-3j * A.imag   # Ar + Ai nearly cancels
    L = np.clongdouble
    exact = A.astype(L) @ B.astype(L)
    nrm = np.linalg.norm(exact.astype(np.complex128))
    e3 = np.linalg.norm((_gauss(A, B) - exact).astype(np.complex128)) / nrm
    e4 = np.linalg.norm((_four(A, B) - exact).astype(np.complex128)) / nrm
    # normwise: a small multiple of the four-product error, both ~1e-16
    assert e3 < 4e-15 and e3 <= 4 * max(e4, 1e-16), (e3, e4)
    # the componentwise bound of the imaginary part
    absA = np.abs(A.real) + np.abs(A.imag)
    absB = np.abs(B.real) + np.abs(B.imag)
    bound = 4 * K * 2.0 ** -53 * (absA @ absB)
    assert np.all(np.abs((_gauss(A, B) - exact).imag.astype(np.float64)) <= bound)
