"""The partition of the cluster L D L^T diagonal-block kernel, restated in NumPy.

`ldlt_diag_cluster_kernel` (csrc/lu.cu) factors a jb x jb diagonal block
(jb <= 256) on 8 CTAs, CTA q holding block rows 32q..32q+31.  Per 32-column
sub-panel p: (A) CTA p eliminates the 32 x 32 diagonal sub-block column by
column, keeping the unscaled column entries U; (B) every CTA q > p takes U
and the pivots from CTA p and eliminates the sub-panel columns of its own
rows; (C) every CTA q > p updates its rows' lower triangle right of the
sub-panel with T[k][c] = d_k l[c][k] gathered from CTAs p+1..q.  This test
walks the same phases, ownership and index ranges in complex128 and checks
the result against a plain column-by-column L D L^T, for full and ragged
blocks (partial last sub-panels, CTAs without rows), so a change of the
partition shows up without a GPU."""
import numpy as np
import pytest

ROWS, CTAS = 32, 8


def _plain_ldlt(a):
    a = a.copy()
    n = a.shape[0]
    for k in range(n):
        col = a[:, k].copy()
        for i in range(k + 1, n):
            a[i, k + 1:i + 1] -= col[i] / col[k] * col[k + 1:i + 1]
            a[i, k] = col[i] / col[k]
    return a


def _cluster_ldlt(blk):
    jb = blk.shape[0]
    # CTA q: rows r0..r0+nr-1 of the block, columns 0..min(r0+32, jb)-1
    S, U = [], []
    for q in range(CTAS):
        r0 = q * ROWS
        nr = max(0, min(ROWS, jb - r0))
        s = np.full((ROWS, CTAS * ROWS), np.nan + 0j)
        s[:nr, :min(r0 + ROWS, jb)] = blk[r0:r0 + nr, :min(r0 + ROWS, jb)]
        S.append(s)
        U.append(np.full((ROWS, ROWS), np.nan + 0j))
    for p in range((jb + ROWS - 1) // ROWS):
        c0 = p * ROWS
        w = min(ROWS, jb - c0)
        # A. the diagonal sub-block on CTA p (rows 0..w-1 of that CTA)
        x = S[p][:w, c0:c0 + w].copy()
        for jj in range(w):
            col, d = x[:, jj].copy(), x[jj, jj]
            for i in range(jj + 1, w):
                l = col[i] / d
                x[i, jj + 1:] -= l * col[jj + 1:]
                U[p][i, jj] = col[i]
                x[i, jj] = l
        low = np.tril(np.ones((w, w), bool))
        S[p][:w, c0:c0 + w][low] = x[low]
        # B. the rows below, CTA by CTA, from CTA p's U and pivots
        dk = np.array([S[p][t, c0 + t] for t in range(w)])
        for q in range(p + 1, CTAS):
            nr = max(0, min(ROWS, jb - q * ROWS))
            for i in range(nr):
                xr = S[q][i, c0:c0 + w].copy()
                for jj in range(w):
                    l = xr[jj] / dk[jj]
                    xr[jj + 1:w] -= l * U[p][jj + 1:w, jj]
                    xr[jj] = l
                S[q][i, c0:c0 + w] = xr
        # C. the lower triangle right of the sub-panel, own rows only
        for q in range(p + 1, CTAS):
            r0, nr = q * ROWS, max(0, min(ROWS, jb - q * ROWS))
            if nr == 0:
                continue
            assert w == ROWS  # a partial sub-panel is the last one: no CTA has rows below it
            cs = c0 + w
            nc = r0 + ROWS - cs
            assert nc // ROWS == q - p <= 7
            T = np.zeros((w, nc), complex)
            for c in range(nc):
                row = cs + c
                if row < jb:
                    owner = row // ROWS
                    assert p + 1 <= owner <= q
                    T[:, c] = dk * S[owner][row % ROWS, c0:c0 + w]
            for i in range(nr):
                cols = np.arange(cs, r0 + i + 1)
                acc = S[q][i, cols]
                assert not np.isnan(acc).any()
                S[q][i, cols] = acc - S[q][i, c0:c0 + w] @ T[:, cols - cs]
    out = blk.copy()
    for q in range(CTAS):
        r0, nr = q * ROWS, max(0, min(ROWS, jb - q * ROWS))
        for r in range(nr):
            out[r0 + r, :r0 + r + 1] = S[q][r, :r0 + r + 1]
    return out


@pytest.mark.parametrize("jb", [256, 200, 100, 33, 32, 7])
def test_cluster_partition_matches_plain_ldlt(jb):
    rng = np.random.default_rng(jb)
    m = rng.standard_normal((jb, jb)) + 1j * rng.standard_normal((jb, jb))
    m = m + m.T + 8 * np.sqrt(jb) * np.eye(jb)
    got = _cluster_ldlt(m)
    ref = _plain_ldlt(m)
    low = np.tril(np.ones((jb, jb), bool))
    assert np.abs(got[low] - ref[low]).max() <= 1e-13 * np.abs(ref[low]).max()
    # the upper triangle is not touched
    assert np.array_equal(np.triu(got, 1), np.triu(m, 1))
