"""The coarsest solve's diagonal-block algebra, in NumPy (no GPU).

`topogpu_b200/csrc/coarsest.cu` splits the band Cholesky factor L of the
coarsest operator into P diagonal blocks (boundaries on 32-row panels, at
least max(4 band, 512) rows each, at most 8 blocks, every block at least
`band` rows), keeps W_q = L_qq^-1 and the couplings G_q = W_q[:, :band] Lc_q
and H_q = (Lc_{q+1} W_q[m-band:, :])^T, and solves K z = r as
  y_q = W_q r_q - G_q y_{q-1}[m_{q-1}-band:]          (q = 0 .. P-1)
  z_q = W_q^T y_q - H_q z_{q+1}[:band]                (q = P-1 .. 0).
This restates that partition and recurrence and checks them against a dense
solve on banded SPD matrices, including the corner structure they rely on.
The device path itself is checked in tests/test_gpu_parity.py: V-cycles
with one and three blocks against the oracle's dense Cholesky, and the
160x80x80 solutions (four blocks) against the oracle's FP64 operator.
"""

import numpy as np
import pytest


def partition(n, band, maxb=8, cnb=32):
    """Block boundaries as coarsest_alloc chooses them."""
    P = max(1, min(maxb, n // max(4 * band, 512)))
    while True:
        b = [0] + [q * n // P // cnb * cnb for q in range(1, P)] + [n]
        if all(b[q + 1] - b[q] >= max(band, 1) for q in range(P)) or P == 1:
            return b
        P -= 1


def banded_spd(n, band, seed):
    rng = np.random.default_rng(seed)
    A = np.zeros((n, n))
    for i in range(n):
        lo = max(0, i - band)
        A[i, lo:i] = rng.uniform(-1, 1, i - lo) * 0.01
    A = A + A.T
    A[np.diag_indices(n)] = 4.0 + band * 0.02
    return A


def block_solve(L, b, band, r):
    P = len(b) - 1
    W = [np.linalg.inv(L[b[q]:b[q + 1], b[q]:b[q + 1]]) for q in range(P)]

    def Lc(q):  # rows b[q] .. b[q]+band-1, columns b[q]-band .. b[q]-1
        return L[b[q]:b[q] + band, b[q] - band:b[q]]

    G = [None] + [W[q][:, :band] @ Lc(q) for q in range(1, P)]
    H = [(Lc(q + 1) @ W[q][-band:, :]).T for q in range(P - 1)] + [None]
    y = np.zeros_like(r)
    for q in range(P):
        v = W[q] @ r[b[q]:b[q + 1]]
        if q > 0:
            v -= G[q] @ y[b[q] - band:b[q]]
        y[b[q]:b[q + 1]] = v
    z = np.zeros_like(r)
    for q in reversed(range(P)):
        v = W[q].T @ y[b[q]:b[q + 1]]
        if q < P - 1:
            v -= H[q] @ z[b[q + 1]:b[q + 1] + band]
        z[b[q]:b[q + 1]] = v
    return z, P


@pytest.mark.parametrize("n,band,P", [(2200, 101, 4), (4100, 128, 8), (1500, 300, 1), (1200, 37, 2), (3000, 256, 2)])
def test_partition_rule(n, band, P):
    b = partition(n, band)
    assert len(b) - 1 == P
    assert b[0] == 0 and b[-1] == n
    assert all(x % 32 == 0 for x in b[1:-1])
    assert all(b[q + 1] - b[q] >= band for q in range(len(b) - 1))


@pytest.mark.parametrize("n,band,seed", [(2200, 101, 0), (1200, 37, 1), (3000, 256, 2), (700, 90, 3)])
def test_block_recurrence_solves_the_system(n, band, seed):
    A = banded_spd(n, band, seed)
    L = np.linalg.cholesky(A)
    b = partition(n, band)
    # the coupling of block q+1 to block q is its band x band corner, upper
    # triangular in corner indices (row b+k reaches columns b-band+l, l >= k)
    for q in range(1, len(b) - 1):
        blk = L[b[q]:b[q + 1], :b[q]]
        corner = np.zeros_like(blk, dtype=bool)
        corner[:band, -band:] = True
        assert not blk[~corner].any()
        assert not np.tril(L[b[q]:b[q] + band, b[q] - band:b[q]], -1).any()
    r = np.random.default_rng(seed + 10).standard_normal(n)
    z, P = block_solve(L, b, band, r)
    ref = np.linalg.solve(A, r)
    assert np.linalg.norm(z - ref) / np.linalg.norm(ref) < 1e-12
