"""Host-side checks of the mixed Fisher's split-product schemes (no GPU).

The GEMM forms A_b from three BF16 planes per operand (six products); the
traces read A_b stored as two planes with the products (0,0), (0,1), (1,0),
(1,1).  The BF16 rounding is emulated here with round-to-nearest-even on the
top 16 bits of the FP32 encoding, so the arithmetic of the schemes is checked
on the CPU against FP64.
"""

import numpy as np

from cosmoforge_b200 import engine_mixed


def _bf16(x):
    b = np.asarray(x, dtype=np.float32).view(np.uint32).astype(np.uint64)
    b = (b + 0x7FFF + ((b >> 16) & 1)) & 0xFFFF0000
    return b.astype(np.uint32).view(np.float32).astype(np.float64)


def _planes(x, n):
    out, r = [], np.asarray(x, dtype=np.float64)
    for _ in range(n):
        h = _bf16(r)
        out.append(h)
        r = r - h
    return out


def test_scheme_tables_are_consistent():
    for name, (planes, ta, tb) in engine_mixed.SCHEMES.items():
        tp, qa, qb = engine_mixed.TRACE[name]
        assert len(ta) == len(tb) and len(qa) == len(qb)
        assert (ta[0], tb[0]) == (0, 0) and (qa[0], qb[0]) == (0, 0)
        assert max(ta + tb) < planes and max(qa + qb) < tp <= planes
        assert len(set(zip(ta, tb))) == len(ta) and len(set(zip(qa, qb))) == len(qa)
    # the square of the second planes stays in the six-product scheme's trace
    _, qa, qb = engine_mixed.TRACE["bf16x6"]
    assert (1, 1) in set(zip(qa, qb))


def test_two_plane_trace_matches_fp64():
    """1/2 sum_kl A_p[k,l] A_q[l,k] from two planes and four products is within
    2e-5 of the magnitude sum of the FP64 contraction (the planes' rounding
    averages over the K^2 products)."""
    rng = np.random.default_rng(7)
    P, K = 5, 48
    base = rng.standard_normal((K, K))
    A = base[None] + 0.3 * rng.standard_normal((P, K, K))
    exact = 0.5 * np.einsum("pkl,qlk->pq", A, A)
    mag = 0.5 * np.einsum("pkl,qlk->pq", np.abs(A), np.abs(A))
    tp, qa, qb = engine_mixed.TRACE["bf16x6"]
    X = _planes(A, tp)
    XT = _planes(A.transpose(0, 2, 1), tp)
    F = sum(0.5 * np.einsum("pkl,qkl->pq", X[a], XT[b]) for a, b in zip(qa, qb))
    assert np.all(np.abs(F - exact) <= 2e-5 * mag)


def test_six_product_gemm_keeps_24_bits():
    """sum_t A_{a_t} B_{b_t} with three planes per operand agrees with the FP64
    product to ~2^-24 of sum |A| |B|."""
    rng = np.random.default_rng(3)
    A = rng.standard_normal((40, 64))
    B = rng.standard_normal((64, 30))
    planes, ta, tb = engine_mixed.SCHEMES["bf16x6"]
    Ap, Bp = _planes(A, planes), _planes(B, planes)
    C = sum(Ap[a] @ Bp[b] for a, b in zip(ta, tb))
    assert np.all(np.abs(C - A @ B) <= 2e-7 * (np.abs(A) @ np.abs(B)))
