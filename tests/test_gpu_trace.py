"""Tensor-core Fisher contraction (trace mode) against an FP64 torch reference.

F[p, q] = scale sum_t sum_{k, l} X_{a_t}[p, k, l] Y_{b_t}[q, k, l] over BF16
split planes.  The kernel accumulates in FP32 inside TMEM for 4 k-tiles and
promotes to FP64, so its error is a few FP32 roundings of the magnitude sum:
the bar is 2e-6 of sum |X_0| |Y_0| per entry.  Cases: the six products of
three planes, and the four of two planes that the mixed Fisher uses on its
stored A_b slabs (Y the transposes of X, as A_p[l, k]).
"""

import ctypes

import pytest
import torch

pytestmark = pytest.mark.gpu

X6 = ((0, 0, 1, 0, 1, 2), (0, 1, 0, 2, 1, 0))
X4 = ((0, 0, 1, 1), (0, 1, 0, 1))


def _arr(v):
    a = (ctypes.c_int * len(v))(*v)
    return a, ctypes.cast(a, ctypes.c_void_p)


def _split(lib, A, ld, planes):
    """BF16 planes of a (P, K1, K2) FP64 array, rows padded to ld."""
    P, K1, K2 = A.shape
    flat = A.reshape(P * K1, K2).contiguous()
    out = torch.zeros((planes, P * K1, ld), dtype=torch.bfloat16, device="cuda")
    assert lib.cf_split_bf16(P * K1, K2, flat.data_ptr(), K2, planes, out.data_ptr(), ld, P * K1 * ld,
                             torch.cuda.current_stream().cuda_stream) == 0
    return out


def _ref(Xp, Yp, terms, P, K1, K2, scale):
    Xd = Xp.double().reshape(Xp.shape[0], P, K1, -1)[..., :K2]
    Yd = Yp.double().reshape(Yp.shape[0], P, K1, -1)[..., :K2]
    F = torch.zeros((P, P), dtype=torch.float64, device="cuda")
    for a, b in zip(*terms):
        F += torch.einsum("pkl,qkl->pq", Xd[a], Yd[b])
    mag = torch.einsum("pkl,qkl->pq", Xd[0].abs(), Yd[0].abs())
    return scale * F, scale * mag


@pytest.mark.parametrize("pairs", [1, 0])
@pytest.mark.parametrize("terms,planes", [(X6, 3), (X4, 2)])
@pytest.mark.parametrize("P,K", [(40, 96), (150, 72), (230, 40)])
def test_trace_matches_fp64(P, K, terms, planes, pairs):
    """pairs = 1: P > 128 runs on CTA pairs (256-row tiles); 0: one CTA per tile."""
    from cosmoforge_b200 import _lib

    lib = _lib.lib()
    prev = lib.cf_umma_set_trace_pairs(pairs)
    g = torch.Generator(device="cuda").manual_seed(P + K)
    # A_p with a common smooth part, so the contraction has cancellation
    base = torch.randn((K, K), dtype=torch.float64, device="cuda", generator=g)
    A = base[None] + 0.3 * torch.randn((P, K, K), dtype=torch.float64, device="cuda", generator=g)
    ld = (K + 7) // 8 * 8
    Xp = _split(lib, A, ld, planes)
    Yp = _split(lib, A.transpose(1, 2).contiguous(), ld, planes)
    pmap = torch.arange(P, dtype=torch.int32, device="cuda")
    err = torch.zeros(1, dtype=torch.int32, device="cuda")
    st = torch.cuda.current_stream().cuda_stream
    ref, mag = _ref(Xp, Yp, terms, P, K, K, 0.5)
    F = torch.zeros((P, P), dtype=torch.float64, device="cuda")
    ka, pa = _arr(terms[0])
    kb, pb = _arr(terms[1])
    rc = lib.cf_umma_trace_bf16_mapped(P, P, K, K, len(terms[0]), pa, pb, Xp.data_ptr(), K * ld, ld, P * K * ld,
                                       planes, Yp.data_ptr(), K * ld, ld, P * K * ld, planes, 0.5, F.data_ptr(), P,
                                       pmap.data_ptr(), pmap.data_ptr(), 0, 0, err.data_ptr(), st)
    lib.cf_umma_set_trace_pairs(prev)
    assert rc == 0
    torch.cuda.synchronize()
    assert int(err.item()) == 0
    assert bool(((F - ref).abs() <= 2e-6 * mag).all()), float(((F - ref).abs() / mag).max())
    # against the exact FP64 contraction of A: the planes' rounding (2^-17 per
    # entry with two planes, unbiased) averages over the K^2 products
    exact = 0.5 * torch.einsum("pkl,qlk->pq", A, A)
    emag = 0.5 * torch.einsum("pkl,qlk->pq", A.abs(), A.abs())
    assert bool(((F - exact).abs() <= (2e-6 if planes == 3 else 2e-5) * emag).all())
