"""tcgen05 split-precision GEMM against an FP64 torch reference of the same product.

Tolerances: one BF16 product (0,0) of BF16-rounded inputs is exact in FP32
up to the FP32 accumulation (1e-5 relative); BF16x3 keeps ~16 significant
bits (2e-4 relative of max |C| for random inputs with cancellation);
BF16x6 ~24 bits (2e-6).
"""

import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu

X3 = ([0, 0, 1], [0, 1, 0])
X6 = ([0, 0, 1, 0, 1, 2], [0, 1, 0, 2, 1, 0])


def _planes(lib, X, planes, ld):
    R, C = X.shape
    out = torch.zeros((planes, R, ld), dtype=torch.bfloat16, device="cuda")
    assert lib.cf_split_bf16(R, C, X.data_ptr(), X.stride(0), planes, out.data_ptr(), ld, R * ld,
                             torch.cuda.current_stream().cuda_stream) == 0
    return out


def _gemm(lib, A, B, terms, planes, with_x=False):
    import ctypes

    M, K = A.shape
    N = B.shape[0]
    ld = (K + 7) // 8 * 8
    Ap = _planes(lib, A, planes, ld)
    Bp = _planes(lib, B, planes, ld)
    ta = (ctypes.c_int * len(terms[0]))(*terms[0])
    tb = (ctypes.c_int * len(terms[1]))(*terms[1])
    Cf = torch.zeros((M, N), dtype=torch.float32, device="cuda")
    err = torch.zeros(1, dtype=torch.int32, device="cuda")
    X = XT = None
    if with_x:
        ldx = (N + 7) // 8 * 8
        ldxt = (M + 7) // 8 * 8
        X = torch.zeros((2, M, ldx), dtype=torch.bfloat16, device="cuda")
        XT = torch.zeros((2, N, ldxt), dtype=torch.bfloat16, device="cuda")
    rc = lib.cf_umma_gemm_bf16(
        M, N, K, len(terms[0]), ctypes.cast(ta, ctypes.c_void_p), ctypes.cast(tb, ctypes.c_void_p),
        Ap.data_ptr(), ld, M * ld, planes, Bp.data_ptr(), ld, N * ld, planes,
        X.data_ptr() if with_x else None, X.shape[2] if with_x else 0, X[0].numel() if with_x else 0, 2,
        XT.data_ptr() if with_x else None, XT.shape[2] if with_x else 0, XT[0].numel() if with_x else 0,
        Cf.data_ptr(), N, err.data_ptr(), torch.cuda.current_stream().cuda_stream)
    assert rc == 0
    torch.cuda.synchronize()
    assert int(err.item()) == 0
    return Cf, X, XT, Ap[:, :, :K], Bp[:, :, :K]


@pytest.mark.parametrize("M,N,K", [(256, 384, 192), (200, 300, 100), (128, 512, 1024)])
def test_umma_single_product_matches_rounded_inputs(M, N, K):
    from cosmoforge_b200 import _lib

    lib = _lib.lib()
    g = torch.Generator(device="cuda").manual_seed(M + N + K)
    A = torch.randn((M, K), dtype=torch.float64, device="cuda", generator=g)
    B = torch.randn((N, K), dtype=torch.float64, device="cuda", generator=g)
    Cf, _, _, Ap, Bp = _gemm(lib, A, B, ([0], [0]), 1)
    # the exact BF16 inputs the kernel consumed (x_0 = bf16(x), rounded once from FP64)
    ref = Ap[0].double() @ Bp[0].double().T
    err = (Cf.double() - ref).abs().max() / ref.abs().max()
    assert err < 1e-5, float(err)


# (M, N, K): one tile; ragged sizes with a partial 32-wide k-slice; several
# promotion chunks per tile and more tiles than SMs (persistent CTAs walk 2).
SHAPES = [(384, 640, 512), (200, 300, 100), (2048, 4352, 2112)]


# GEMM forms (cf_umma_set_all_planes): 1 = all planes of a 32-wide k-slice per
# stage, 2 = the same on CTA pairs (three planes; two planes fall back to 1),
# 0 = 64-wide k-tiles term by term.
@pytest.mark.parametrize("form", [1, 2, 0])
@pytest.mark.parametrize("M,N,K", SHAPES)
@pytest.mark.parametrize("terms,planes,tol", [(X3, 2, 2e-4), (X6, 3, 2e-6), (X3, 3, 2e-4)])
def test_umma_split_products(terms, planes, tol, M, N, K, form):
    from cosmoforge_b200 import _lib

    lib = _lib.lib()
    g = torch.Generator(device="cuda").manual_seed(7 + M + K)
    A = torch.randn((M, K), dtype=torch.float64, device="cuda", generator=g)
    B = torch.randn((N, K), dtype=torch.float64, device="cuda", generator=g)
    prev = lib.cf_umma_set_all_planes(form)
    try:
        Cf, _, _, _, _ = _gemm(lib, A, B, terms, planes)
    finally:
        lib.cf_umma_set_all_planes(prev)
    ref = A @ B.T
    err = (Cf.double() - ref).abs().max() / ref.abs().max()
    assert err < tol, float(err)


def test_umma_split_outputs_and_transpose():
    from cosmoforge_b200 import _lib

    lib = _lib.lib()
    g = torch.Generator(device="cuda").manual_seed(3)
    M, N, K = 256, 272, 128
    A = torch.randn((M, K), dtype=torch.float64, device="cuda", generator=g)
    B = torch.randn((N, K), dtype=torch.float64, device="cuda", generator=g)
    Cf, X, XT, _, _ = _gemm(lib, A, B, X3, 2, with_x=True)
    xs = X[0, :, :N].double() + X[1, :, :N].double()
    xts = XT[0, :, :M].double() + XT[1, :, :M].double()
    c = Cf.double()
    assert ((xs - c).abs() <= 2.0**-15 * c.abs() + 1e-30).all()
    assert torch.equal(xs, xts.T)
