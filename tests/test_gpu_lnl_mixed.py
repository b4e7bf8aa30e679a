"""Mixed-precision pixel likelihood (FP32 Cholesky, FP64-refined chi2).

Checked against the reference's own outputs on the golden fixtures (the
same cases the FP64 path matches to 1e-10) and against the FP64 device path
on random SPD batches.  Tolerances, measured on B200 with margin:
  chi2 (one FP64 refinement step)   relative 1e-8
  ln|C| and lnL (FP32 factor)       absolute 3e-3 (lnL values are O(7e3): FP32
                                    rounding of the Schur complements, ~1e-4 per
                                    entry, against pivots near the noise level)
  FP32 factor L                      relative 1e-5 of max |L| on well-conditioned batches
"""

import numpy as np
import pytest
import torch

from cosmoforge_b200 import workloads
from cosmoforge_b200.layout import build_layout
from golden_cases import load, params_of

pytestmark = pytest.mark.gpu

CHI2_REL = 1e-8
LNL_ABS = 3e-3


def _spd_batch(n, batch, seed):
    g = torch.Generator(device="cuda").manual_seed(seed)
    R = torch.randn((batch, n, n), dtype=torch.float64, device="cuda", generator=g)
    return R @ R.transpose(1, 2) / n + torch.eye(n, dtype=torch.float64, device="cuda")


@pytest.mark.parametrize("group", [4, 2])
@pytest.mark.parametrize("n,batch", [(200, 3), (333, 2), (1000, 3), (1312, 2)])
def test_potrf_f32_matches_fp64_factor(n, batch, group):
    """Passes of 4 (default) or 2 panels: ragged last passes (n not a multiple
    of 256 or 128), narrow in-pass updates of K = 64 .. 192."""
    from cosmoforge_b200 import _lib

    lib = _lib.lib()
    C = _spd_batch(n, batch, n)
    A = C.float().contiguous()
    info = torch.zeros(batch, dtype=torch.int32, device="cuda")
    work = torch.empty(lib.cf_potrf_f32_workspace(n, batch) // 4 + 1, dtype=torch.float32, device="cuda")
    prev = lib.cf_potrf_f32_set_group(group)
    try:
        assert lib.cf_potrf_f32(n, A.data_ptr(), n, n * n, batch, work.data_ptr(), info.data_ptr(),
                                torch.cuda.current_stream().cuda_stream) == 0
    finally:
        lib.cf_potrf_f32_set_group(prev)
    assert int(info.abs().max()) == 0
    L64 = torch.linalg.cholesky(C)
    L32 = torch.tril(A.double())
    err = float((L32 - L64).abs().max() / L64.abs().max())
    print(f"n={n}: factor error {err:.2e}")
    assert err <= 1e-5


def test_potrf_f32_reports_first_bad_pivot():
    from cosmoforge_b200 import _lib

    lib = _lib.lib()
    n, batch = 150, 3
    C = _spd_batch(n, batch, 5)
    C[1, 70, :] = 0.0
    C[1, :, 70] = 0.0
    C[1, 70, 70] = -1.0
    A = C.float().contiguous()
    info = torch.zeros(batch, dtype=torch.int32, device="cuda")
    work = torch.empty(lib.cf_potrf_f32_workspace(n, batch) // 4 + 1, dtype=torch.float32, device="cuda")
    assert lib.cf_potrf_f32(n, A.data_ptr(), n, n * n, batch, work.data_ptr(), info.data_ptr(),
                            torch.cuda.current_stream().cuda_stream) == 0
    assert info.cpu().tolist() == [0, 71, 0]


def _check(chi2, lnl, ref_chi2, ref_lnl, tag):
    e_chi2 = float(np.max(np.abs(chi2 / ref_chi2 - 1)))
    e_lnl = float(np.max(np.abs(lnl - ref_lnl)))
    print(f"{tag}: chi2 rel {e_chi2:.2e}  |dlnL| {e_lnl:.2e}")
    assert e_chi2 <= CHI2_REL
    assert e_lnl <= LNL_ABS


def test_lnl_mixed_fortran_picslike():
    from cosmoforge_b200 import engine

    d = load("fortran_picslike_nside8_B")
    L = build_layout(params_of(d), d["mask"], d["beam"])
    E = engine.Engine(L)
    cl = np.stack([L.smoothed_cl_table({"BB": c}) for c in d["point_cl_BB"]])
    chi2, ld, lnl, info = E.lnl(cl, torch.from_numpy(d["noise"]).cuda(), torch.from_numpy(d["maps"]),
                                precision="mixed")
    assert int(info.abs().max()) == 0
    _check(chi2.cpu().numpy()[:, 0], lnl.cpu().numpy()[:, 0], d["ref_chi2"][:, 0], d["ref_lnl"][:, 0],
           "fortran_picslike")


def test_lnl_mixed_tqu_batch():
    from cosmoforge_b200 import engine

    d = load("picslike_tqu_nside8")
    L = build_layout(params_of(d), d["mask"], d["beam"])
    E = engine.Engine(L)
    cl = np.stack([L.smoothed_cl_table(workloads.model_cls(t, L.lmax_signal)) for t in d["thetas"]])
    N = torch.from_numpy(np.diag(d["noise_diag"])).cuda()
    chi2, ld, lnl, info = E.lnl(cl, N, torch.from_numpy(d["maps"]), noise_scale=d["thetas"][:, 4],
                                precision="mixed")
    assert int(info.abs().max()) == 0
    _check(chi2.cpu().numpy()[:, 0], lnl.cpu().numpy()[:, 0], d["ref_chi2"][:, 0], d["ref_lnl"][:, 0],
           "picslike_tqu")


@pytest.mark.parametrize("build", ["direct", "basis"])
def test_lnl_mixed_config3_sobol_batch(build):
    """256 Sobol points of the five-parameter box against the FP64 device path;
    the refinement reads the FP64 C in both builds (the basis build writes the
    FP32 copy to factor from the same GEMM epilogue)."""
    from cosmoforge_b200 import engine

    pb = workloads.config3()
    L = build_layout(pb.params, pb.mask, pb.beam)
    E = engine.Engine(L)
    th = workloads.sobol_points(256, seed=1)
    cl = np.stack([L.smoothed_cl_table(workloads.model_cls(t, L.lmax_signal)) for t in th])
    N = torch.from_numpy(pb.noise).cuda()
    g = torch.Generator(device="cuda").manual_seed(0)
    X = torch.randn((L.n, 2), dtype=torch.float64, device="cuda", generator=g) * 10.0
    c64, _, l64, i64 = E.lnl(cl, N, X, noise_scale=th[:, 4], build=build)
    cm, _, lm, im = E.lnl(cl, N, X, noise_scale=th[:, 4], precision="mixed", build=build)
    assert int(i64.abs().max()) == 0 and int(im.abs().max()) == 0
    _check(cm.cpu().numpy(), lm.cpu().numpy(), c64.cpu().numpy(), l64.cpu().numpy(), f"config3 sobol {build}")


@pytest.mark.parametrize("maps", ["drawn", "synthetic"])
def test_lnl_mixed_tensor_core_build(maps):
    """build "basis_tc": C(theta) in FP32 from BF16x6 products on the tensor
    cores and the refinement against that FP32 C, so chi2 is first order in
    C's rounding.  On maps drawn from the fiducial covariance (chi2 ~ n
    across the box): chi2 to 1e-5 relative and lnL to 1e-2; on the synthetic
    maps of the test above (chi2 ~ 8 n): 2e-5 and 0.05."""
    from cosmoforge_b200 import engine, qube

    pb = workloads.config3()
    L = build_layout(pb.params, pb.mask, pb.beam)
    E = engine.Engine(L)
    N = torch.from_numpy(pb.noise).cuda()
    if maps == "drawn":
        X = qube.draw_maps(L, pb.cls, N, 2, seed=3)
    else:
        g = torch.Generator(device="cuda").manual_seed(0)
        X = torch.randn((L.n, 2), dtype=torch.float64, device="cuda", generator=g) * 10.0
    th = workloads.sobol_points(128, seed=2)
    cl = np.stack([L.smoothed_cl_table(workloads.model_cls(t, L.lmax_signal)) for t in th])
    c64, _, l64, _ = E.lnl(cl, N, X, noise_scale=th[:, 4], build="basis")
    cm, _, lm, im = E.lnl(cl, N, X, noise_scale=th[:, 4], precision="mixed", build="basis_tc")
    assert int(im.abs().max()) == 0
    e_chi2 = float((cm / c64 - 1).abs().max())
    e_lnl = float((lm - l64).abs().max())
    print(f"basis_tc, {maps} maps: chi2 rel {e_chi2:.2e}  |dlnL| {e_lnl:.2e}")
    bars = (1e-5, 1e-2) if maps == "drawn" else (2e-5, 0.05)
    assert e_chi2 <= bars[0] and e_lnl <= bars[1]
    with pytest.raises(ValueError):
        E.lnl(cl[:2], N, X, precision="fp64", build="basis_tc")


@pytest.mark.parametrize("dtype", [torch.float32, torch.float64])
def test_potrf_batch_copies_bitwise_identical(dtype):
    """Every copy of one matrix in a batch gets the same factor, bit for bit.

    Guards the diagonal-block kernels against intra-CTA races: 192 copies of
    an n = 520 problem run 1728 diagonal-block factorisations.
    """
    from cosmoforge_b200 import _lib

    lib = _lib.lib()
    n, batch = 520, 192
    C = _spd_batch(n, 1, 11).to(dtype).repeat(batch, 1, 1).contiguous()
    info = torch.zeros(batch, dtype=torch.int32, device="cuda")
    st = torch.cuda.current_stream().cuda_stream
    if dtype == torch.float32:
        work = torch.empty(lib.cf_potrf_f32_workspace(n, batch) // 4 + 1, dtype=dtype, device="cuda")
        rc = lib.cf_potrf_f32(n, C.data_ptr(), n, n * n, batch, work.data_ptr(), info.data_ptr(), st)
    else:
        work = torch.empty(lib.cf_potrf_workspace(n, batch) // 8 + 1, dtype=dtype, device="cuda")
        rc = lib.cf_potrf(n, C.data_ptr(), n, n * n, batch, work.data_ptr(), info.data_ptr(), st)
    assert rc == 0
    assert int(info.abs().max()) == 0
    Lf = torch.tril(C)
    assert bool((Lf == Lf[:1]).all())


@pytest.mark.parametrize("M,N,K,batch,lower", [(300, 300, 128, 3, 0), (1184, 1184, 128, 2, 1), (517, 64, 64, 4, 0),
                                               (130, 200, 96, 1, 0), (64, 64, 200, 1, 0)])
def test_sgemm_bf16x6_matches_fp64_product(M, N, K, batch, lower):
    """cf_sgemm_bf16x6 (BF16x6 split products on tcgen05) against the product
    of the same FP32 operands in FP64: ~24-bit products, so the error must sit
    at the FP32 level (2e-6 of the largest |A||B| sum); alpha / beta, ragged
    tiles, batches and skipped upper tiles included."""
    from cosmoforge_b200 import _lib

    lib = _lib.lib()
    g = torch.Generator(device="cuda").manual_seed(M + N + K)
    A = torch.randn((batch, M, K), device="cuda", generator=g)
    B = A if lower else torch.randn((batch, N, K), device="cuda", generator=g)
    C0 = torch.randn((batch, M, N), device="cuda", generator=g)
    ref = -torch.bmm(A.double(), B.double().transpose(1, 2)) + 0.5 * C0.double()
    scale = torch.bmm(A.double().abs(), B.double().abs().transpose(1, 2)).max()
    prev = lib.cf_sgemm_bf16x6_set_stages(1)
    try:
        for stages in (1, 2):
            lib.cf_sgemm_bf16x6_set_stages(stages)
            C = C0.clone()
            info = torch.zeros(batch, dtype=torch.int32, device="cuda")
            rc = lib.cf_sgemm_bf16x6(M, N, K, -1.0, A.data_ptr(), K, M * K, B.data_ptr(), K, N * K, 0.5, C.data_ptr(),
                                     N, M * N, batch, lower, info.data_ptr(), torch.cuda.current_stream().cuda_stream)
            assert rc == 0
            torch.cuda.synchronize()
            assert int(info.abs().max()) == 0
            if lower:  # tiles strictly above the diagonal are skipped: only rows >= the tile's columns are written
                r = torch.arange(M, device="cuda")[:, None] // 128
                c = torch.arange(N, device="cuda")[None, :] // 128
                keep = (c <= r)[None]
                err = ((C.double() - ref).abs() * keep).max()
                assert bool((C[~keep.expand_as(C)] == C0[~keep.expand_as(C0)]).all())
            else:
                err = (C.double() - ref).abs().max()
            assert float(err / scale) <= 2e-6, (stages, float(err / scale))
    finally:
        lib.cf_sgemm_bf16x6_set_stages(prev)


def test_sgemm_bf16x6_timed_out_wait_sets_info():
    from cosmoforge_b200 import _lib

    lib = _lib.lib()
    A = torch.randn((2, 256, 256), device="cuda")
    C = torch.zeros((2, 256, 256), device="cuda")
    info = torch.zeros(2, dtype=torch.int32, device="cuda")
    st = torch.cuda.current_stream().cuda_stream
    lib.cf_sgemm_bf16x6_set_wait_limit(0)
    try:
        assert lib.cf_sgemm_bf16x6(256, 256, 256, 1.0, A.data_ptr(), 256, 65536, A.data_ptr(), 256, 65536, 0.0,
                                   C.data_ptr(), 256, 65536, 2, 0, info.data_ptr(), st) == 0
        torch.cuda.synchronize()
    finally:
        lib.cf_sgemm_bf16x6_set_wait_limit(-1)
    assert set(info.cpu().tolist()) == {_lib.CF_ERR_TIMEOUT}
    info.zero_()
    assert lib.cf_sgemm_bf16x6(256, 256, 256, 1.0, A.data_ptr(), 256, 65536, A.data_ptr(), 256, 65536, 0.0,
                               C.data_ptr(), 256, 65536, 2, 0, info.data_ptr(), st) == 0
    torch.cuda.synchronize()
    assert int(info.abs().max()) == 0
    ref = torch.bmm(A.double(), A.double().transpose(1, 2))
    assert float((C.double() - ref).abs().max() / ref.abs().max()) <= 2e-6


@pytest.mark.parametrize("n,batch", [(1312, 8), (200, 64)])
def test_potrf_f32_tensor_cores_vs_simt(n, batch):
    """The FP32 factor with tensor-core products stays as close to the FP64
    factor as the SIMT FP32 factor does (both at FP32 rounding level)."""
    from cosmoforge_b200 import _lib

    lib = _lib.lib()
    g = torch.Generator(device="cuda").manual_seed(n)
    R = torch.randn((batch, n, n), dtype=torch.float64, device="cuda", generator=g)
    A64 = R @ R.transpose(1, 2) / n + torch.eye(n, dtype=torch.float64, device="cuda")
    L64 = torch.linalg.cholesky(A64)
    st = torch.cuda.current_stream().cuda_stream
    errs = {}
    prev = lib.cf_potrf_f32_set_tensor(1)
    try:
        for mode in (1, 0):
            lib.cf_potrf_f32_set_tensor(mode)
            A = A64.float().contiguous()
            work = torch.empty(lib.cf_potrf_f32_workspace(n, batch) // 4 + 1, dtype=torch.float32, device="cuda")
            info = torch.zeros(batch, dtype=torch.int32, device="cuda")
            assert lib.cf_potrf_f32(n, A.data_ptr(), n, n * n, batch, work.data_ptr(), info.data_ptr(), st) == 0
            torch.cuda.synchronize()
            assert int(info.abs().max()) == 0
            Lf = torch.tril(A.double())
            errs[mode] = float((Lf - L64).abs().max() / L64.abs().max())
    finally:
        lib.cf_potrf_f32_set_tensor(prev)
    assert errs[1] <= max(4 * errs[0], 2e-6), errs


@pytest.mark.parametrize("n,batch", [(200, 3), (333, 2), (1312, 4)])
def test_chi2_with_block_inverses_matches_substitution(n, batch):
    """The chi2 kernels that solve 64-row blocks with the factors' kept
    diagonal-block inverses against the 32-row substitution kernels: FP64 to
    1e-12 relative, the FP64-refined mixed chi2 to 1e-10."""
    from cosmoforge_b200 import _lib

    lib = _lib.lib()
    st = torch.cuda.current_stream().cuda_stream
    C = _spd_batch(n, batch, 7 + n)
    g = torch.Generator(device="cuda").manual_seed(n)
    X = torch.randn((n, 2), dtype=torch.float64, device="cuda", generator=g) * 3.0
    # FP64
    L = C.clone()
    info = torch.zeros(batch, dtype=torch.int32, device="cuda")
    work = torch.empty(lib.cf_potrf_workspace(n, batch) // 8 + 1, dtype=torch.float64, device="cuda")
    assert lib.cf_potrf(n, L.data_ptr(), n, n * n, batch, work.data_ptr(), info.data_ptr(), st) == 0
    c_sub = torch.empty((batch, 2), dtype=torch.float64, device="cuda")
    c_inv = torch.empty_like(c_sub)
    ld1 = torch.empty(batch, dtype=torch.float64, device="cuda")
    ld2 = torch.empty_like(ld1)
    assert lib.cf_chi2_logdet(n, L.data_ptr(), n, n * n, batch, X.data_ptr(), 2, 0, 2, None, c_sub.data_ptr(),
                              ld1.data_ptr(), st) == 0
    assert lib.cf_chi2_logdet_dinv(n, L.data_ptr(), n, n * n, work.data_ptr(), lib.cf_potrf_dinv_stride(n), batch,
                                   X.data_ptr(), 2, 0, 2, c_inv.data_ptr(), ld2.data_ptr(), st) == 0
    assert float(((c_inv - c_sub).abs() / c_sub).max()) <= 1e-12
    assert torch.equal(ld1, ld2)
    # mixed
    L32 = C.float().contiguous()
    work32 = torch.empty(lib.cf_potrf_f32_workspace(n, batch) // 4 + 1, dtype=torch.float32, device="cuda")
    assert lib.cf_potrf_f32(n, L32.data_ptr(), n, n * n, batch, work32.data_ptr(), info.data_ptr(), st) == 0
    assert lib.cf_chi2_logdet_mixed(n, L32.data_ptr(), n, n * n, C.data_ptr(), n, n * n, batch, X.data_ptr(), 2, 0,
                                    2, c_sub.data_ptr(), ld1.data_ptr(), st) == 0
    assert lib.cf_chi2_logdet_mixed_dinv(n, L32.data_ptr(), n, n * n, work32.data_ptr(),
                                         lib.cf_potrf_f32_dinv_stride(n), C.data_ptr(), n, n * n, batch,
                                         X.data_ptr(), 2, 0, 2, c_inv.data_ptr(), ld2.data_ptr(), st) == 0
    torch.cuda.synchronize()
    assert int(info.abs().max()) == 0
    assert float(((c_inv - c_sub).abs() / c_sub).max()) <= 1e-10
