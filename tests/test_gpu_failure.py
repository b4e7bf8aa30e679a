"""Failure paths, made on the host or through a wait bound; no GPU fault is involved.

* A timed-out wait: ``cf_umma_set_wait_limit(0)`` makes the tcgen05 kernel's
  first unsatisfied barrier wait give up.  The launch must drain what it
  issued, free its TMEM and raise its error flag, which ``cf_umma_status``
  turns into ``CF_ERR_TIMEOUT`` (and the Python layer into a DeviceError);
  with the default bound restored the next launch on the same context must
  succeed and be exact.
* Non-finite inputs: a NaN or an Inf planted in an SPD matrix must give the
  factorisation status LAPACK's ``dpotrf`` gives for the same matrix (the
  1-based index of the first failed pivot; the reference's
  ``matrix_inverse_symm`` raises ``ValueError("dpotrf failed ...")`` on it,
  ``cosmocore/basics/linalg.py:200-214``), in FP64 and FP32 and through
  ``cf_spd_inverse``; the likelihood reports it per point.
"""

import ctypes

import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu

X6 = ([0, 0, 1, 0, 1, 2], [0, 1, 0, 2, 1, 0])


def _gemm_case(lib, M, N, K):
    g = torch.Generator(device="cuda").manual_seed(11)
    A = torch.randn((3, M, K), device="cuda", generator=g).to(torch.bfloat16)
    B = torch.randn((3, N, K), device="cuda", generator=g).to(torch.bfloat16)
    Cf = torch.full((M, N), float("nan"), device="cuda", dtype=torch.float32)
    err = torch.zeros(1, dtype=torch.int32, device="cuda")
    ta = (ctypes.c_int * 6)(*X6[0])
    tb = (ctypes.c_int * 6)(*X6[1])
    st = torch.cuda.current_stream().cuda_stream

    def run():
        rc = lib.cf_umma_gemm_bf16(M, N, K, 6, ctypes.cast(ta, ctypes.c_void_p), ctypes.cast(tb, ctypes.c_void_p),
                                   A.data_ptr(), K, M * K, 3, B.data_ptr(), K, N * K, 3, None, 0, 0, 0, None, 0, 0,
                                   Cf.data_ptr(), N, err.data_ptr(), st)
        assert rc == 0

    ref = sum(A[a].double() @ B[b].double().T for a, b in zip(*X6))
    return run, Cf, err, ref


@pytest.mark.parametrize("form", [1, 2])
def test_timed_out_wait_reports_timeout_and_context_survives(form):
    """form 1: one CTA per tile; form 2: CTA pairs (the leader's MMAs write both
    CTAs' TMEM; both drain and meet at the final cluster barrier)."""
    from cosmoforge_b200 import _lib

    lib = _lib.lib()
    st = torch.cuda.current_stream().cuda_stream
    run, Cf, err, ref = _gemm_case(lib, 384, 512, 1024)
    prev_form = lib.cf_umma_set_all_planes(form)
    try:
        prev = lib.cf_umma_set_wait_limit(0)
        try:
            run()
            assert lib.cf_umma_status(err.data_ptr(), st) == _lib.CF_ERR_TIMEOUT
            with pytest.raises(_lib.DeviceError, match="timeout"):
                _lib.check(lib.cf_umma_status(err.data_ptr(), st), "tensor-core kernel")
        finally:
            lib.cf_umma_set_wait_limit(-1)
        assert prev == 2_000_000_000
        err.zero_()
        run()
        assert lib.cf_umma_status(err.data_ptr(), st) == _lib.CF_OK
    finally:
        lib.cf_umma_set_all_planes(prev_form)
    got = Cf.double()
    assert float((got - ref).abs().max() / ref.abs().max()) < 1e-5


def test_timed_out_wait_through_the_mixed_fisher():
    from cosmoforge_b200 import _lib, engine, engine_mixed, workloads
    from cosmoforge_b200.layout import build_layout

    pb = workloads.config0()
    pb.params["lmax"] = 8
    L = build_layout(pb.params, pb.mask, pb.beam)
    E = engine.Engine(L)
    C = E.signal(L.smoothed_cl_table(pb.cls)) + torch.from_numpy(pb.noise).cuda()
    Cinv = E.spd_inverse(C)
    lib = _lib.lib()
    lib.cf_umma_set_wait_limit(0)
    try:
        with pytest.raises(_lib.DeviceError, match="timeout"):
            engine_mixed.fisher(E, Cinv)
    finally:
        lib.cf_umma_set_wait_limit(-1)
    F = engine_mixed.fisher(E, Cinv)  # the next call on the same context succeeds
    assert bool(torch.isfinite(F).all())


def _spd(n, seed):
    rng = np.random.default_rng(seed)
    M = rng.standard_normal((n, n))
    return M @ M.T / n + np.eye(n)


def _lapack_info(A):
    """LAPACK's dpotrf status by its own rule (dpotf2: the 1-based index of the
    first pivot that is not positive or is NaN), from a plain unblocked
    Cholesky.  scipy's dpotrf is not used for this: the OpenBLAS build here
    only tests the pivot for <= 0, so it lets NaN pivots through."""
    A = np.array(A, dtype=np.float64, copy=True)
    n = A.shape[0]
    with np.errstate(all="ignore"):
        for j in range(n):
            d = A[j, j] - np.dot(A[j, :j], A[j, :j])
            if not d > 0.0:
                return j + 1
            ljj = np.sqrt(d)
            A[j, j] = ljj
            A[j + 1:, j] = (A[j + 1:, j] - A[j + 1:, :j] @ A[j, :j]) / ljj
    return 0


@pytest.mark.parametrize("where,value", [((5, 3), np.nan), ((70, 70), np.nan), ((130, 2), np.inf),
                                         ((40, 40), -np.inf), ((90, 17), -np.inf)])
def test_non_finite_entries_give_lapack_info(where, value):
    from cosmoforge_b200 import _lib

    lib = _lib.lib()
    n = 200
    A = _spd(n, 3)
    i, j = where
    A[i, j] = A[j, i] = value
    expect = _lapack_info(A)
    assert expect > 0
    st = torch.cuda.current_stream().cuda_stream
    for dt, ws_fn, fn in ((torch.float64, lib.cf_potrf_workspace, lib.cf_potrf),
                          (torch.float32, lib.cf_potrf_f32_workspace, lib.cf_potrf_f32)):
        X = torch.from_numpy(A).to("cuda", dt)
        work = torch.empty(ws_fn(n, 1) // 4 + 1, dtype=torch.float32, device="cuda")
        info = torch.zeros(1, dtype=torch.int32, device="cuda")
        assert fn(n, X.data_ptr(), n, n * n, 1, work.data_ptr(), info.data_ptr(), st) == 0
        torch.cuda.synchronize()
        assert int(info.item()) == expect, (dt, int(info.item()), expect)
    # the Jacobi-scaled inverse reports the same pivot (the scaling keeps NaN / Inf where they are)
    X = torch.from_numpy(A).cuda()
    work = torch.empty(lib.cf_spd_inverse_workspace(n, 1) // 8 + 1, dtype=torch.float64, device="cuda")
    info = torch.zeros(1, dtype=torch.int32, device="cuda")
    assert lib.cf_spd_inverse(n, X.data_ptr(), n, n * n, 1, work.data_ptr(), info.data_ptr(), st) == 0
    torch.cuda.synchronize()
    scaled = A.copy()
    d = np.abs(np.diag(scaled))
    d[d == 0] = 1.0
    s = 1.0 / np.sqrt(d)
    with np.errstate(all="ignore"):
        scaled = scaled * s[:, None] * s[None, :]
    assert int(info.item()) == _lapack_info(scaled)


def test_likelihood_reports_a_non_finite_point():
    from cosmoforge_b200 import engine, workloads
    from cosmoforge_b200.layout import build_layout

    pb = workloads.config3()
    L = build_layout(pb.params, pb.mask, pb.beam)
    E = engine.Engine(L)
    N = torch.from_numpy(pb.noise).cuda()
    x = torch.randn((L.n, 1), dtype=torch.float64, device="cuda") * 10.0
    th = workloads.sobol_points(4, seed=2)
    cl = np.stack([L.smoothed_cl_table(workloads.model_cls(t, L.lmax_signal)) for t in th])
    cl[2, 0, 5] = np.nan  # a NaN in one point's TT table
    for prec in ("fp64", "mixed"):
        _, _, lnl, info = E.lnl(cl, N, x, precision=prec)
        info = info.cpu().numpy()
        assert info[2] > 0 and np.all(info[[0, 1, 3]] == 0), (prec, info)
        assert bool(torch.isfinite(lnl[[0, 1, 3]]).all())


def test_potrf_f32_tensor_core_timeout():
    """A bounded wait of the FP32 factor's tensor-core GEMMs that runs out
    marks the problem with CF_ERR_TIMEOUT (-3) in info (the kernel drains its
    MMAs and frees its TMEM first), and the next call on the same context
    factors exactly."""
    from cosmoforge_b200 import _lib

    lib = _lib.lib()
    n, batch = 300, 4
    A64 = torch.stack([torch.from_numpy(_spd(n, 20 + b)) for b in range(batch)]).cuda()
    st = torch.cuda.current_stream().cuda_stream

    def run():
        A = A64.float().contiguous()
        work = torch.empty(lib.cf_potrf_f32_workspace(n, batch) // 4 + 1, dtype=torch.float32, device="cuda")
        info = torch.zeros(batch, dtype=torch.int32, device="cuda")
        assert lib.cf_potrf_f32(n, A.data_ptr(), n, n * n, batch, work.data_ptr(), info.data_ptr(), st) == 0
        torch.cuda.synchronize()
        return A, info

    lib.cf_sgemm_bf16x6_set_wait_limit(0)
    try:
        _, info = run()
    finally:
        lib.cf_sgemm_bf16x6_set_wait_limit(-1)
    assert (info.cpu().numpy() == _lib.CF_ERR_TIMEOUT).all(), info
    A, info = run()
    assert int(info.abs().max()) == 0
    L64 = torch.linalg.cholesky(A64)
    assert float((torch.tril(A.double()) - L64).abs().max() / L64.abs().max()) <= 1e-5
