"""C(theta) = S(theta) + s N from the per-multipole basis (engine.SignalBasis).

The basis path forms each block region of C as one GEMM of the points'
beam-smoothed tables against basis matrices the pair kernel built once
(``cosmocore/signal_kernels.py:164-502`` per basis entry), so it differs from
the direct per-point build only in the order of the multipole sum.  Checks:
C against the direct build at 1e-13 (relative to the largest entry), the
lower-triangle build with its FP32 copy against the full one (bit for bit),
the FP32 tensor-core build at 1e-6, the likelihood through the basis against
the reference's outputs at 1e-10, and the basis and direct likelihoods on 256
Sobol points (FP64 at 1e-10, mixed at 1e-6 relative).
"""

import numpy as np
import pytest
import torch

from golden_cases import load, params_of

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def config3():
    from cosmoforge_b200 import engine, workloads
    from cosmoforge_b200.layout import build_layout

    pb = workloads.config3()
    L = build_layout(pb.params, pb.mask, pb.beam)
    E = engine.Engine(L)
    N = torch.from_numpy(pb.noise).cuda()
    th = workloads.sobol_points(96, seed=4)
    cl = torch.from_numpy(np.stack([L.smoothed_cl_table(workloads.model_cls(t, L.lmax_signal)) for t in th])).cuda()
    return E, L, N, th, cl


def test_basis_covariance_matches_direct_build(config3):
    E, L, N, th, cl = config3
    s = torch.from_numpy(th[:, 4].copy()).cuda()
    Cb = E.signal_basis(N).covariance(cl, s)
    Cd = E.signal(cl) + s[:, None, None] * N[None]
    err = float((Cb - Cd).abs().max() / Cd.abs().max())
    assert err <= 1e-13, err
    # a table with every spectrum set (EB, TB included) exercises the full basis
    cl2 = cl.clone()
    cl2[:, :, 2:] += 0.01 * cl[:, :1, 2:]
    Cb2 = E.signal_basis(N).covariance(cl2, s)
    Cd2 = E.signal(cl2) + s[:, None, None] * N[None]
    assert float((Cb2 - Cd2).abs().max() / Cd2.abs().max()) <= 1e-13


def test_basis_covariance_f32_on_tensor_cores(config3):
    """The mixed likelihood's build: BF16x6 split products of the same basis,
    written transposed into FP32 matrices (cf_umma_gemm_bf16_scatter), twice.
    Bar: 1e-6 of the largest entry (BF16x6 keeps ~24 bits; FP32 output)."""
    E, L, N, th, cl = config3
    s = torch.from_numpy(th[:, 4].copy()).cuda()
    basis = E.signal_basis(N)
    Cd = basis.covariance(cl, s)
    B, n = cl.shape[0], L.n
    C1 = torch.full((B, n, n), float("nan"), dtype=torch.float32, device="cuda")
    C2 = torch.full_like(C1, float("nan"))
    err = basis.covariance_f32(cl, s, C1, C2)
    assert int(err.item()) == 0
    assert torch.equal(C1, C2)  # both destinations, every entry written
    e = float((C1.double() - Cd).abs().max() / Cd.abs().max())
    assert e <= 1e-6, e


def test_basis_covariance_lower_and_fp32_copy(config3):
    """The likelihood's build: lower triangle only (mirror spans left out,
    tiles right of each row of a diagonal block skipped) with the FP32 copy
    from the same epilogue.  Every lower entry equals the full build's bit for
    bit, and the copy is its FP32 rounding."""
    E, L, N, th, cl = config3
    s = torch.from_numpy(th[:, 4].copy()).cuda()
    basis = E.signal_basis(N)
    full = basis.covariance(cl, s)
    B, n = cl.shape[0], L.n
    C = torch.full((B, n, n), float("nan"), dtype=torch.float64, device="cuda")
    C32 = torch.full((B, n, n), float("nan"), dtype=torch.float32, device="cuda")
    basis.covariance(cl, s, out=C, lower=True, out32=C32)
    low = torch.tril(torch.ones((n, n), dtype=torch.bool, device="cuda"))
    assert torch.equal(C[:, low], full[:, low])
    assert torch.equal(C32[:, low], full[:, low].float())


def test_basis_likelihood_matches_reference():
    from cosmoforge_b200 import engine, workloads
    from cosmoforge_b200.layout import build_layout

    d = load("picslike_tqu_nside8")
    L = build_layout(params_of(d), d["mask"], d["beam"])
    E = engine.Engine(L)
    cl = np.stack([L.smoothed_cl_table(workloads.model_cls(t, L.lmax_signal)) for t in d["thetas"]])
    N = torch.from_numpy(np.diag(d["noise_diag"])).cuda()
    chi2, _, lnl, info = E.lnl(cl, N, torch.from_numpy(d["maps"]), noise_scale=d["thetas"][:, 4], build="basis")
    assert int(info.abs().max()) == 0
    assert np.max(np.abs(chi2.cpu().numpy()[:, 0] / d["ref_chi2"][:, 0] - 1)) <= 1e-10
    assert np.max(np.abs(lnl.cpu().numpy()[:, 0] / d["ref_lnl"][:, 0] - 1)) <= 1e-10


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_basis_and_direct_likelihoods_agree(config3, precision):
    from cosmoforge_b200 import workloads

    E, L, N, _, _ = config3
    th = workloads.sobol_points(256, seed=9)
    cl = np.stack([L.smoothed_cl_table(workloads.model_cls(t, L.lmax_signal)) for t in th])
    g = torch.Generator(device="cuda").manual_seed(1)
    X = torch.randn((L.n, 2), dtype=torch.float64, device="cuda", generator=g) * 10.0
    _, _, lb, ib = E.lnl(cl, N, X, noise_scale=th[:, 4], precision=precision, build="basis")
    _, _, ld, idd = E.lnl(cl, N, X, noise_scale=th[:, 4], precision=precision, build="direct")
    assert int(ib.abs().max()) == 0 and int(idd.abs().max()) == 0
    tol = 1e-10 if precision == "fp64" else 1e-6
    assert float(((lb - ld).abs() / ld.abs()).max()) <= tol
