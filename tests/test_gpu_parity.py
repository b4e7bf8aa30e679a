"""Device path (plain FP64) against the oracle and the reference's golden outputs.

Tolerances: 1e-13 relative for S and dC (same recurrences, FMA allowed),
1e-11 for the intermediate C^-1, and the drop-in's stated 1e-10 relative for F, q, bias, C_hat, chi2
and lnL against the reference's own outputs on the same inputs.
"""

import numpy as np
import pytest
import torch

from cosmoforge_b200 import workloads
from cosmoforge_b200.layout import build_layout
from golden_cases import QML_CASES, cls_of, load, noise_of, params_of

pytestmark = pytest.mark.gpu


def _rel(a, b):
    a = np.asarray(a)
    b = np.asarray(b)
    return float(np.max(np.abs(a - b)) / np.max(np.abs(b)))


@pytest.fixture(scope="module")
def engine_mod():
    from cosmoforge_b200 import engine

    return engine


@pytest.fixture(scope="module", params=QML_CASES)
def solved(request, engine_mod):
    d = load(request.param)
    L = build_layout(params_of(d), d["mask"], d["beam"])
    E = engine_mod.Engine(L)
    N = torch.from_numpy(noise_of(d)).cuda()
    maps = torch.from_numpy(d["maps"]).cuda()
    r = engine_mod.qml_solve(E, cls_of(d), N, maps)
    torch.cuda.synchronize()
    return d, L, E, {k: v.cpu().numpy() for k, v in r.items()}


def test_signal(solved):
    d, L, E, r = solved
    rows = d["s_rows_idx"]
    assert _rel(r["S"][rows], d["ref_signal_rows"]) <= 1e-13
    assert _rel(np.diag(r["S"]), d["ref_signal_diag"]) <= 1e-13
    assert np.array_equal(r["S"], r["S"].T)


def test_inverse(solved):
    # C^-1 is an intermediate; its agreement is bounded by cond(C) * eps (the
    # full-sky nside-4 cases reach a few 1e-12), the outputs are held to 1e-10.
    d, L, E, r = solved
    assert _rel(np.diag(r["Cinv"]), d["ref_cinv_diag"]) <= 1e-11


def test_fisher(solved):
    d, L, E, r = solved
    R = d["ref_fisher"]
    corr = np.sqrt(np.outer(np.diag(R), np.diag(R)))
    assert np.max(np.abs(r["fisher"] - R) / corr) <= 1e-10
    assert _rel(r["fisher"], R) <= 1e-10


def test_qml(solved):
    d, L, E, r = solved
    assert _rel(r["bias"], d["ref_noise_bias_raw"]) <= 1e-10
    assert _rel(r["q"], d["ref_q_raw"]) <= 1e-10
    assert _rel(r["clhat"], d["ref_clhat"]) <= 1e-10
    assert _rel(r["noise_bias"], d["ref_noise_bias"]) <= 1e-8


def test_fused_reduce_matches_reference(solved):
    """Bias and q with the derivative entries reduced where they are built
    (the drop-in Spectra path) against the reference's raw outputs and the
    blocks-in-HBM path."""
    d, L, E, r = solved
    Cinv = torch.from_numpy(r["Cinv"]).cuda()
    N = torch.from_numpy(noise_of(d)).cuda()
    X = torch.from_numpy(d["maps"]).cuda()
    _, b_f, q_f = E.fisher_qml(Cinv, N, X, want_fisher=False, fused_reduce=True)
    _, b_d, q_d = E.fisher_qml(Cinv, N, X, want_fisher=False, fused_reduce=False)
    b_f, q_f, b_d, q_d = (t.cpu().numpy() for t in (b_f, q_f, b_d, q_d))
    assert _rel(b_f, d["ref_noise_bias_raw"]) <= 1e-10
    # the reference's q is net of the noise bias when remove_nb is set
    assert _rel(q_f - b_f[None, :] if L.remove_nb else q_f, d["ref_q_raw"]) <= 1e-10
    assert _rel(b_f, b_d) <= 1e-10 and _rel(q_f, q_d) <= 1e-10


def test_derivatives_match_oracle(solved):
    from oracle import oracle as orc

    d, L, E, r = solved
    W = L.param_weights()
    for p in sorted({0, L.nbins - 1, L.n_params // 2, L.n_params - 1}):
        ref = orc.binned_derivative(L, p, W)
        got = E.derivative_dense(p).cpu().numpy()
        assert _rel(got, ref) <= 1e-13, p


def test_lnl_fortran_picslike(engine_mod):
    d = load("fortran_picslike_nside8_B")
    L = build_layout(params_of(d), d["mask"], d["beam"])
    E = engine_mod.Engine(L)
    cl = np.stack([L.smoothed_cl_table({"BB": c}) for c in d["point_cl_BB"]])
    chi2, ld, lnl, info = E.lnl(cl, torch.from_numpy(d["noise"]).cuda(), torch.from_numpy(d["maps"]))
    assert int(info.abs().max()) == 0
    chi2, lnl = chi2.cpu().numpy(), lnl.cpu().numpy()
    assert np.max(np.abs(chi2[:, 0] / d["ref_chi2"][:, 0] - 1)) <= 1e-10
    assert np.max(np.abs(lnl[:, 0] / d["ref_lnl"][:, 0] - 1)) <= 1e-10
    assert np.max(np.abs(chi2[:, 0] / d["fort_chi2"] - 1)) <= 1e-9


def test_lnl_tqu_batch(engine_mod):
    d = load("picslike_tqu_nside8")
    L = build_layout(params_of(d), d["mask"], d["beam"])
    E = engine_mod.Engine(L)
    cl = np.stack([L.smoothed_cl_table(workloads.model_cls(t, L.lmax_signal)) for t in d["thetas"]])
    N = torch.from_numpy(np.diag(d["noise_diag"])).cuda()
    chi2, ld, lnl, info = E.lnl(cl, N, torch.from_numpy(d["maps"]), noise_scale=d["thetas"][:, 4])
    assert int(info.abs().max()) == 0
    chi2, lnl = chi2.cpu().numpy(), lnl.cpu().numpy()
    assert np.max(np.abs(chi2[:, 0] / d["ref_chi2"][:, 0] - 1)) <= 1e-10
    assert np.max(np.abs(lnl[:, 0] / d["ref_lnl"][:, 0] - 1)) <= 1e-10


def test_not_positive_definite_reports_info(engine_mod):
    d = load("config0_tt_nside8")
    L = build_layout(params_of(d), d["mask"], d["beam"])
    E = engine_mod.Engine(L)
    A = torch.eye(L.n, dtype=torch.float64, device="cuda")
    A[7, 7] = -1.0
    with pytest.raises(ValueError, match="info=8"):
        E.spd_inverse(A)
