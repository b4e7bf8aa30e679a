"""Parity at the benchmarked size: the TQU nside-16 problem (n = 5952, 276 parameters).

The FP64 device path (S, C^-1, F, raw bias, raw q, F^-1, C_hat) runs in full;
the oracle (C restatement of the pair kernels, LAPACK ``dpotrf``/``dpotri``,
OpenBLAS products) recomputes on the host what fits in seconds:

* the whole S and the whole C^-1 (``cosmocore/signal_kernels.py:390-537``,
  ``cosmocore/basics/linalg.py:152-219``);
* A_p = C^-1 dC_p for eight parameters that cover every spectrum (TT, EE, BB,
  EB, TE, TB), and F_pq = 1/2 Tr(A_p A_q) for all 36 pairs among them, which
  include the TT x EE, EB and TB cross blocks (``qube/fisher.py:501-607``);
* raw bias_p = 1/2 Tr(C^-1 N C^-1 dC_p) and q_p = 1/2 y^T dC_p y, y = C^-1 x
  (``qube/spectra.py:1124-1186``).

Bars: S 1e-13 and C^-1 1e-11 (relative to the largest entry), F 1e-10
(correlation-normalised), bias and q 1e-10 (relative).  F^-1 and C_hat are
checked on the device against host FP64 products of the device F and q
(1e-10).  The mixed path (BF16x6 split products on tcgen05, forms picked by
the autotuner as in the benchmark) must meet its stated targets against the
FP64 path on the same problem: max |dF_bb| / F_bb <= 1e-5 and
max |dC_hat| <= 1e-3 sigma.
"""

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

# (spectrum index, bin) in the reference's TQU order TT, EE, BB, EB, TE, TB
PICKS = [(0, 0), (0, 45), (1, 3), (2, 20), (3, 10), (4, 0), (4, 30), (5, 44)]


@pytest.fixture(scope="module")
def solved():
    import torch

    from cosmoforge_b200 import engine, qube, workloads
    from cosmoforge_b200.layout import build_layout
    from oracle import oracle as orc

    pb = workloads.config1()
    L = build_layout(pb.params, pb.mask, pb.beam)
    assert (L.n, L.n_params) == (5952, 276)
    E = engine.Engine(L)
    N = torch.from_numpy(pb.noise).cuda()
    X = qube.draw_maps(L, pb.cls, N, nsims=1, seed=0)
    r = engine.qml_solve(E, pb.cls, N, X)
    torch.cuda.synchronize()
    dev = {k: (v.cpu().numpy() if hasattr(v, "cpu") else v) for k, v in r.items()}
    xh = X.cpu().numpy()

    # oracle on the host
    S = orc.signal_matrix(L, L.smoothed_cl_table(pb.cls))
    Cinv = orc.matrix_inverse_symm(S + pb.noise)
    W = L.param_weights()
    params = [s * L.nbins + b for s, b in PICKS]
    A, AT, bias, q = [], [], [], []
    M = Cinv @ (pb.noise @ Cinv)
    Y = Cinv @ xh
    for p in params:
        dC = orc.binned_derivative(L, p, W)
        a = Cinv @ dC
        A.append(a)
        AT.append(np.ascontiguousarray(a.T))
        bias.append(0.5 * orc.trace_product(M, dC))
        q.append(0.5 * float(np.sum(Y * (dC @ Y))))
    F = np.zeros((len(params), len(params)))
    for i in range(len(params)):
        for j in range(i, len(params)):
            F[i, j] = F[j, i] = 0.5 * orc.trace_product(A[i], A[j], AT[j])
    ora = dict(S=S, Cinv=Cinv, F=F, bias=np.array(bias), q=np.array(q), params=params)
    return dict(E=E, L=L, pb=pb, N=N, X=X, dev=dev, ora=ora, Cinv_dev=r["Cinv"])


def test_signal_and_inverse_at_n5952(solved):
    d, o = solved["dev"], solved["ora"]
    assert np.max(np.abs(d["S"] - o["S"])) <= 1e-13 * np.max(np.abs(o["S"]))
    assert np.max(np.abs(d["Cinv"] - o["Cinv"])) <= 1e-11 * np.max(np.abs(o["Cinv"]))


def test_fisher_entries_every_spectrum_pair(solved):
    d, o = solved["dev"], solved["ora"]
    idx = o["params"]
    Fd = d["fisher"][np.ix_(idx, idx)]
    Fo = o["F"]
    corr = np.sqrt(np.outer(np.diag(Fo), np.diag(Fo)))
    assert np.all(np.diag(Fo) > 0)
    assert np.max(np.abs(Fd - Fo) / corr) <= 1e-10


def test_bias_and_q_sampled_parameters(solved):
    d, o, L = solved["dev"], solved["ora"], solved["L"]
    idx = o["params"]
    bias = d["bias"][idx]
    # the device q has the bias removed when remove_nb is set (the reference default)
    q = d["q"][0, idx] + (bias if L.remove_nb else 0.0)
    assert np.max(np.abs(bias - o["bias"]) / np.abs(o["bias"])) <= 1e-10
    qs = np.maximum(np.abs(o["q"]), np.abs(o["bias"]))
    assert np.max(np.abs(q - o["q"]) / qs) <= 1e-10


def test_inverse_fisher_and_clhat_against_host_products(solved):
    from oracle import oracle as orc

    d = solved["dev"]
    Finv = orc.matrix_inverse_symm(d["fisher"])
    assert np.max(np.abs(d["invfisher"] - Finv)) <= 1e-10 * np.max(np.abs(Finv))
    ch = d["q"] @ Finv
    assert np.max(np.abs(d["clhat"] - ch)) <= 1e-10 * np.max(np.abs(ch))


def test_mixed_path_meets_stated_tolerances(solved):
    import torch

    from cosmoforge_b200 import autotune, engine_mixed

    E, N, X, L = solved["E"], solved["N"], solved["X"], solved["L"]
    Cinv = solved["Cinv_dev"]
    forms, _ = autotune.tune_fisher(E, Cinv, "bf16x6", use_cache=False)
    Fm, bm, qm = engine_mixed.fisher_qml(E, Cinv, N, X, scheme="bf16x6", forms=forms)
    if L.remove_nb:
        qm = qm - bm[None, :]
    Finv_m = E.spd_inverse(Fm.clone())
    ch_m = E.gemm(qm, Finv_m).cpu().numpy()
    torch.cuda.synchronize()
    d = solved["dev"]
    Fd = d["fisher"]
    Fm = Fm.cpu().numpy()
    rel_diag = np.max(np.abs(np.diag(Fm) - np.diag(Fd)) / np.diag(Fd))
    sigma = np.sqrt(np.diag(d["invfisher"]))
    shift = np.max(np.abs(ch_m - d["clhat"]) / sigma[None, :])
    assert rel_diag <= 1e-5, rel_diag
    assert shift <= 1e-3, shift
