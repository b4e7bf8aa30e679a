"""Mixed-precision Fisher (tcgen05 BF16 split products) against the FP64 device path.

Error metric: max |F_mixed - F_fp64| / sqrt(F_ii F_jj) (entries normalised by
their Fisher correlation scale) and max relative error of the diagonal.
Tolerances (measured on B200, with margin): BF16x6 (~24-bit products, FP32
tensor-core accumulation promoted every 16 k-tiles) 5e-5 on both metrics;
BF16x3 (~16-bit) 3e-3, its error is amplified by the cancellation in
C^-1 dC_b on high signal-to-noise problems.  C_hat moves by |dC_hat| / sigma
below 1e-3 in both.
"""

import numpy as np
import pytest
import torch

from cosmoforge_b200.layout import build_layout
from golden_cases import cls_of, load, noise_of, params_of

pytestmark = pytest.mark.gpu

TOL = {"bf16x3": (3e-3, 3e-3), "bf16x6": (5e-5, 5e-5)}


def _case(name, drop=0):
    d = load(name)
    mask = d["mask"].copy()
    N = noise_of(d)
    maps = d["maps"]
    if drop:
        # deactivate a few pixels so segment sizes are not multiples of 8
        act = np.flatnonzero(mask[:, 0] > 0.5)[:drop]
        keep = np.ones(int((mask[:, 0] > 0.5).sum()), bool)
        keep[:drop] = False
        mask[act, 0] = 0.0
        nt = keep.size
        sel = np.concatenate([np.flatnonzero(keep), np.arange(nt, N.shape[0])])
        N = N[np.ix_(sel, sel)]
        maps = maps[sel]
    return d, params_of(d), mask, N, maps


@pytest.mark.parametrize("name,drop", [("tqu_cut_nside4", 0), ("tqu_cut_nside4", 3), ("config0_tt_nside8", 5),
                                       ("nside4_TEB", 0)])
@pytest.mark.parametrize("scheme", ["bf16x3", "bf16x6"])
def test_mixed_fisher_matches_fp64(name, drop, scheme):
    from cosmoforge_b200 import engine, engine_mixed

    d, p, mask, N, maps = _case(name, drop)
    L = build_layout(p, mask, d["beam"])
    E = engine.Engine(L)
    Nd = torch.from_numpy(N).cuda()
    S = E.signal(L.smoothed_cl_table(cls_of(d)))
    Cinv = E.spd_inverse(S + Nd)
    F64, _, _ = E.fisher_qml(Cinv)
    Fm = engine_mixed.fisher(E, Cinv, scheme)
    F64, Fm = F64.cpu().numpy(), Fm.cpu().numpy()
    corr = np.sqrt(np.outer(np.diag(F64), np.diag(F64)))
    e_corr = np.max(np.abs(Fm - F64) / corr)
    e_diag = np.max(np.abs(np.diag(Fm) / np.diag(F64) - 1))
    print(f"{name} drop={drop} {scheme}: corr {e_corr:.2e} diag {e_diag:.2e}")
    assert e_corr <= TOL[scheme][0]
    assert e_diag <= TOL[scheme][1]
    # the estimator moves by much less than its error bar
    Finv = np.linalg.inv(F64)
    Finv_m = np.linalg.inv(Fm)
    sig = np.sqrt(np.diag(Finv))
    q = np.random.default_rng(0).standard_normal(F64.shape[0]) @ np.linalg.cholesky(F64).T
    assert np.max(np.abs(q @ Finv_m - q @ Finv) / sig) < (1e-3 if scheme == "bf16x6" else 1e-2)


# |dC_hat| / sigma bound per case.  The full-sky nside-4 TQU fixture is nearly
# noiseless (N = 0.013 / 1.3e-4 muK^2) with an ill-conditioned Fisher matrix;
# 24-bit products leave ~3e-2 sigma there, which is why the plain FP64 path
# stays available for such problems.
QML_SIGMA_TOL = {"tqu_cut_nside4": 1e-3, "config0_tt_nside8": 1e-3, "nside4_TQU": 5e-2}


@pytest.mark.parametrize("name", sorted(QML_SIGMA_TOL))
def test_mixed_qml_matches_fp64(name):
    """Noise bias, raw q and C_hat of the BF16x6 path against plain FP64."""
    from cosmoforge_b200 import engine, engine_mixed

    d, p, mask, N, maps = _case(name)
    L = build_layout(p, mask, d["beam"])
    E = engine.Engine(L)
    Nd = torch.from_numpy(N).cuda()
    X = torch.from_numpy(maps).cuda()
    S = E.signal(L.smoothed_cl_table(cls_of(d)))
    Cinv = E.spd_inverse(S + Nd)
    F64, b64, q64 = E.fisher_qml(Cinv, Nd, X)
    Fm, bm, qm = engine_mixed.fisher_qml(E, Cinv, Nd, X, scheme="bf16x6")
    F64, b64, q64 = F64.cpu().numpy(), b64.cpu().numpy(), q64.cpu().numpy()
    Fm, bm, qm = Fm.cpu().numpy(), bm.cpu().numpy(), qm.cpu().numpy()
    assert np.max(np.abs(bm - b64)) / np.max(np.abs(b64)) < 1e-5
    assert np.max(np.abs(qm - q64)) / np.max(np.abs(q64)) < 1e-5
    Finv = np.linalg.inv(F64)
    sig = np.sqrt(np.diag(Finv))
    c64 = (q64 - b64) @ Finv
    cm = (qm - bm) @ np.linalg.inv(Fm)
    print(f"{name}: |dC_hat|/sigma {np.max(np.abs(cm - c64) / sig):.2e}")
    assert np.max(np.abs(cm - c64) / sig) < QML_SIGMA_TOL[name]


@pytest.mark.parametrize("name", ["tqu_cut_nside4", "config0_tt_nside8"])
def test_mixed_dropin_classes_match_fp64(name):
    """Fisher / Spectra with precision="mixed" (F and the noise bias from the
    tensor-core pass in Fisher.run, raw q from the FP64 derivative entries in
    Spectra.run; q net of the bias carries the bias's error) against the same
    classes in plain FP64."""
    from cosmoforge_b200 import qube

    d, p, mask, N, maps = _case(name)
    out = {}
    for prec in ("fp64", "mixed"):
        f = qube.Fisher(p, basis=False, mask=mask, noise_cov1=N, cls_data=cls_of(d), beam=d["beam"],
                        precision=prec)
        f.run()
        s = qube.Spectra(p, fisher=f, maps1=maps)
        s.run()
        out[prec] = (f.get_fisher_matrix(), s.get_noise_bias(), s.qml_results, s.get_power_spectra(),
                     s.qml_noise_bias)
    F64, nb64, q64, c64, b64 = out["fp64"]
    Fm, nbm, qm, cm, bm = out["mixed"]
    corr = np.sqrt(np.outer(np.diag(F64), np.diag(F64)))
    sig = np.sqrt(np.diag(np.linalg.inv(F64)))
    e_f = np.max(np.abs(Fm - F64) / corr)
    e_b = np.max(np.abs(bm - b64)) / np.max(np.abs(b64))
    e_q = np.max(np.abs(qm - q64)) / np.max(np.abs(q64))
    e_c = np.max(np.abs(cm - c64) / sig)
    print(f"{name}: F {e_f:.1e} bias {e_b:.1e} q {e_q:.1e} C_hat {e_c:.1e} sigma")
    assert e_f <= 5e-5 and e_b <= 1e-5 and e_q <= 1e-5 and e_c <= 1e-3
    assert np.max(np.abs(nbm - nb64) / sig) <= 1e-3
