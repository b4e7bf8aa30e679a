"""Harmonic basis on the device against the oracle and the reference.

* V from cf_harmonic_operator against the NumPy restatement: 1e-12 of the
  largest entry.
* F, raw bias, raw q of the device harmonic estimator against the reference
  run with basis="harmonic": 1e-10 relative; C_hat 1e-9 (the reference's
  harmonic F^-1 carries ~2e-10 of rounding on the config-0 case, the same
  amount by which its own harmonic and pixel-space C_hat differ).
* The drop-in classes with basis="harmonic" and with the default basis (which
  the reference's cost model sends to the harmonic basis on these problems).
* The compressed pixel basis (epsilon, noise-weighted eigen-truncation)
  through the drop-in classes against the reference's PixelBasis run.
* At the TQU nside-16 size (n = 5952, l = 2..47): harmonic F against the
  pixel-space FP64 F of the same engine; they differ by the rounding of the
  pixel-space spin-2 kernels (~1e-8), not by the method.
"""

import numpy as np
import pytest
import torch

from cosmoforge_b200 import workloads
from cosmoforge_b200.layout import build_layout
from golden_cases import cls_of, load, noise_of, params_of, smoothed_cls

pytestmark = pytest.mark.gpu

HARMONIC = [("tqu_cut_nside4", "harmonic_tqu_cut_nside4"), ("config0_tt_nside8", "harmonic_config0_tt_nside8"),
            ("nside4_TEB", "harmonic_nside4_TEB")]


def _rel(a, b):
    a, b = np.asarray(a), np.asarray(b)
    return float(np.max(np.abs(a - b)) / np.max(np.abs(b)))


@pytest.mark.parametrize("name", ["tqu_cut_nside4", "config0_tt_nside8", "nside4_TEB"])
def test_operator_matches_oracle(name):
    from cosmoforge_b200 import engine, harmonic
    from oracle import harmonic_oracle as ho

    d = load(name)
    L = build_layout(params_of(d), d["mask"], d["beam"])
    plan = harmonic.HarmonicPlan(engine.Engine(L))
    ref = ho.harmonic_operator(L, L.lmin, L.lmax)
    got = plan.V.cpu().numpy()
    assert got.shape == ref.shape
    assert np.max(np.abs(got - ref)) <= 1e-12 * np.max(np.abs(ref))


@pytest.mark.parametrize("src,hname", HARMONIC)
def test_harmonic_estimator_matches_reference(src, hname):
    from cosmoforge_b200 import engine, harmonic

    d, h = load(src), load(hname)
    L = build_layout(params_of(d), d["mask"], d["beam"])
    E = engine.Engine(L)
    r = harmonic.qml_solve(E, cls_of(d), torch.from_numpy(noise_of(d)).cuda(), torch.from_numpy(d["maps"]).cuda())
    r = {k: v.cpu().numpy() for k, v in r.items()}
    e = {k: _rel(r[a], h[b]) for k, a, b in (("F", "fisher", "ref_fisher"), ("bias", "bias", "ref_noise_bias_raw"),
                                             ("q", "q", "ref_q_raw"), ("C_hat", "clhat", "ref_clhat"))}
    print(src, {k: f"{v:.1e}" for k, v in e.items()})
    assert e["F"] <= 1e-10 and e["bias"] <= 1e-10 and e["q"] <= 1e-10 and e["C_hat"] <= 1e-9


@pytest.mark.parametrize("basis", ["harmonic", None])
def test_dropin_classes_harmonic(basis):
    from cosmoforge_b200 import qube

    d, h = load("tqu_cut_nside4"), load("harmonic_tqu_cut_nside4")
    p = params_of(d)
    f = qube.Fisher(p, basis=basis, mask=d["mask"], noise_cov1=noise_of(d), cls_data=cls_of(d), beam=d["beam"])
    f.run()
    assert f.method == "harmonic"
    s = qube.Spectra(p, fisher=f, maps1=d["maps"])
    s.run()
    assert _rel(f.get_fisher_matrix(), h["ref_fisher"]) <= 1e-10
    assert _rel(s.qml_results, h["ref_q_raw"]) <= 1e-10
    assert _rel(s.qml_noise_bias, h["ref_noise_bias_raw"]) <= 1e-10
    assert _rel(s.get_power_spectra(), h["ref_clhat"]) <= 1e-9
    assert _rel(s.get_noise_bias(), h["ref_noise_bias"]) <= 1e-8


def test_harmonic_matches_pixel_at_config1_size():
    from cosmoforge_b200 import engine, harmonic

    pb = workloads.config1()
    L = build_layout(pb.params, pb.mask, pb.beam)
    E = engine.Engine(L)
    N = torch.from_numpy(pb.noise).cuda()
    plan = harmonic.HarmonicPlan(E)
    tab = L.smoothed_cl_table(pb.cls)
    Sh = plan.signal(tab)
    Sp = E.signal(tab)
    e_s = float((Sh - Sp).abs().max() / Sp.abs().max())
    Cinv = E.spd_inverse(Sp + N)
    Fh, _, _ = plan.fisher_qml(Cinv)
    Fp, _, _ = E.fisher_qml(Cinv)
    Fh, Fp = Fh.cpu().numpy(), Fp.cpu().numpy()
    corr = np.sqrt(np.outer(np.diag(Fp), np.diag(Fp)))
    e_f = float(np.max(np.abs(Fh - Fp) / corr))
    print(f"n = {L.n}, modes = {plan.nm}: |dS| {e_s:.1e}, F corr-normalised {e_f:.1e}")
    assert e_s <= 2e-8 and e_f <= 2e-8


@pytest.mark.parametrize("name,basis", [
    ("compressed_tqu_cut_nside4", {"method": "pixel", "epsilon": 1e-3}),
    ("compressed_config0_tt_nside8", {"method": "pixel", "epsilon": 1e-3}),
    ("compressed_mf_tqu_cut_nside4", {"method": "pixel", "mode_fraction": [0.7, 0.6]}),
    ("compressed_h_config0_tt_nside8", {"method": "pixel", "epsilon": 1e-2, "compression_target": "harmonic"}),
    ("compressed_tc_config0_tt_nside8", {"method": "pixel", "epsilon": 1e-3, "compression_target": "total_covariance",
                                         "C_ell": "TT"}),
    ("compressed_snr_config0_tt_nside8", {"method": "pixel", "epsilon": 1e-4, "compression_target": "snr",
                                          "C_ell": "TT"}),
    ("compressed_eb_tqu_cut_nside4", {"method": "pixel", "epsilon": [1e-3, (1e-3, 1e-2)]}),
    ("compressed_tc_eb_tqu_cut_nside4", {"method": "pixel", "epsilon": [1e-3, (2e-3, 1e-2)],
                                         "compression_target": "total_covariance", "C_ell": ("TT", "EE", "BB")})])
def test_compressed_dropin_matches_reference(name, basis):
    """The eigen-truncated pixel basis (cuSOLVER eigenvectors) through the
    drop-in classes against the reference's run with the same basis dict:
    same kept dimension; F, raw bias, raw q, C_hat 1e-10."""
    from cosmoforge_b200 import qube

    d = load(name)
    p = params_of(d)
    basis = dict(basis)
    if isinstance(basis.get("C_ell"), str):  # the fixture's beam-smoothed spectra, as the reference run got them
        basis["C_ell"] = smoothed_cls(d)[basis["C_ell"]]
    elif isinstance(basis.get("C_ell"), tuple):
        sm = smoothed_cls(d)
        basis["C_ell"] = {k: sm[k] for k in basis["C_ell"]}
    f = qube.Fisher(p, basis=basis, mask=d["mask"], noise_cov1=noise_of(d), cls_data=cls_of(d), beam=d["beam"])
    f.run()
    assert f.method == "compressed" and f.dim == int(d["ref_dim"])
    s = qube.Spectra(p, fisher=f, maps1=d["maps"])
    s.run()
    e = {"F": _rel(f.get_fisher_matrix(), d["ref_fisher"]), "q": _rel(s.qml_results, d["ref_q_raw"]),
         "bias": _rel(s.qml_noise_bias, d["ref_noise_bias_raw"]), "C_hat": _rel(s.get_power_spectra(), d["ref_clhat"])}
    print(name, f.dim, {k: f"{v:.1e}" for k, v in e.items()})
    assert max(e.values()) <= 1e-10
