"""The Spectra drop-in's methods beyond run() (qube/spectra.py:1206-2240).

* ``compute()`` after ``setup()`` gives what ``run()`` gives (to rounding: atomics);
* ``convolve_theory_for_inference`` is W_bp C_l with the reference's own
  bandpower window (fixture ``bandpower_*``: the window
  ``get_bandpower_window_function`` returned in the reference run), for every
  accepted input form (dict, n_ell, lmax + 1, spectrum-major flat);
* ``get_effective_ells`` equals the reference's (and the bin midpoints with
  ``use_midpoint``);
* ``convolve_theory`` is F C_b (the window of the raw estimates);
* ``write_power_spectra`` writes the mean spectra and errors as (bins x
  spectra) tables and, in convolved mode, the mean y and the window.
"""

import numpy as np
import pytest

from golden_cases import cls_of, load, noise_of, params_of

pytestmark = pytest.mark.gpu


def _rel(a, b):
    return float(np.max(np.abs(np.asarray(a) - np.asarray(b))) / np.max(np.abs(np.asarray(b))))


@pytest.fixture(scope="module", params=["bandpower_tt_nside8", "bandpower_tqu_cut_nside4"])
def runs(request):
    from cosmoforge_b200 import qube

    d = load(request.param)
    p = params_of(d) | {"nsims": 2}
    f = qube.Fisher(p, basis=False, mask=d["mask"], noise_cov1=noise_of(d), cls_data=cls_of(d), beam=d["beam"])
    f.run()
    n = f.layout.n
    maps = np.random.default_rng(3).standard_normal((n, 2)) * 10.0
    s1 = qube.Spectra(p, fisher=f, maps1=maps)
    s1.run()
    s2 = qube.Spectra(p, fisher=f, maps1=maps)
    s2.setup()
    s2.compute()
    return d, p, f, s1, s2


def test_compute_after_setup_equals_run(runs):
    """Same kernels on the same inputs; the build-and-reduce kernel adds its
    per-block partial sums with atomics, so the two agree to rounding (q to
    1e-13; C_hat through F^-1 to the parity bar, 1e-10)."""
    _, _, _, s1, s2 = runs
    assert _rel(s2.qml_results, s1.qml_results) <= 1e-13
    assert _rel(s2.get_power_spectra(), s1.get_power_spectra()) <= 1e-10
    assert _rel(s2.get_noise_bias(), s1.get_noise_bias()) <= 1e-10


def test_convolve_theory_for_inference_all_input_forms(runs):
    d, p, f, s, _ = runs
    lmin, lmax = int(p["lmin"]), int(p["lmax"])
    n_ell = lmax - lmin + 1
    labels = f.layout.labels()
    rng = np.random.default_rng(0)
    th = {lab: rng.uniform(0.5, 2.0, lmax + 1) for lab in labels}
    vec = np.concatenate([th[lab][lmin: lmax + 1] for lab in labels])
    ref = d["ref_window"] @ vec
    assert _rel(s.convolve_theory_for_inference(th), ref) <= 1e-10
    if len(labels) == 1:
        assert _rel(s.convolve_theory_for_inference(th[labels[0]]), ref) <= 1e-10
        assert _rel(s.convolve_theory_for_inference(th[labels[0]][lmin:lmax + 1]), ref) <= 1e-10
    else:
        assert _rel(s.convolve_theory_for_inference(vec), ref) <= 1e-10
        with pytest.raises(ValueError):
            s.convolve_theory_for_inference(vec[:-1])
    with pytest.raises(KeyError):
        s.convolve_theory_for_inference({labels[0]: th[labels[0]]} if len(labels) > 1 else {"XX": vec})
    assert vec.size == len(labels) * n_ell


def test_effective_ells_and_convolve_theory(runs):
    d, _, f, s, _ = runs
    assert _rel(s.get_effective_ells(), d["ref_eff_ells"]) <= 1e-10
    assert np.array_equal(s.get_effective_ells(use_midpoint=True), s.bins.lmid)
    cb = np.random.default_rng(1).uniform(1, 2, f.layout.n_params)
    assert _rel(s.convolve_theory(cb), f.get_fisher_matrix() @ cb) <= 1e-14


def test_write_power_spectra(runs, tmp_path):
    _, _, f, s, _ = runs
    nb, ns = f.layout.nbins, f.layout.nspectra
    fn = str(tmp_path / "cl.dat")
    s.write_power_spectra(filename=fn)
    tab = np.loadtxt(fn).reshape(nb, ns)
    assert np.allclose(tab.T.ravel(), s.get_power_spectra().mean(axis=0), rtol=1e-15, atol=0)
    err = np.loadtxt(str(tmp_path / "cl_errors.dat")).reshape(nb, ns)
    assert np.allclose(err.T.ravel(), s.get_error_bars(), rtol=1e-15, atol=0)
    s.write_power_spectra(mode="convolved", filename=fn)
    assert np.allclose(np.loadtxt(fn), s.qml_results.mean(axis=0), rtol=1e-15, atol=0)
    assert np.allclose(np.loadtxt(str(tmp_path / "cl_window.dat")), f.get_fisher_matrix(), rtol=1e-15, atol=0)
    with pytest.raises(ValueError):
        s.write_power_spectra(mode="bogus")
