"""Pin the CPU oracle against the reference's outputs and Fortran known answers.

Tolerances follow the reference's own tests:
src/cosmoforge.qube/tests/test_fortran_validation.py:28-35 (S 1e-10,
C^-1 1e-12, F diagonal 1e-6, C_hat 1e-10, noise bias 1e-6),
src/cosmoforge.qube/tests/test_fisher.py:82-130 and test_spectra.py:85-120
(rtol 1e-5, atol 1e-3), src/cosmoforge.picslike/tests/
test_fortran_validation.py:37-42 (chi2, lnL 1e-9).  Against the reference's
own Python outputs (same inputs, same LAPACK) the bar is 1e-10 relative.
"""

import numpy as np
import pytest

from cosmoforge_b200 import workloads
from cosmoforge_b200.layout import build_layout
from golden_cases import QML_CASES, cls_of, load, noise_of, params_of
from oracle import oracle as orc


def _solve(name):
    d = load(name)
    L = build_layout(params_of(d), d["mask"], d["beam"])
    return d, L, orc.qml_solve(L, cls_of(d), noise_of(d), d["maps"])


@pytest.fixture(scope="module", params=QML_CASES)
def solved(request):
    return _solve(request.param)


def _rel(a, b):
    return float(np.max(np.abs(a - b)) / np.max(np.abs(b)))


def test_signal_matches_reference(solved):
    d, L, r = solved
    rows = d["s_rows_idx"]
    assert _rel(r["S"][rows], d["ref_signal_rows"]) <= 1e-13
    assert _rel(np.diag(r["S"]), d["ref_signal_diag"]) <= 1e-13


def test_inverse_matches_reference(solved):
    d, L, r = solved
    assert _rel(np.diag(r["Cinv"]), d["ref_cinv_diag"]) <= 1e-12


def test_fisher_matches_reference(solved):
    d, L, r = solved
    F, R = r["fisher"], d["ref_fisher"]
    corr = np.sqrt(np.outer(np.diag(R), np.diag(R)))
    assert np.max(np.abs(F - R) / corr) <= 1e-10
    np.testing.assert_allclose(L.beam_smoothing_vector(), d["ref_beam_smoothing"], rtol=1e-14)


def test_qml_matches_reference(solved):
    d, L, r = solved
    assert _rel(r["q"], d["ref_q_raw"]) <= 1e-10
    assert _rel(r["bias"], d["ref_noise_bias_raw"]) <= 1e-10
    assert _rel(r["clhat"], d["ref_clhat"]) <= 1e-10
    assert _rel(r["noise_bias"], d["ref_noise_bias"]) <= 1e-8


def test_labels_follow_reference_order(solved):
    d, L, _ = solved
    if "spectra_labels" in d:
        assert L.labels() == [str(s) for s in d["spectra_labels"]]


def test_fortran_qube_known_answers():
    d, L, r = _solve("fortran_qube_nside8_B")
    rows = d["s_rows_idx"]
    fs = d["fort_signal_rows"]
    rel = np.abs(r["S"][rows] - fs) / np.where(np.abs(fs) > 1e-20, np.abs(fs), 1.0)
    assert rel.max() < 1e-10
    assert np.max(np.abs(np.diag(r["Cinv"]) / d["fort_invcov_diag"] - 1)) < 1e-12
    b = L.beam_smoothing_vector()
    raw = r["fisher"] / np.outer(b, b)
    ell = np.arange(L.lmin, L.lmin + raw.shape[0], dtype=np.float64)
    dd = ell * (ell + 1) / (2 * np.pi)
    raw = raw * np.outer(dd, dd)
    assert np.max(np.abs(np.diag(raw) / d["fort_fisher_diag"] - 1)) < 1e-6
    n = min(r["clhat"].shape[1], d["fort_spectra"].shape[0])
    assert np.max(np.abs(r["clhat"][0, :n] / d["fort_spectra"][:n] - 1)) < 1e-10
    assert np.max(np.abs(r["noise_bias"][:n] / d["fort_noise_bias"][:n] - 1)) < 1e-6


@pytest.mark.parametrize("fields", ["T", "QU", "TQU", "TEB"])
def test_nside4_fortran_fisher_and_spectra(fields):
    d, L, r = _solve(f"nside4_{fields}")
    b = L.beam_smoothing_vector()
    np.testing.assert_allclose(r["fisher"] / np.outer(b, b), d["fort_fisher_raw"],
                               rtol=1e-5, atol=1e-3)
    np.testing.assert_allclose(r["clhat"], d["fort_spectra"], rtol=1e-5, atol=1e-3)


def test_picslike_fortran_known_answers():
    d = load("fortran_picslike_nside8_B")
    L = build_layout(params_of(d), d["mask"], d["beam"])
    for k in range(3):
        chi2, _, lnl = orc.lnl_point(L, {"BB": d["point_cl_BB"][k]}, d["noise"], d["maps"])
        assert abs(chi2[0] / d["fort_chi2"][k] - 1) < 1e-9
        assert abs(lnl[0] / d["fort_lnl"][k] - 1) < 1e-9
        assert abs(chi2[0] / d["ref_chi2"][k, 0] - 1) < 1e-12


def test_picslike_tqu_matches_reference():
    d = load("picslike_tqu_nside8")
    L = build_layout(params_of(d), d["mask"], d["beam"])
    for k in range(0, len(d["thetas"]), 3):
        cls = workloads.model_cls(d["thetas"][k], L.lmax_signal)
        chi2, _, lnl = orc.lnl_point(L, cls, np.diag(d["noise_diag"]), d["maps"])
        assert abs(chi2[0] / d["ref_chi2"][k, 0] - 1) < 1e-12
        assert abs(lnl[0] / d["ref_lnl"][k, 0] - 1) < 1e-12


def test_rotation_angle_degenerate_pairs():
    # Identical / antipodal pointings give a zero cross product: angles (0, 0)
    # (cosmocore/basics/geometry.py:85-86); a pole pointing takes the epsilon bump.
    v = np.array([0.3, 0.4, np.sqrt(1 - 0.25)])
    assert orc.rotation_angle(v, v) == (0.0, 0.0)
    assert orc.rotation_angle(v, -v) == (0.0, 0.0)
    a12, a21 = orc.rotation_angle(np.array([0.0, 0.0, 1.0]), np.array([1.0, 0.0, 0.0]))
    assert np.isfinite(a12) and np.isfinite(a21)
