"""Host side of the PICSLike drop-in: the parameter grid read the reference's way.

``ParameterGrid`` (``picslike/parameter_grid.py:85-505``): Cartesian product
of the ranges in name order, theory files named
``<root_dir>/<root_filename>_<name><value:.6g>_....txt``, the fiducial kept
outside [lmin, lmax]; ``LikelihoodResult`` (``picslike/likelihood_result.py``):
best fit as a name -> value dict, marginals, highest-density intervals,
pickle round trip.  No device is needed.
"""

import math
from types import SimpleNamespace

import numpy as np
import pytest

from cosmoforge_b200.picslike import LikelihoodResult, ParameterGrid


def _write(path, cols: dict, lmax: int):
    ell = np.arange(2, lmax + 1, dtype=np.float64)
    labels = sorted(cols)
    np.savetxt(path, np.column_stack([ell] + [np.asarray(cols[k])[2:lmax + 1] for k in labels]),
               header="ell " + " ".join(labels))


def test_grid_from_files_blends_the_fiducial(tmp_path):
    lmax = 12
    core = SimpleNamespace(nside=4, lmin=3, lmax=8, fiducialfile=str(tmp_path / "fid.txt"),
                           input_convention="Cl")
    fid = {"TT": np.full(lmax + 1, 5.0)}
    _write(tmp_path / "fid.txt", fid, lmax)
    ranges = {"a": np.linspace(0.5, 1.5, 3), "b": np.array([1.0, 2.0])}
    for a in ranges["a"]:
        for b in ranges["b"]:
            _write(tmp_path / f"th_a{a:.6g}_b{b:.6g}.txt", {"TT": np.full(lmax + 1, a * b)}, lmax)
    g = ParameterGrid(core, ranges, root_dir=str(tmp_path), root_filename="th", lmax_signal=lmax)
    assert g.get_total_points() == 6 and g.get_grid_shape() == (3, 2)
    assert g.grid_points[1] == (0.5, 2.0)
    s = g.get_spectrum((1.5, 2.0))["TT"]
    assert np.all(s[3:9] == 3.0) and np.all(s[9:] == 5.0) and np.all(s[2:3] == 5.0)
    assert g.get_points_for_process(1, 4) == [g.grid_points[1], g.grid_points[5]]
    with pytest.raises(KeyError):
        g.get_spectrum((9.0, 9.0))


def test_missing_theory_file_or_spectrum_is_an_error(tmp_path):
    core = SimpleNamespace(nside=4, lmin=2, lmax=8)
    with pytest.raises(ValueError):
        ParameterGrid(core, {"a": np.array([1.0])}, theoretical_spectra={})
    with pytest.raises(ValueError):
        ParameterGrid(core, {"a": np.array([1.0])})


def test_likelihood_result_accessors(tmp_path):
    core = SimpleNamespace(nside=4)
    ranges = {"x": np.linspace(-2, 2, 41), "y": np.array([0.0, 1.0])}
    pts = [(x, y) for x in ranges["x"] for y in ranges["y"]]
    g = ParameterGrid(core, ranges, theoretical_spectra={p: {} for p in pts})
    chi2 = np.array([(x - 0.3) ** 2 / 0.25 + y for x, y in pts])
    r = LikelihoodResult(g, chi2, -0.5 * chi2)
    assert r.get_best_fit() == {"x": pytest.approx(0.3), "y": 0.0}
    lo, hi = r.get_confidence_intervals(0.68)["x"]
    assert lo < 0.3 < hi and hi - lo == pytest.approx(1.0, abs=0.15)
    m = r.get_marginalized_likelihood("y")
    assert m.sum() == pytest.approx(1.0) and m[0] / m[1] == pytest.approx(math.exp(0.5))
    r.save(tmp_path / "r.pkl")
    back = LikelihoodResult.load(tmp_path / "r.pkl")
    assert np.array_equal(back.chi_squared_values, chi2)
    with pytest.raises(ValueError):
        LikelihoodResult(g, chi2[:-1], chi2)
