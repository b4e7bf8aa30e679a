"""The drop-in PICSLike class driven the reference's way, against the reference's outputs.

The grid comes from ``params.parameters`` ({name: [start, stop, num]}) with one
theory file per point under ``root_dir`` named
``<root_filename>_<name><value:.6g>.txt`` and the fiducial in
``fiducialfile``, as ``picslike/picslike.py:409-431`` and
``picslike/parameter_grid.py:85-260`` read them.  The test writes those files
from the fixture's spectra, runs ``PICSLike(params, basis=False, ...).run()``
and compares chi2 and lnL with the reference's run on the same inputs
(``tests/golden/make_golden.py``) at 1e-10 relative.  It also checks the
accessor contract (RuntimeError before compute, best fit as a name -> value
dict, one result per simulation, saved results that load back).  With
``basis="harmonic"`` the reference evaluates the same Gaussian by
Sherman-Morrison-Woodbury; this package evaluates it in pixel space and is
compared with the reference's harmonic run at 1e-9 (lnL) / 5e-9 (chi2).
"""

import math

import numpy as np
import pytest
import torch

from golden_cases import load, params_of

pytestmark = pytest.mark.gpu


def _write_table(path, spectra: dict, lmax: int, dl: bool):
    ell = np.arange(2, lmax + 1, dtype=np.float64)
    labels = sorted(spectra)
    cols = [ell]
    for k in labels:
        v = np.asarray(spectra[k], dtype=np.float64)[2: lmax + 1]
        cols.append(v * ell * (ell + 1.0) / (2.0 * math.pi) if dl else v)
    np.savetxt(path, np.column_stack(cols), fmt="%.18e", header="ell " + " ".join(labels))


def test_picslike_fortran_grid_from_files(tmp_path):
    from cosmoforge_b200.picslike import LikelihoodResult, PICSLike

    d = load("fortran_picslike_nside8_B")
    r_values = np.linspace(0.0, 2.5e-5, 3)
    lmax_sig = int(d["p_lmax_signal"])
    for r, cl in zip(r_values, d["point_cl_BB"]):
        _write_table(tmp_path / f"fine_dls_r_likelihood_r{r:.6g}.txt", {"BB": cl}, lmax_sig, dl=True)
    # outside [lmin, lmax] every point holds the fiducial
    _write_table(tmp_path / "fiducial_dls.txt", {"BB": d["point_cl_BB"][0]}, lmax_sig, dl=True)
    p = params_of(d) | dict(input_convention="Dl", parameters={"r": [0.0, 2.5e-05, 3]},
                            root_dir=str(tmp_path), root_filename="fine_dls_r_likelihood",
                            fiducialfile=str(tmp_path / "fiducial_dls.txt"))
    pl = PICSLike(p, basis=False, mask=d["mask"], noise_cov1=d["noise"],
                  cls_data={"BB": d["point_cl_BB"][0]}, beam=d["beam"], maps1=d["maps"])
    with pytest.raises(RuntimeError):
        pl.get_log_likelihood()
    with pytest.raises(RuntimeError):
        pl.get_best_fit()
    with pytest.raises(RuntimeError):
        pl.get_simulation_results()
    pl.run()
    assert pl.parameter_grid.get_total_points() == 3
    chi2, lnl = pl.get_chi_squared(), pl.get_log_likelihood()
    assert np.max(np.abs(chi2 / d["ref_chi2"][:, 0] - 1)) <= 1e-10
    assert np.max(np.abs(lnl / d["ref_lnl"][:, 0] - 1)) <= 1e-10
    assert np.max(np.abs(chi2 / d["fort_chi2"] - 1)) <= 1e-9
    bf = pl.get_best_fit()
    assert list(bf) == ["r"] and bf["r"] == float(r_values[int(np.argmax(d["ref_lnl"][:, 0]))])
    sims = pl.get_simulation_results()
    assert len(sims) == 1 and np.array_equal(sims[0].log_likelihood_values, lnl)
    with pytest.raises(ValueError):
        pl.set_simulation_index(1)
    pl.set_simulation_index(0)
    pl.save_results(str(tmp_path / "out" / "like.pkl"))
    back = LikelihoodResult.load(tmp_path / "out" / "like.pkl")
    assert np.array_equal(back.chi_squared_values, chi2)
    assert (tmp_path / "out" / "like_sim_00.pkl").exists()


@pytest.mark.parametrize("basis", [False, "pixel", "harmonic"])
def test_picslike_tqu_grid_from_files(tmp_path, basis):
    from cosmoforge_b200 import workloads
    from cosmoforge_b200.picslike import PICSLike

    d = load("picslike_tqu_nside8")
    p0 = params_of(d)
    lmax_sig = int(p0["lmax_signal"])
    thetas = d["thetas"]
    for i, t in enumerate(thetas):
        _write_table(tmp_path / f"tqu_idx{float(i):.6g}.txt", workloads.model_cls(t, lmax_sig), lmax_sig,
                     dl=False)
    fid = workloads.model_cls(workloads.THETA_CENTRE, lmax_sig)
    _write_table(tmp_path / "fid.txt", fid, lmax_sig, dl=False)
    p = p0 | dict(input_convention="Cl", parameters={"idx": [0.0, float(len(thetas) - 1), len(thetas)]},
                  root_dir=str(tmp_path), root_filename="tqu", fiducialfile=str(tmp_path / "fid.txt"))
    pl = PICSLike(p, basis=basis, mask=d["mask"], noise_cov1=np.diag(d["noise_diag"]), cls_data=fid,
                  beam=d["beam"], maps1=d["maps"], batch_size=3)
    pl.run()
    chi2, lnl = pl.get_chi_squared(), pl.get_log_likelihood()
    # the reference's harmonic branch (Sherman-Morrison-Woodbury) rounds
    # differently from its pixel path: 4e-10 (lnL) and 2e-9 (chi2) between them
    ref = load("picslike_tqu_harmonic_nside8") if basis == "harmonic" else d
    tol_chi2, tol_lnl = (5e-9, 1e-9) if basis == "harmonic" else (1e-10, 1e-10)
    ref_chi2, ref_lnl = ref["ref_chi2"].reshape(len(thetas), -1)[:, 0], ref["ref_lnl"].reshape(len(thetas), -1)[:, 0]
    assert np.max(np.abs(chi2 / ref_chi2 - 1)) <= tol_chi2
    assert np.max(np.abs(lnl / ref_lnl - 1)) <= tol_lnl
    assert pl.get_best_fit() == {"idx": float(np.argmax(ref_lnl))}


def test_picslike_in_memory_grid_and_mixed_precision():
    from types import SimpleNamespace

    from cosmoforge_b200 import workloads
    from cosmoforge_b200.picslike import ParameterGrid, PICSLike

    d = load("picslike_tqu_nside8")
    p = params_of(d)
    lmax_sig = int(p["lmax_signal"])
    spectra = {(float(i),): workloads.model_cls(t, lmax_sig) for i, t in enumerate(d["thetas"])}
    grid = ParameterGrid(SimpleNamespace(nside=int(p["nside"])), {"idx": np.arange(len(spectra), dtype=float)},
                         theoretical_spectra=spectra, lmax_signal=lmax_sig)
    for prec, tol in (("fp64", 1e-10), ("mixed", 3e-3)):
        pl = PICSLike(p, basis=False, mask=d["mask"], noise_cov1=np.diag(d["noise_diag"]),
                      cls_data=spectra[(0.0,)], beam=d["beam"], maps1=d["maps"], parameter_grid=grid,
                      precision=prec)
        pl.run()
        lnl = pl.get_log_likelihood()
        if prec == "fp64":
            assert np.max(np.abs(lnl / d["ref_lnl"][:, 0] - 1)) <= tol
        else:
            assert np.max(np.abs(lnl - d["ref_lnl"][:, 0])) <= tol


def test_graph_replayed_batches_equal_eager_batches():
    """PICSLike grids larger than one batch replay one captured CUDA graph per
    batch (engine.LnlGraph); the results equal a single eager batch bit for bit
    (every point's arithmetic is independent of the other points of its batch)."""
    from types import SimpleNamespace

    from cosmoforge_b200 import engine, workloads
    from cosmoforge_b200.layout import build_layout
    from cosmoforge_b200.picslike import ParameterGrid, PICSLike

    d = load("picslike_tqu_nside8")
    p = params_of(d)
    lmax_sig = int(p["lmax_signal"])
    spectra = {(float(i),): workloads.model_cls(t, lmax_sig) for i, t in enumerate(d["thetas"])}
    grid = ParameterGrid(SimpleNamespace(nside=8), {"idx": np.arange(len(spectra), dtype=float)},
                         theoretical_spectra=spectra, lmax_signal=lmax_sig)
    out = {}
    for bs in (3, 256):
        pl = PICSLike(p, basis=False, mask=d["mask"], noise_cov1=np.diag(d["noise_diag"]), cls_data=spectra[(0.0,)],
                      beam=d["beam"], maps1=d["maps"], parameter_grid=grid, batch_size=bs)
        pl.run()
        out[bs] = (pl.get_chi_squared(), pl.get_log_likelihood())
    assert np.array_equal(out[3][0], out[256][0]) and np.array_equal(out[3][1], out[256][1])

    # config 3, 200 points through a 128-point graph (a full and a partial replay), basis build
    pb = workloads.config3()
    L = build_layout(pb.params, pb.mask, pb.beam)
    E = engine.Engine(L)
    N = torch.from_numpy(pb.noise).cuda()
    g = torch.Generator(device="cuda").manual_seed(5)
    X = torch.randn((L.n, 1), dtype=torch.float64, device="cuda", generator=g) * 10.0
    th = workloads.sobol_points(200, seed=6)
    cl = np.stack([L.smoothed_cl_table(workloads.model_cls(t, L.lmax_signal)) for t in th])
    for prec in ("fp64", "mixed"):
        G = engine.LnlGraph(E, N, X, 128, precision=prec)
        got = [G(cl[b0:b0 + 128], th[b0:b0 + 128, 4]) for b0 in (0, 128)]
        lnl_g = torch.cat([r[2] for r in got]).cpu().numpy()
        _, _, lnl_e, info = E.lnl(cl, N, X, noise_scale=th[:, 4], precision=prec, build="basis")
        assert int(info.abs().max()) == 0
        assert np.array_equal(lnl_g, lnl_e.cpu().numpy()), prec
