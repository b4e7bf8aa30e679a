"""Generate the golden fixtures under ``tests/golden/`` from the reference.

This script is the only committed code that reads the reference tree.  It
runs the reference package (ggalloni/CosmoForge v1.3.0) from its sources,
importing it through the stand-ins in ``_standins/`` (a closed-form
``healpy`` and an ``astropy.io.fits`` import shim), with every input
injected through the in-memory seams and ``basis=False`` (the traditional
pixel path, the one the device path restates); the ``harmonic_*`` cases run
``basis="harmonic"`` on the inputs of a pixel-path fixture.  It writes one compressed
``.npz`` per case holding the inputs, the reference's outputs and, where the
reference's own tests ship them, the Fortran known answers.

Usage::

    COSMOFORGE_REFERENCE=<reference checkout> python tests/golden/make_golden.py [case ...]

``COSMOFORGE_REFERENCE`` names the root of a checkout of the reference
sources (the directory holding ``src/cosmoforge.*``).  The fixtures it
writes are small and committed, so tests never need the reference.
"""

from __future__ import annotations

import os
import sys
import time
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
REPO = HERE.parent.parent
if not os.environ.get("COSMOFORGE_REFERENCE"):
    raise SystemExit("set COSMOFORGE_REFERENCE to the root of a reference checkout")
REF = Path(os.environ["COSMOFORGE_REFERENCE"]) / "src"
QUBE_DATA = REF / "cosmoforge.qube" / "tests" / "data"
PL_DATA = REF / "cosmoforge.picslike" / "tests" / "data"

os.environ.setdefault("NUMBA_CACHE_DIR", "/tmp/cf_golden_numba_cache")
sys.path[:0] = [
    str(HERE / "_standins"),
    str(HERE),
    str(REPO),
    str(REF / "cosmoforge.cosmocore"),
    str(REF / "cosmoforge.qube"),
    str(REF / "cosmoforge.picslike"),
]

from fits_min import read_bintable, read_image_hdus  # noqa: E402

from cosmoforge_b200 import workloads  # noqa: E402


def _sample_rows(n: int, k: int = 12) -> np.ndarray:
    return np.unique(np.linspace(0, n - 1, k).astype(np.int64))


def _dl_to_cl(ell, dl):
    ell = np.asarray(ell, dtype=np.float64)
    out = np.zeros_like(dl)
    nz = ell > 0
    out[nz] = dl[nz] * 2.0 * np.pi / (ell[nz] * (ell[nz] + 1.0))
    return out


def _cls_from_dl_table(path, labels, lmax_signal):
    """{label: C_l} (l-indexed, physical) from a Dl text table with header."""
    with open(path) as fh:
        header = fh.readline().lstrip("#").split()
    tab = np.loadtxt(path)
    ell = tab[:, 0].astype(int)
    out = {}
    for lab in labels:
        col = header.index(lab) if lab in header else None
        cl = np.zeros(lmax_signal + 1)
        if col is not None:
            sel = ell <= lmax_signal
            cl[ell[sel]] = _dl_to_cl(ell[sel], tab[sel, col])
        out[lab] = cl
    return out


def _run_qml(params, mask, noise, cls, beam, maps):
    from qube import Fisher, Spectra

    t0 = time.perf_counter()
    f = Fisher(params, basis=False, mask=mask, noise_cov1=noise, cls_data=cls, beam=beam)
    f.run()
    t1 = time.perf_counter()
    s = None
    if maps is not None:
        s = Spectra(params, fisher=f, basis=False, maps1=maps)
        s.run()
    t2 = time.perf_counter()
    return f, s, (t1 - t0, t2 - t1)


def _run_qml_basis(params, mask, noise, cls, beam, maps, basis):
    from qube import Fisher, Spectra

    f = Fisher(params, basis=basis, mask=mask, noise_cov1=noise, cls_data=cls, fiducial_cls=cls, beam=beam)
    f.run()
    s = Spectra(params, fisher=f, basis=basis, maps1=maps)
    s.run()
    return f, s


def _spectra_labels(f):
    from cosmocore.conventions.cmb import spectrum_key_to_label

    return [spectrum_key_to_label(k, labels=list(f.params.labels), spins=tuple(f.params.spins))
            for k in f.spectra_list]


def _qml_outputs(f, s, prefix="ref_"):
    out = {
        prefix + "fisher": np.asarray(f.get_fisher_matrix()),
        prefix + "beam_smoothing": np.asarray(f.beam_smoothing),
        prefix + "cinv_diag": np.diag(f.noise_cov1).copy(),
    }
    S = f.signal_matrix
    rows = _sample_rows(S.shape[0])
    out["s_rows_idx"] = rows
    out[prefix + "signal_rows"] = np.ascontiguousarray(S[rows, :])
    out[prefix + "signal_diag"] = np.diag(S).copy()
    if s is not None:
        out[prefix + "q_raw"] = np.asarray(s.qml_results)
        out[prefix + "noise_bias_raw"] = np.asarray(s.qml_noise_bias)
        out[prefix + "clhat"] = np.asarray(s.get_power_spectra())
        out[prefix + "noise_bias"] = np.asarray(s.get_noise_bias())
        out[prefix + "invfisher"] = np.asarray(s.invfisher)
    return out


def _params_arrays(params):
    return {
        "p_nside": params["nside"],
        "p_spins": np.array(params["spins"]),
        "p_labels": np.array(params["labels"]),
        "p_lmin": params["lmin"],
        "p_lmax": params["lmax"],
        "p_lmax_signal": params["lmax_signal"],
        "p_output_convention": params.get("output_convention", "Cl"),
        "p_remove_nb": int(params.get("remove_nb", True)),
        "p_delta_ell": int(params.get("delta_ell", 1)),
    }


def _cls_arrays(cls):
    return {f"cl_{k}": np.asarray(v, dtype=np.float64) for k, v in cls.items()}


def _save(name, **arrays):
    path = HERE / f"{name}.npz"
    np.savez_compressed(path, **arrays)
    print(f"wrote {path.relative_to(REPO)} ({path.stat().st_size / 1024:.0f} KiB)")


def _draw_map(S, N, seed, nsims=1):
    C = S + N
    L = np.linalg.cholesky(C)
    z = np.random.default_rng(seed).standard_normal((C.shape[0], nsims))
    return L @ z


# --------------------------------------------------------------------------
# Cases
# --------------------------------------------------------------------------


def case_fortran_qube_nside8():
    """qube Fortran known answers: nside 8, full sky, one spin-0 field 'B'.

    Inputs mirror src/cosmoforge.qube/tests/data/nside8/B/fortran_reference/
    config.yaml (Dl in/out, injected beam, lmax 24, lmax_signal 32); checks
    follow src/cosmoforge.qube/tests/test_fortran_validation.py:26-175.
    """
    D = QUBE_DATA / "nside8" / "B" / "fortran_reference"
    mask = read_bintable(str(D / "mask.fits"))["T"]
    mp = read_bintable(str(D / "map.fits"))
    bt = read_bintable(str(D / "beam.fits"))
    L = 32
    beam = np.stack([bt["TEMPERATURE"][: L + 1], bt["GRADIENT"][: L + 1], bt["CURL"][: L + 1]])
    cls = _cls_from_dl_table(D / "input_dls.txt", ["BB"], L)
    n = int((mask > 0.5).sum())
    ncov = np.fromfile(D / "input_ncov.bin").reshape(n, n)
    assert np.count_nonzero(ncov - np.diag(np.diag(ncov))) == 0
    maps = mp["U_POLARISATION"][mask > 0.5][:, None]
    params = dict(nside=8, spins=[0], labels=["B"], lmin=2, lmax=24, lmax_signal=L,
                  delta_ell=1, ordering="RING", nsims=1, remove_nb=True,
                  input_convention="Dl", output_convention="Dl", smoothing_type="file",
                  apply_pixwin=False, do_cross=False, feedback=0)
    f, s, (tf, ts) = _run_qml(params, mask, ncov, cls, beam, maps)
    fort_S = np.fromfile(D / "signal.bin").reshape(n, n)
    rows = _sample_rows(n)
    out = dict(
        mask=mask[:, None], noise_diag=np.diag(ncov).copy(), maps=maps, beam=beam,
        **_cls_arrays(cls), **_params_arrays(params),
        **_qml_outputs(f, s),
        fort_signal_rows=np.ascontiguousarray(fort_S[rows, :]),
        fort_invcov_diag=np.diag(np.fromfile(D / "invcov.bin").reshape(n, n)).copy(),
        fort_fisher_diag=np.diag(np.loadtxt(D / "fisher.dat")).copy(),
        fort_spectra=np.loadtxt(D / "spectra.dat")[:, 1],
        fort_noise_bias=np.loadtxt(D / "noise_bias.dat")[:, 1],
        ref_time_fisher_s=tf, ref_time_spectra_s=ts,
    )
    _save("fortran_qube_nside8_B", **out)


def case_nside4(fields: str):
    """nside-4 traditional Fisher / spectra references for T, QU, TQU, TEB.

    Mirrors src/cosmoforge.qube/tests/test_fisher.py:82-130 and
    test_spectra.py:85-120 (full sky, lmax 8, Dl input, injected beam).
    """
    D = QUBE_DATA / "nside4" / fields
    import yaml

    cfg = yaml.safe_load(open(D / "config.yaml"))
    spins = cfg["spins"]
    labels = cfg["labels"]
    mk = read_bintable(str(D / "mask.fits"))
    mask = np.stack(list(mk.values()), axis=1)
    L = 16
    btab = read_bintable(str(REF / "cosmoforge.qube" / "scripts" / "beam_440TP_pixwin16.fits"))
    bcols = list(btab.values())
    beam = np.stack([bcols[0][: L + 1], bcols[1][: L + 1], bcols[2][: L + 1]])
    all_labels = []
    for sp, lab in zip(spins, _field_labels(spins, labels)):
        all_labels.append(lab)
    spec_labels = _all_spectra_labels(spins, labels)
    cls = _cls_from_dl_table(D / "dls.txt", spec_labels, L)
    ncov_full = np.fromfile(D / "NCVM1.bin")
    ntot = int(round(np.sqrt(ncov_full.size)))
    ncov_full = ncov_full.reshape(ntot, ntot)
    from cosmocore.geometry import active_pixel_index

    idx = active_pixel_index(mask)
    ncov = ncov_full[np.ix_(idx, idx)]
    assert np.count_nonzero(ncov - np.diag(np.diag(ncov))) == 0
    maps_file = QUBE_DATA / "nside4" / "maps" / ("all_sims_TEB.fits" if fields == "TEB" else "all_sims_TQU.fits")
    sims = read_image_hdus(str(maps_file))
    phys = cfg.get("physical_labels", labels)
    phys = [c for p in phys for c in (p if len(p) > 1 and p == "QU" else [p])]
    fmap = {"T": 0, "Q": 1, "U": 2, "E": 1, "B": 2}
    nsims = int(cfg["nsims"])
    npix = mask.shape[0]
    maps = np.empty((len(idx), nsims))
    for k in range(nsims):
        full = sims[f"SIM_{k:03d}"]  # (3, npix)
        vec = np.concatenate([full[fmap[lab]] for lab in phys])
        maps[:, k] = vec[idx]
    params = dict(nside=4, spins=spins, labels=labels, lmin=2, lmax=int(cfg["lmax"]),
                  lmax_signal=L, delta_ell=1, ordering="RING", nsims=nsims, remove_nb=True,
                  input_convention="Dl", output_convention="Cl", smoothing_type="file",
                  apply_pixwin=False, do_cross=False, feedback=0)
    if "physical_labels" in cfg:
        params["physical_labels"] = cfg["physical_labels"]
    f, s, (tf, ts) = _run_qml(params, mask, ncov, cls, beam, maps)
    out = dict(
        mask=mask, noise_diag=np.diag(ncov).copy(), maps=maps, beam=beam,
        **_cls_arrays(cls), **_params_arrays(params), **_qml_outputs(f, s),
        spectra_labels=np.array(_spectra_labels(f)),
        fort_fisher_raw=np.loadtxt(D / "ref_fisher.dat"),
        fort_spectra=np.loadtxt(D / "ref_spectra.txt"),
        ref_time_fisher_s=tf, ref_time_spectra_s=ts,
    )
    _save(f"nside4_{fields}", **out)


def _field_labels(spins, labels):
    out, c = [], 0
    for sp in spins:
        if sp == 0:
            out.append(labels[c])
            c += 1
        else:
            out.append(labels[c] + labels[c + 1])
            c += 2
    return out


def _all_spectra_labels(spins, labels):
    return ["TT", "EE", "BB", "TE", "TB", "EB"] if 2 in spins else [
        a + b for i, a in enumerate(labels) for b in labels[i:]]


def case_config0():
    """The spin-0 TT problem: nside 8, |z| > sin 20, l = 2..24, seed-0 map."""
    pb = workloads.config0()
    f, _, _ = _run_qml(pb.params, pb.mask, pb.noise, pb.cls, pb.beam, None)
    maps = _draw_map(f.signal_matrix, pb.noise, seed=0)
    # Warm timing (the first run above compiled the JIT kernels).
    f, s, (tf, ts) = _run_qml(pb.params, pb.mask, pb.noise, pb.cls, pb.beam, maps)
    out = dict(mask=pb.mask, noise_diag=pb.noise_diag, maps=maps, beam=pb.beam,
               **_cls_arrays(pb.cls), **_params_arrays(pb.params), **_qml_outputs(f, s),
               spectra_labels=np.array(_spectra_labels(f)),
               ref_time_fisher_s=tf, ref_time_spectra_s=ts)
    _save("config0_tt_nside8", **out)


def case_tqu_cut():
    """TQU with a |z| cut, a low-rank-plus-diagonal noise and two maps.

    A shrunken config-1 problem (nside 4, l = 2..10, lmax_signal 16) that
    exercises the spin-2 rotation angles on a cut sky and a dense N.
    """
    pb = workloads.config1(seed=3, nside=4, lmax=10, lmax_signal=16, n_lowrank=8)
    f, _, _ = _run_qml(pb.params | {"nsims": 2}, pb.mask, pb.noise, pb.cls, pb.beam, None)
    maps = _draw_map(f.signal_matrix, pb.noise, seed=1, nsims=2)
    f, s, (tf, ts) = _run_qml(pb.params | {"nsims": 2}, pb.mask, pb.noise, pb.cls, pb.beam, maps)
    out = dict(mask=pb.mask, noise=pb.noise, maps=maps, beam=pb.beam,
               **_cls_arrays(pb.cls), **_params_arrays(pb.params | {"nsims": 2}),
               **_qml_outputs(f, s), spectra_labels=np.array(_spectra_labels(f)),
               ref_time_fisher_s=tf, ref_time_spectra_s=ts)
    _save("tqu_cut_nside4", **out)


def _bandpower(params, mask, noise, cls, beam):
    """Reference Fisher with its bandpower window function and effective multipoles."""
    from qube import Fisher

    f = Fisher(params, basis=False, mask=mask, noise_cov1=noise, cls_data=cls, beam=beam)
    f.run()
    W = f.get_bandpower_window_function()
    eff = f.get_effective_ells()
    return f, W, eff


def case_bandpower_tt():
    """Bandpower window of the config-0 TT problem binned by 3 multipoles (l = 2..24)."""
    pb = workloads.config0()
    params = pb.params | {"delta_ell": 3}
    f, W, eff = _bandpower(params, pb.mask, pb.noise, pb.cls, pb.beam)
    _save("bandpower_tt_nside8", mask=pb.mask, noise_diag=pb.noise_diag, beam=pb.beam,
          **_cls_arrays(pb.cls), **_params_arrays(params), ref_fisher=f.get_fisher_matrix(),
          ref_window=W, ref_eff_ells=eff, spectra_labels=np.array(_spectra_labels(f)))


def case_bandpower_tqu():
    """Bandpower window of the cut-sky TQU case binned by 3 multipoles (l = 2..10)."""
    pb = workloads.config1(seed=3, nside=4, lmax=10, lmax_signal=16, n_lowrank=8)
    params = pb.params | {"delta_ell": 3}
    f, W, eff = _bandpower(params, pb.mask, pb.noise, pb.cls, pb.beam)
    _save("bandpower_tqu_cut_nside4", mask=pb.mask, noise=pb.noise, beam=pb.beam,
          **_cls_arrays(pb.cls), **_params_arrays(params), ref_fisher=f.get_fisher_matrix(),
          ref_window=W, ref_eff_ells=eff, spectra_labels=np.array(_spectra_labels(f)))


def _compressed_case(src: str, name: str, basis: dict):
    """The reference's compressed pixel basis (V-based, eigen-truncated) on the
    inputs of an existing pixel-path fixture."""
    d = np.load(HERE / f"{src}.npz")
    params = {"nside": int(d["p_nside"]), "spins": [int(x) for x in d["p_spins"]],
              "labels": [str(x) for x in d["p_labels"]], "lmin": int(d["p_lmin"]), "lmax": int(d["p_lmax"]),
              "lmax_signal": int(d["p_lmax_signal"]), "output_convention": str(d["p_output_convention"]),
              "remove_nb": bool(int(d["p_remove_nb"])), "nsims": int(d["maps"].shape[1])}
    noise = d["noise"] if "noise" in d.files else np.diag(d["noise_diag"])
    cls = {k[3:]: d[k] for k in d.files if k.startswith("cl_")}
    f, s = _run_qml_basis(params, d["mask"], noise, cls, d["beam"], d["maps"], dict(basis))
    out = {k: d[k] for k in d.files if not k.startswith("ref_") and not k.startswith("fort_")
           and k not in ("s_rows_idx",)}
    out.update(ref_fisher=np.asarray(f.get_fisher_matrix()), ref_q_raw=np.asarray(s.qml_results),
               ref_noise_bias_raw=np.asarray(s.qml_noise_bias), ref_clhat=np.asarray(s.get_power_spectra()),
               ref_noise_bias=np.asarray(s.get_noise_bias()), ref_invfisher=np.asarray(s.invfisher),
               ref_basis=np.array(repr({k: v for k, v in basis.items() if k != "C_ell"})),
               ref_dim=int(f.basis_manager.dim))
    _save(name, **out)


def _smoothed_cl(src: str) -> dict:
    """{label: C_l b_l^2} of a fixture's spectra with its beam (T, E, B rows): the
    beam-smoothed C_l a user passes as a compressed basis's ``C_ell``."""
    d = np.load(HERE / f"{src}.npz")
    beam = d["beam"]
    row = {"T": 0, "E": 1, "B": 2}
    out = {}
    for k in d.files:
        if k.startswith("cl_"):
            lab = k[3:]
            c = np.asarray(d[k], dtype=np.float64)
            n = min(c.size, beam.shape[1])
            out[lab] = c[:n] * beam[row[lab[0]], :n] * beam[row[lab[1]], :n]
    return out


def _harmonic_case(src: str, name: str):
    """The reference's harmonic-basis path (basis="harmonic") on the inputs of
    an existing pixel-path fixture: F, raw q, noise bias and C_hat."""
    d = np.load(HERE / f"{src}.npz")
    params = {"nside": int(d["p_nside"]), "spins": [int(x) for x in d["p_spins"]],
              "labels": [str(x) for x in d["p_labels"]], "lmin": int(d["p_lmin"]), "lmax": int(d["p_lmax"]),
              "lmax_signal": int(d["p_lmax_signal"]), "output_convention": str(d["p_output_convention"]),
              "remove_nb": bool(int(d["p_remove_nb"])), "nsims": int(d["maps"].shape[1])}
    noise = d["noise"] if "noise" in d.files else np.diag(d["noise_diag"])
    cls = {k[3:]: d[k] for k in d.files if k.startswith("cl_")}
    f, s = _run_qml_basis(params, d["mask"], noise, cls, d["beam"], d["maps"], "harmonic")
    out = {k: d[k] for k in d.files if not k.startswith("ref_") and not k.startswith("fort_")
           and k not in ("s_rows_idx",)}
    out.update(ref_fisher=np.asarray(f.get_fisher_matrix()), ref_q_raw=np.asarray(s.qml_results),
               ref_noise_bias_raw=np.asarray(s.qml_noise_bias), ref_clhat=np.asarray(s.get_power_spectra()),
               ref_noise_bias=np.asarray(s.get_noise_bias()), ref_invfisher=np.asarray(s.invfisher),
               ref_basis=np.array("harmonic"))
    _save(name, **out)


def _picslike_points(params, mask, noise, beam, maps, fid_cls, point_cls):
    """Run the reference PICSLike over explicit per-point spectra."""
    from picslike import PICSLike
    from picslike.parameter_grid import ParameterGrid

    pl = PICSLike(params, basis=False, mask=mask, noise_cov1=noise, cls_data=fid_cls,
                  fiducial_cls=fid_cls, beam=beam, maps1=maps)
    pl.setup_fields()
    pl.setup_geometry()
    pl.setup_covariance_matrices()
    pl.setup_cls(lmax=pl.lmax_signal)
    pl.setup_beams(lmax=pl.lmax_signal)
    pl.setup_maps()
    keys = [(float(i),) for i in range(len(point_cls))]
    pl.parameter_grid = ParameterGrid(
        core_params=pl.params, parameter_ranges={"idx": np.arange(len(point_cls), dtype=float)},
        theoretical_spectra={k: v for k, v in zip(keys, point_cls)}, lmax_signal=pl.lmax_signal)
    chi2, lnl = [], []
    t0 = time.perf_counter()
    for k in keys:
        c, l = pl._compute_likelihood_point(k)
        chi2.append(np.atleast_1d(c))
        lnl.append(np.atleast_1d(l))
    dt = time.perf_counter() - t0
    return np.array(chi2), np.array(lnl), dt, pl


def case_fortran_picslike_nside8():
    """PICSLike Fortran known answers (nside 8 full sky, field 'B', r grid).

    Mirrors src/cosmoforge.picslike/tests/test_fortran_validation.py:31-426:
    three r points of linspace(0, 2.5e-5, 3), lmin 2, lmax 16,
    lmax_signal 32, fiducial spectra outside [lmin, lmax].
    """
    D = PL_DATA / "nside8" / "B" / "fortran_reference"
    mask = read_bintable(str(D / "mask.fits"))["T"]
    mp = read_bintable(str(D / "map.fits"))
    bt = read_bintable(str(D / "beam.fits"))
    L = 32
    beam = np.stack([bt["TEMPERATURE"][: L + 1], bt["GRADIENT"][: L + 1], bt["CURL"][: L + 1]])
    n = int((mask > 0.5).sum())
    ncov = np.fromfile(D / "ncov_B_only.bin").reshape(n, n)
    maps = mp["U_POLARISATION"][mask > 0.5][:, None]
    fid = _cls_from_dl_table(D / "fiducial_dls.txt", ["BB"], L)
    r_values = np.linspace(0.0, 2.5e-5, 3)
    # The reference reads one theory file per r point; its file names carry
    # r formatted with %g.  Blend with the fiducial outside [lmin, lmax].
    point_cls = []
    for r in r_values:
        fname = D / "theory_spectra" / f"fine_dls_r_likelihood_r{r:g}.txt"
        th = _cls_from_dl_table(fname, ["BB"], L)
        bl = fid["BB"].copy()
        bl[2:17] = th["BB"][2:17]
        point_cls.append({"BB": bl})
    params = dict(nside=8, spins=[0], labels=["B"], lmin=2, lmax=16, lmax_signal=L,
                  ordering="RING", nsims=1, remove_nb=True, input_convention="Dl",
                  output_convention="Cl", smoothing_type="file", apply_pixwin=False,
                  do_cross=False, feedback=0)
    chi2, lnl, dt, _ = _picslike_points(params, mask, ncov, beam, maps, fid, point_cls)
    res = np.loadtxt(D / "results.txt")
    sel = res[:, 1] < 3
    out = dict(mask=mask[:, None], noise=ncov, maps=maps, beam=beam,
               point_cl_BB=np.stack([p["BB"] for p in point_cls]),
               **_params_arrays(params), ref_chi2=chi2, ref_lnl=lnl,
               fort_lnl=res[sel, 2], fort_chi2=res[sel, 3], ref_time_s=dt)
    _save("fortran_picslike_nside8_B", **out)


def case_picslike_tqu():
    """Five-parameter TQU likelihood on the nside-8 config-3 geometry.

    Eight scrambled-Sobol theta points; the noise scale s is fixed at 1
    because the reference's noise does not depend on theta.
    """
    pb = workloads.config3()
    thetas = workloads.sobol_points(8, seed=7)
    thetas[:, 4] = 1.0
    point_cls = [workloads.model_cls(t, pb.params["lmax_signal"]) for t in thetas]
    from qube import Fisher

    f = Fisher(pb.params, basis=False, mask=pb.mask, noise_cov1=pb.noise, cls_data=pb.cls,
               beam=pb.beam)
    f.run()
    maps = _draw_map(f.signal_matrix, pb.noise, seed=0)
    chi2, lnl, dt, _ = _picslike_points(pb.params, pb.mask, pb.noise, pb.beam, maps,
                                        pb.cls, point_cls)
    out = dict(mask=pb.mask, noise_diag=pb.noise_diag, maps=maps, beam=pb.beam,
               thetas=thetas, **_params_arrays(pb.params), ref_chi2=chi2, ref_lnl=lnl,
               ref_time_s=dt, ref_time_per_point_s=dt / len(thetas))
    _save("picslike_tqu_nside8", **out)



def case_picslike_tqu_harmonic():
    """The reference's PICSLike run end to end (``run()``) with ``basis="harmonic"``.

    Same inputs and points as ``picslike_tqu_nside8``; the grid is given the
    reference's way: ``params.parameters = {"idx": [0, 7, 8]}`` with one theory
    file per point (``root_dir/root_filename_idx<i>.txt``, C_l columns) and a
    fiducial file, as ``picslike/picslike.py:409-431`` reads them.  The harmonic
    branch evaluates chi2 and ln|C| by Sherman-Morrison-Woodbury
    (``picslike/picslike.py:597-622``).
    """
    import tempfile

    from picslike import PICSLike

    base = dict(np.load(HERE / "picslike_tqu_nside8.npz"))
    pb = workloads.config3()
    lmax_sig = int(pb.params["lmax_signal"])
    thetas = base["thetas"]

    def write(path, cls):
        ell = np.arange(2, lmax_sig + 1, dtype=np.float64)
        labels = sorted(cls)
        np.savetxt(path, np.column_stack([ell] + [np.asarray(cls[k])[2:lmax_sig + 1] for k in labels]),
                   fmt="%.18e", header="ell " + " ".join(labels))

    with tempfile.TemporaryDirectory() as tmp:
        for i, t in enumerate(thetas):
            write(f"{tmp}/tqu_idx{float(i):.6g}.txt", workloads.model_cls(t, lmax_sig))
        write(f"{tmp}/fid.txt", pb.cls)
        params = dict(pb.params, input_convention="Cl", root_dir=tmp, root_filename="tqu",
                      fiducialfile=f"{tmp}/fid.txt",
                      parameters={"idx": [0.0, float(len(thetas) - 1), len(thetas)]})
        pl = PICSLike(params, basis="harmonic", mask=pb.mask, noise_cov1=pb.noise, cls_data=pb.cls,
                      fiducial_cls=pb.cls, beam=pb.beam, maps1=base["maps"])
        t0 = time.perf_counter()
        pl.run()
        dt = time.perf_counter() - t0
    out = {k: base[k] for k in base if not k.startswith("ref_")}
    out.update(ref_chi2=np.asarray(pl.get_chi_squared()), ref_lnl=np.asarray(pl.get_log_likelihood()),
               ref_basis=np.array("harmonic"), ref_time_s=dt)
    _save("picslike_tqu_harmonic_nside8", **out)

CASES = {
    "fortran_qube": case_fortran_qube_nside8,
    "nside4_T": lambda: case_nside4("T"),
    "nside4_QU": lambda: case_nside4("QU"),
    "nside4_TQU": lambda: case_nside4("TQU"),
    "nside4_TEB": lambda: case_nside4("TEB"),
    "config0": case_config0,
    "tqu_cut": case_tqu_cut,
    "fortran_picslike": case_fortran_picslike_nside8,
    "picslike_tqu": case_picslike_tqu,
    "picslike_tqu_harmonic": case_picslike_tqu_harmonic,
    "bandpower_tt": case_bandpower_tt,
    "bandpower_tqu": case_bandpower_tqu,
    "harmonic_tqu_cut": lambda: _harmonic_case("tqu_cut_nside4", "harmonic_tqu_cut_nside4"),
    "harmonic_config0": lambda: _harmonic_case("config0_tt_nside8", "harmonic_config0_tt_nside8"),
    "harmonic_nside4_TEB": lambda: _harmonic_case("nside4_TEB", "harmonic_nside4_TEB"),
    "compressed_tqu_cut": lambda: _compressed_case("tqu_cut_nside4", "compressed_tqu_cut_nside4",
                                                   {"method": "pixel", "epsilon": 1e-3}),
    "compressed_config0": lambda: _compressed_case("config0_tt_nside8", "compressed_config0_tt_nside8",
                                                   {"method": "pixel", "epsilon": 1e-3}),
    "compressed_mf_tqu_cut": lambda: _compressed_case(
        "tqu_cut_nside4", "compressed_mf_tqu_cut_nside4", {"method": "pixel", "mode_fraction": [0.7, 0.6]}),
    "compressed_h_config0": lambda: _compressed_case(
        "config0_tt_nside8", "compressed_h_config0_tt_nside8",
        {"method": "pixel", "epsilon": 1e-2, "compression_target": "harmonic"}),
    "compressed_tc_config0": lambda: _compressed_case(
        "config0_tt_nside8", "compressed_tc_config0_tt_nside8",
        {"method": "pixel", "epsilon": 1e-3, "compression_target": "total_covariance",
         "C_ell": _smoothed_cl("config0_tt_nside8")["TT"]}),
    "compressed_snr_config0": lambda: _compressed_case(
        "config0_tt_nside8", "compressed_snr_config0_tt_nside8",
        {"method": "pixel", "epsilon": 1e-4, "compression_target": "snr",
         "C_ell": _smoothed_cl("config0_tt_nside8")["TT"]}),
    "compressed_eb_tqu_cut": lambda: _compressed_case(
        "tqu_cut_nside4", "compressed_eb_tqu_cut_nside4", {"method": "pixel", "epsilon": [1e-3, (1e-3, 1e-2)]}),
    "compressed_tc_eb_tqu_cut": lambda: _compressed_case(
        "tqu_cut_nside4", "compressed_tc_eb_tqu_cut_nside4",
        {"method": "pixel", "epsilon": [1e-3, (2e-3, 1e-2)], "compression_target": "total_covariance",
         "C_ell": {k: _smoothed_cl("tqu_cut_nside4")[k] for k in ("TT", "EE", "BB")}}),
}

if __name__ == "__main__":
    names = sys.argv[1:] or list(CASES)
    for nm in names:
        t = time.perf_counter()
        CASES[nm]()
        print(f"  {nm}: {time.perf_counter() - t:.1f} s")
