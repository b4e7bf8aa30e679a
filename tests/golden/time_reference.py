"""Time the reference's own CPU path (Numba + OpenBLAS) beside the oracle port.

Runs the reference package from the checkout named by ``COSMOFORGE_REFERENCE``
(imported through the stand-ins in ``_standins/``, inputs injected through the
in-memory seams, ``basis=False``) on the host's cores and prints one JSON
object.  The same workloads are timed through the oracle port (``oracle/``:
the C restatement of the pair kernels with OpenMP, LAPACK / OpenBLAS) so that
the port's speed relative to the reference is measured on one machine.

Protocol: ``NUMBA_NUM_THREADS`` = ``OPENBLAS_NUM_THREADS`` = the usable
cores, one untimed warm-up call (JIT compilation), then the median of
``--repeats`` timed calls (``time.perf_counter``).

Workloads:

* config 0 (TT nside 8, n = 480, 23 bandpowers): ``Fisher.run()`` +
  ``Spectra.run()`` + ``get_power_spectra()``, one map;
* config 3 (TQU nside 8, n = 1312): PICSLike lnL over 64 Sobol points
  (``_compute_likelihood_point`` per point after the reference's set-up);
* config 1 slices (TQU nside 16, n = 5952): the full problem keeps 276
  C^-1 dC_b matrices of 283 MB each (78 GB) and does not fit this host, so
  two slices of the Fisher axis (lmax 3 and 5: 12 and 24 of the 276
  parameters) are timed and the per-parameter cost taken from their
  difference.

Usage::

    COSMOFORGE_REFERENCE=<reference checkout> python tests/golden/time_reference.py [--repeats 3]
"""

from __future__ import annotations

import argparse
import json
import os
import platform
import statistics
import sys
import time
from pathlib import Path

HERE = Path(__file__).resolve().parent
REPO = HERE.parent.parent
if not os.environ.get("COSMOFORGE_REFERENCE"):
    raise SystemExit("set COSMOFORGE_REFERENCE to the root of a reference checkout")
REF = Path(os.environ["COSMOFORGE_REFERENCE"]) / "src"
try:
    CORES = len(os.sched_getaffinity(0))
except AttributeError:
    CORES = os.cpu_count() or 1
for var in ("NUMBA_NUM_THREADS", "OPENBLAS_NUM_THREADS", "OMP_NUM_THREADS"):
    os.environ[var] = str(CORES)
os.environ.setdefault("NUMBA_CACHE_DIR", "/tmp/cf_golden_numba_cache")
sys.path[:0] = [str(HERE / "_standins"), str(HERE), str(REPO), str(REF / "cosmoforge.cosmocore"),
                str(REF / "cosmoforge.qube"), str(REF / "cosmoforge.picslike")]

import numpy as np  # noqa: E402

from cosmoforge_b200 import workloads  # noqa: E402
from cosmoforge_b200.layout import build_layout  # noqa: E402


def _median_time(fn, repeats):
    fn()
    ts = []
    for _ in range(repeats):
        t0 = time.perf_counter()
        fn()
        ts.append(time.perf_counter() - t0)
    return statistics.median(ts), ts


def _draw(S, N, seed):
    C = S + N
    return np.linalg.cholesky(C) @ np.random.default_rng(seed).standard_normal((C.shape[0], 1))


def qml_reference(pb, maps):
    from qube import Fisher, Spectra

    def run():
        f = Fisher(pb.params, basis=False, mask=pb.mask, noise_cov1=pb.noise, cls_data=pb.cls, beam=pb.beam)
        f.run()
        s = Spectra(pb.params, fisher=f, basis=False, maps1=maps)
        s.run()
        s.get_power_spectra()

    return run


def qml_port(pb, maps):
    from oracle import oracle as orc

    L = build_layout(pb.params, pb.mask, pb.beam)

    def run():
        orc.qml_solve(L, pb.cls, pb.noise, maps)

    return run


def lnl_reference(pb, maps, thetas):
    from picslike import PICSLike
    from picslike.parameter_grid import ParameterGrid

    pl = PICSLike(pb.params, basis=False, mask=pb.mask, noise_cov1=pb.noise, cls_data=pb.cls,
                  fiducial_cls=pb.cls, beam=pb.beam, maps1=maps)
    pl.setup_fields()
    pl.setup_geometry()
    pl.setup_covariance_matrices()
    pl.setup_cls(lmax=pl.lmax_signal)
    pl.setup_beams(lmax=pl.lmax_signal)
    pl.setup_maps()
    keys = [(float(i),) for i in range(len(thetas))]
    pl.parameter_grid = ParameterGrid(
        core_params=pl.params, parameter_ranges={"idx": np.arange(len(thetas), dtype=float)},
        theoretical_spectra={k: workloads.model_cls(t, pl.lmax_signal) for k, t in zip(keys, thetas)},
        lmax_signal=pl.lmax_signal)

    def run():
        for k in keys:
            pl._compute_likelihood_point(k)

    return run


def lnl_port(pb, maps, thetas):
    from oracle import oracle as orc

    L = build_layout(pb.params, pb.mask, pb.beam)

    def run():
        for t in thetas:
            orc.lnl_point(L, workloads.model_cls(t, L.lmax_signal), pb.noise, maps)

    return run


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--repeats", type=int, default=3)
    ap.add_argument("--skip-config1", action="store_true")
    a = ap.parse_args()
    out = {"cores": CORES, "cpu": platform.processor() or platform.machine(), "repeats": a.repeats}
    try:
        out["cpu"] = next(ln.split(":", 1)[1].strip() for ln in open("/proc/cpuinfo") if "model name" in ln)
    except (OSError, StopIteration):
        pass

    pb0 = workloads.config0()
    L0 = build_layout(pb0.params, pb0.mask, pb0.beam)
    from oracle import oracle as orc

    maps0 = _draw(orc.signal_matrix(L0, L0.smoothed_cl_table(pb0.cls)), pb0.noise, 0)
    for name, mk in (("reference", qml_reference), ("port", qml_port)):
        t, ts = _median_time(mk(pb0, maps0), a.repeats)
        out[f"config0_{name}"] = {"seconds_per_solve": t, "solves_per_s": 1.0 / t, "runs_s": ts}

    pb3 = workloads.config3()
    L3 = build_layout(pb3.params, pb3.mask, pb3.beam)
    maps3 = _draw(orc.signal_matrix(L3, L3.smoothed_cl_table(pb3.cls)), pb3.noise, 0)
    th = workloads.sobol_points(64, seed=5)
    th[:, 4] = 1.0  # the reference keeps N fixed
    for name, mk in (("reference", lnl_reference), ("port", lnl_port)):
        t, ts = _median_time(mk(pb3, maps3, th), a.repeats)
        out[f"config3_{name}"] = {"points": len(th), "seconds": t, "evals_per_s": len(th) / t, "runs_s": ts}

    if not a.skip_config1:
        res = {}
        for lmax in (3, 5):
            pb1 = workloads.config1(lmax=lmax)
            L1 = build_layout(pb1.params, pb1.mask, pb1.beam)
            maps1 = np.random.default_rng(0).standard_normal((L1.n, 1)) * 30.0
            for name, mk in (("reference", qml_reference), ("port", qml_port)):
                fn = mk(pb1, maps1)
                t0 = time.perf_counter()
                fn()  # one call each: minutes at this size
                res[(name, L1.n_params)] = time.perf_counter() - t0
        for name in ("reference", "port"):
            t12, t24 = res[(name, 12)], res[(name, 24)]
            t_param = (t24 - t12) / 12.0
            t_fixed = t12 - 12 * t_param
            out[f"config1_slices_{name}"] = {
                "seconds_12_params": t12, "seconds_24_params": t24, "seconds_per_param": t_param,
                "seconds_fixed": t_fixed,
                "extrapolated_seconds_per_276_param_solve_linear": t_fixed + 276 * t_param,
                "note": "linear in the parameter count; the 276 x 277 / 2 Fisher traces of the full "
                        "solve grow quadratically and are not in this figure"}
    print(json.dumps(out, indent=1))


if __name__ == "__main__":
    main()
