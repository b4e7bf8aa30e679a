"""Drop-in ``PICSLike``: exact pixel likelihood over a parameter grid.

Same constructor, pipeline and outputs as ``picslike.PICSLike``
(``picslike/picslike.py:160-250, 377-431, 479-664, 666-853``): ``run()`` builds
the grid from ``params.parameters`` (``{name: [start, stop, num]}``, one
``numpy.linspace`` per name, Cartesian product) with theory spectra read from
``root_dir/root_filename_<name><value:.6g>...txt`` and blended with
``fiducialfile`` outside [lmin, lmax] (``picslike/parameter_grid.py:85-260``);
per point theta, C(theta) = S(theta) + N, chi2 = x^T C^-1 x per simulation,
ln|C| and lnL = -(chi2 + ln|C|)/2 (the 2 pi constant omitted, as in the
reference).  Results are one ``LikelihoodResult`` per simulation plus their
mean, with the reference's accessors (``RuntimeError`` before ``compute()``).

The points run in batches on the GPU: C(theta) = S(theta) + s N for all
points of a batch (one GEMM per block region against a per-multipole basis
built once, ``engine.SignalBasis``, for batches of 64 or more), one batched
Cholesky, and chi2 / ln|C| from the factor; a grid of more than one batch
replays one captured CUDA graph per batch (``engine.LnlGraph``).
``precision="mixed"`` factors C in FP32 and refines chi2 in FP64 (one step
against the FP64 C); ln|C| then carries the FP32 factor's rounding.

Extensions beyond the reference's signature (keyword-only): a grid supplied
in memory (``parameter_grid=``: a ``ParameterGrid``, any object with
``grid_points`` and ``get_spectrum(point)``, or a ``(points, spectra_fn)``
pair) used when ``params.parameters`` is empty; ``noise_scale_fn(point)``
scaling N per point (the reference keeps N fixed); ``batch_size``;
``precision``; ``device``.

Basis: the reference's traditional path (``basis=False``), ``"pixel"``
(pixel-direct, the same exact likelihood) and ``"harmonic"`` (its
Sherman-Morrison-Woodbury form, exact as well) all evaluate the full-rank
Gaussian of C = S + N; here every one of them is evaluated in pixel space,
which equals the reference's harmonic result to rounding.  Compressed bases
(``epsilon`` / ``mode_fraction``) change the likelihood and are not
implemented.
"""

from __future__ import annotations

import itertools
import pickle
from copy import deepcopy
from pathlib import Path

import numpy as np
import torch

from . import engine as eng
from . import fileio
from .qube import _Base, _check_basis


class ParameterGrid:
    """Parameter grid and theory spectra (``picslike/parameter_grid.py:85-505``).

    ``parameter_ranges``: {name: 1-D values}; the grid is their Cartesian
    product in name order.  Spectra are given as {point: {label: C_l}} or read
    from ``root_dir/root_filename_<name><value:.6g>_...txt`` with the
    fiducial (``core_params.fiducialfile``) kept outside [lmin, lmax].
    """

    def __init__(self, core_params, parameter_ranges: dict, theoretical_spectra: dict | None = None,
                 root_dir: str | None = None, root_filename: str | None = None,
                 lmax_signal: int | None = None):
        self.core_params = core_params
        self.lmax_signal = lmax_signal if lmax_signal is not None else 4 * int(core_params.nside)
        self.parameter_names = list(parameter_ranges.keys())
        self.parameter_ranges = deepcopy(parameter_ranges)
        self.grid_points = self._generate_grid_points()
        if theoretical_spectra is not None:
            self.theoretical_spectra = deepcopy(theoretical_spectra)
        else:
            if root_dir is None or root_filename is None:
                raise ValueError("Either theoretical_spectra or both root_dir and root_filename "
                                 "must be provided to read spectra from files.")
            self.root_dir = root_dir
            self.root_filename = root_filename
            self.read_theoretical_spectra()
        self._validate_spectra()

    def _generate_grid_points(self) -> list:
        if not self.parameter_ranges:
            return []
        return list(itertools.product(*[self.parameter_ranges[k] for k in self.parameter_names]))

    def point_filename(self, point) -> str:
        tag = "_".join(f"{self.parameter_names[i]}{v:.6g}" for i, v in enumerate(point))
        return f"{self.root_dir}/{self.root_filename}_{tag}.txt"

    def read_theoretical_spectra(self) -> None:
        p = self.core_params
        lmin, lmax = getattr(p, "lmin", None), getattr(p, "lmax", None)
        fid_file = getattr(p, "fiducialfile", None)
        conv = getattr(p, "input_convention", "Cl")
        fid = None
        if fid_file is not None and lmin is not None and lmax is not None:
            fid = fileio.read_cls(str(fid_file).strip(), self.lmax_signal, conv)
        self.theoretical_spectra = {}
        for point in self.grid_points:
            spec = fileio.read_cls(self.point_filename(point), self.lmax_signal, conv)
            self.theoretical_spectra[point] = (self._blend_spectra(spec, fid, int(lmin), int(lmax))
                                               if fid is not None else spec)

    @staticmethod
    def _blend_spectra(param_spectrum: dict, fiducial_spectrum: dict, lmin: int, lmax: int) -> dict:
        """Fiducial outside [lmin, lmax], the point's spectrum inside (l-indexed arrays)."""
        out = {}
        for key, arr in param_spectrum.items():
            if key not in fiducial_spectrum:
                out[key] = np.array(arr, copy=True)
                continue
            fid = fiducial_spectrum[key]
            n = min(len(arr), len(fid))
            res = np.array(fid[:n], copy=True)
            lo, hi = max(0, lmin), min(n - 1, lmax)
            if lo <= hi:
                res[lo: hi + 1] = arr[lo: hi + 1]
            out[key] = res
        return out

    def _validate_spectra(self) -> None:
        missing = [p for p in self.grid_points if p not in self.theoretical_spectra]
        if missing:
            raise ValueError(f"Missing theoretical spectra for {len(missing)} grid points")

    def get_total_points(self) -> int:
        return len(self.grid_points)

    def get_points_for_process(self, rank: int, size: int) -> list:
        if size <= 0:
            raise ValueError(f"Invalid MPI size: {size}")
        if rank < 0 or rank >= size:
            raise ValueError(f"Invalid MPI rank {rank} for size {size}")
        return self.grid_points[rank::size]

    def get_spectrum(self, param_point):
        try:
            return self.theoretical_spectra[param_point]
        except KeyError as exc:
            raise KeyError(f"No theoretical spectrum found for parameters: {param_point}") from exc

    def get_parameter_dict(self, param_point) -> dict:
        if len(param_point) != len(self.parameter_names):
            raise ValueError(f"Parameter point has {len(param_point)} values, "
                             f"expected {len(self.parameter_names)}")
        return dict(zip(self.parameter_names, param_point))

    def get_grid_shape(self) -> tuple:
        return tuple(len(self.parameter_ranges[k]) for k in self.parameter_names)

    def get_parameter_index(self, param_point) -> int:
        try:
            return self.grid_points.index(param_point)
        except ValueError as exc:
            raise ValueError(f"Parameter point {param_point} not found in grid") from exc

    def add_spectrum(self, param_point, spectrum) -> None:
        self.theoretical_spectra[param_point] = deepcopy(spectrum)

    def __len__(self) -> int:
        return len(self.grid_points)

    def __iter__(self):
        return iter(self.grid_points)

    def __contains__(self, param_point) -> bool:
        return param_point in self.grid_points


class _ListGrid:
    """Explicit points with a spectra function (in-memory grid of any shape)."""

    def __init__(self, points, spectra_fn, names=None):
        self.grid_points = [tuple(np.atleast_1d(p).tolist()) for p in points]
        self._fn = spectra_fn
        k = len(self.grid_points[0]) if self.grid_points else 0
        self.parameter_names = list(names) if names is not None else [f"p{i}" for i in range(k)]
        self.parameter_ranges = {nm: np.unique([p[i] for p in self.grid_points])
                                 for i, nm in enumerate(self.parameter_names)}

    def get_spectrum(self, point):
        return self._fn(point)

    def get_total_points(self):
        return len(self.grid_points)

    def get_parameter_dict(self, point) -> dict:
        return dict(zip(self.parameter_names, point))

    def __len__(self) -> int:
        return len(self.grid_points)


class LikelihoodResult:
    """chi2 / lnL per grid point (``picslike/likelihood_result.py:30-416``)."""

    def __init__(self, parameter_grid, chi_squared_values, log_likelihood_values):
        n = parameter_grid.get_total_points()
        if len(chi_squared_values) != n:
            raise ValueError(f"Chi-squared array length {len(chi_squared_values)} doesn't match grid size {n}")
        if len(log_likelihood_values) != n:
            raise ValueError(f"Log-likelihood array length {len(log_likelihood_values)} "
                             f"doesn't match grid size {n}")
        self.parameter_grid = parameter_grid
        self.chi_squared_values = np.array(chi_squared_values, copy=True)
        self.log_likelihood_values = np.array(log_likelihood_values, copy=True)
        self.likelihood_values = np.exp(self.log_likelihood_values - np.max(self.log_likelihood_values))

    def get_best_fit(self) -> dict:
        k = int(np.argmax(self.likelihood_values))
        return self.parameter_grid.get_parameter_dict(self.parameter_grid.grid_points[k])

    def get_chi_squared_minimum(self) -> float:
        return float(np.min(self.chi_squared_values))

    def get_maximum_likelihood(self) -> float:
        return float(np.max(self.likelihood_values))

    def get_marginalized_likelihood(self, parameter_name: str) -> np.ndarray:
        g = self.parameter_grid
        if parameter_name not in g.parameter_names:
            raise ValueError(f"Parameter '{parameter_name}' not found in grid")
        i = g.parameter_names.index(parameter_name)
        vals = np.asarray(g.parameter_ranges[parameter_name])
        coord = np.array([p[i] for p in g.grid_points])
        marg = np.array([self.likelihood_values[coord == v].sum() for v in vals])
        tot = marg.sum()
        return marg / tot if tot > 0 else marg

    def get_confidence_intervals(self, confidence_level: float = 0.68) -> dict:
        """Highest-density interval per parameter on its marginal: grid values
        taken by decreasing likelihood until their mass reaches the level; the
        bounds are the extreme values kept."""
        out = {}
        for name in self.parameter_grid.parameter_names:
            vals = np.asarray(self.parameter_grid.parameter_ranges[name])
            lk = self.get_marginalized_likelihood(name)
            tot = lk.sum()
            if tot == 0:
                out[name] = (float(vals[0]), float(vals[-1]))
                continue
            order = np.argsort(lk)[::-1]
            mass = np.cumsum(lk[order]) / tot
            keep = vals[order[: int(np.searchsorted(mass, confidence_level)) + 1]]
            out[name] = (float(keep.min()), float(keep.max()))
        return out

    def get_summary_statistics(self) -> dict:
        return {"best_fit_parameters": self.get_best_fit(),
                "chi_squared_minimum": self.get_chi_squared_minimum(),
                "maximum_likelihood": self.get_maximum_likelihood(),
                "confidence_intervals_68": self.get_confidence_intervals(0.68),
                "confidence_intervals_95": self.get_confidence_intervals(0.95),
                "total_parameter_points": len(self.parameter_grid),
                "parameter_names": list(self.parameter_grid.parameter_names)}

    def save(self, output_path) -> None:
        output_path = Path(output_path)
        output_path.parent.mkdir(parents=True, exist_ok=True)
        with open(output_path, "wb") as fh:
            pickle.dump(self, fh)

    @classmethod
    def load(cls, input_path) -> "LikelihoodResult":
        input_path = Path(input_path)
        if not input_path.exists():
            raise FileNotFoundError(f"Results file not found: {input_path}")
        with open(input_path, "rb") as fh:
            return pickle.load(fh)

    def __repr__(self) -> str:
        return (f"LikelihoodResult(parameters={len(self.parameter_grid.parameter_names)}, "
                f"grid_points={len(self.parameter_grid)}, chi2_min={self.get_chi_squared_minimum():.3f})")


_NOT_COMPUTED = "Likelihood not computed. Call compute_likelihood_grid() first."


class PICSLike(_Base):
    def __init__(self, params=None, basis=None, mask=None, noise_cov1=None, noise_cov2=None,
                 cls_data=None, fiducial_cls=None, beam=None, maps1=None, maps2=None, *,
                 params_file=None, parameter_grid=None, noise_scale_fn=None, batch_size: int = 256,
                 precision: str = "fp64", device=None, **kwargs):
        if _check_basis(basis) == "compressed":
            raise NotImplementedError("PICSLike: compressed bases (epsilon / mode_fraction) are not implemented")
        self._basis_req = _check_basis(basis)
        super().__init__(params, params_file, mask, noise_cov1, noise_cov2, cls_data, fiducial_cls,
                         beam, precision, device, kwargs)
        if maps1 is None and not getattr(self.params, "inputmapfile1", None):
            raise ValueError("no maps: inject maps1= or set params.inputmapfile1")
        self._maps_in = maps1  # None: read from inputmapfile1 once the layout is known
        if isinstance(parameter_grid, tuple):
            parameter_grid = _ListGrid(*parameter_grid)
        self.parameter_grid = parameter_grid
        self.noise_scale_fn = noise_scale_fn
        self.batch_size = int(batch_size)
        self.likelihood_result = None
        self.simulation_results = None
        self.simulation_index = 0
        self.maps1 = None
        self.maps2 = None
        self._ready = False

    # -- set-up (picslike/picslike.py:334-431) ------------------------------
    def setup_parameter_grid(self) -> None:
        """Grid from ``params.parameters``: linspace per name, theory files blended with the fiducial."""
        spec = dict(getattr(self.params, "parameters", None) or {})
        if not spec:
            if self.parameter_grid is None:
                raise ValueError("no parameter grid: set params.parameters (with root_dir and "
                                 "root_filename) or pass parameter_grid=")
            return
        self.parameter_names = list(spec.keys())
        self.parameter_ranges = {k: np.linspace(*spec[k]) for k in self.parameter_names}
        self.parameter_grid = ParameterGrid(self.params, self.parameter_ranges,
                                            root_dir=getattr(self.params, "root_dir", None),
                                            root_filename=getattr(self.params, "root_filename", None),
                                            lmax_signal=self.lmax_signal)

    def setup(self):
        self._setup()
        self.engine = eng.Engine(self.layout, self.device)
        if self._maps_in is None:
            from .qube import _read_maps_file

            self._maps_in = _read_maps_file(self)
        X = self._maps_in
        if isinstance(X, torch.Tensor):
            X = X.to(self.device, torch.float64)
        else:
            X = torch.from_numpy(np.ascontiguousarray(np.asarray(X, dtype=np.float64))).to(self.device)
        if X.dim() == 1:
            X = X[:, None]
        if X.shape[0] != self.layout.n:
            raise ValueError(f"injected maps have {X.shape[0]} rows, expected {self.layout.n}")
        self._dev_X = X.contiguous()
        self.maps1 = self._maps_in
        self._ready = True

    def set_simulation_index(self, sim_idx: int) -> None:
        """Which simulation to report (0-based); checked against the maps' columns."""
        X = self.maps1 if self.maps1 is not None else self._maps_in
        if X is not None:
            ncol = 1 if np.ndim(X) == 1 else int(X.shape[1])
            if sim_idx < 0 or sim_idx > ncol - 1:
                raise ValueError(f"Simulation index {sim_idx} out of range [0, {ncol - 1}]")
        self.simulation_index = int(sim_idx)

    # -- evaluation ---------------------------------------------------------
    def compute_points(self, spectra: list, noise_scale=None):
        """chi2 (B, nsims), ln|C| (B,), lnL (B, nsims) on the device for explicit spectra dicts.

        Grids of more than one batch run every batch as a replay of one
        captured CUDA graph (engine.LnlGraph); a single batch runs eagerly."""
        L = self.layout
        chi2s, lds, lnls = [], [], []
        runner = None
        if len(spectra) > self.batch_size:
            key = (self.batch_size, self.precision)
            if getattr(self, "_graph_key", None) != key:
                self._graph = eng.LnlGraph(self.engine, self._dev_N, self._dev_X, self.batch_size, self.precision)
                self._graph_key = key
            runner = self._graph
        for b0 in range(0, len(spectra), self.batch_size):
            part = spectra[b0: b0 + self.batch_size]
            cl = np.stack([L.smoothed_cl_table(c) for c in part])
            sc = None if noise_scale is None else np.asarray(noise_scale[b0: b0 + len(part)], dtype=np.float64)
            if runner is not None:
                chi2, ld, lnl, info = runner(cl, sc)
            else:
                chi2, ld, lnl, info = self.engine.lnl(cl, self._dev_N, self._dev_X, noise_scale=sc,
                                                      precision=self.precision)
            bad = info.cpu().numpy()
            if np.any(bad != 0):
                k = int(np.flatnonzero(bad)[0])
                raise ValueError(f"dpotrf failed with info={int(bad[k])} at point {b0 + k}")
            chi2s.append(chi2)
            lds.append(ld)
            lnls.append(lnl)
        return torch.cat(chi2s), torch.cat(lds), torch.cat(lnls)

    def compute(self) -> None:
        """Likelihood over every grid point and simulation (picslike/picslike.py:479-546)."""
        if self.parameter_grid is None:
            raise ValueError("no parameter grid: call setup_parameter_grid() or pass parameter_grid=")
        if not self._ready:
            self.setup()
        grid = self.parameter_grid
        pts = list(grid.grid_points)
        spectra = [grid.get_spectrum(p) for p in pts]
        scale = None if self.noise_scale_fn is None else [self.noise_scale_fn(p) for p in pts]
        chi2, _, lnl = self.compute_points(spectra, scale)
        chi2 = chi2.cpu().numpy()
        lnl = lnl.cpu().numpy()
        self.simulation_results = [LikelihoodResult(grid, chi2[:, i], lnl[:, i]) for i in range(chi2.shape[1])]
        self.likelihood_result = LikelihoodResult(grid, chi2.mean(axis=1), lnl.mean(axis=1))

    def run(self) -> None:
        self.setup_parameter_grid()
        self.setup()
        self.compute()

    # -- outputs (picslike/picslike.py:666-800) -----------------------------
    def get_chi_squared(self) -> np.ndarray:
        if self.likelihood_result is None:
            raise RuntimeError(_NOT_COMPUTED)
        return self.likelihood_result.chi_squared_values

    def get_log_likelihood(self) -> np.ndarray:
        if self.likelihood_result is None:
            raise RuntimeError(_NOT_COMPUTED)
        return self.likelihood_result.log_likelihood_values

    def get_best_fit(self) -> dict:
        if self.likelihood_result is None:
            raise RuntimeError(_NOT_COMPUTED)
        return self.likelihood_result.get_best_fit()

    def get_simulation_results(self) -> list:
        if self.simulation_results is None:
            raise RuntimeError("Simulation results not available. Call compute() first.")
        return self.simulation_results

    def get_mean_likelihood_result(self) -> LikelihoodResult:
        if self.likelihood_result is None:
            raise RuntimeError("Likelihood not computed. Call compute() first.")
        return self.likelihood_result

    def save_results(self, output_path: str) -> None:
        """Mean result at ``output_path``, simulation i at ``<stem>_sim_<ii><suffix>`` beside it."""
        if self.likelihood_result is None:
            raise RuntimeError("No results to save. Run compute() first.")
        self.likelihood_result.save(output_path)
        base = Path(output_path)
        for i, r in enumerate(self.simulation_results or []):
            r.save(str(base.parent / f"{base.stem}_sim_{i:02d}{base.suffix}"))
