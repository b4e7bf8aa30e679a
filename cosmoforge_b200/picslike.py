"""Drop-in ``PICSLike``: exact pixel likelihood over many parameter points.

Same constructor and outputs as ``picslike.PICSLike`` (``picslike/picslike.py:
160-250, 479-664, 812-853``): per point theta, C(theta) = S(theta) + N,
chi2 = x^T C^-1 x per simulation, ln|C| and lnL = -(chi2 + ln|C|)/2 (the 2 pi
constant omitted, as in the reference).  Points run in batches: one batched
build of S(theta) for all points of a batch, one batched Cholesky, and
chi2 / ln|C| from the factor, all on the GPU.  ``precision="mixed"`` factors
C in FP32 and refines chi2 in FP64 (one step against the FP64 C); ln|C| then
carries the FP32 factor's rounding.

The parameter grid is supplied in memory: ``parameter_grid`` is any object
with ``grid_points`` (list of tuples) and ``get_spectrum(point) -> {label:
C_l}`` (the interface of ``picslike.parameter_grid.ParameterGrid``), or a
``(points, spectra_fn)`` pair.  ``noise_scale_fn(point)`` optionally scales
N per point (the reference keeps N fixed; default 1).
"""

from __future__ import annotations

import numpy as np
import torch

from . import engine as eng
from .qube import _Base, _check_basis


class _ListGrid:
    def __init__(self, points, spectra_fn):
        self.grid_points = [tuple(np.atleast_1d(p).tolist()) for p in points]
        self._fn = spectra_fn

    def get_spectrum(self, point):
        return self._fn(point)

    def get_total_points(self):
        return len(self.grid_points)


class LikelihoodResult:
    """Per-point chi2 / lnL with the reference's accessor names."""

    def __init__(self, points, chi2, lnl):
        self.grid_points = points
        self.chi_squared_values = chi2
        self.log_likelihood_values = lnl

    def get_best_fit(self):
        k = int(np.argmax(self.log_likelihood_values))
        return self.grid_points[k], float(self.log_likelihood_values[k])


class PICSLike(_Base):
    def __init__(self, params=None, basis=None, mask=None, noise_cov1=None, noise_cov2=None,
                 cls_data=None, fiducial_cls=None, beam=None, maps1=None, maps2=None, *,
                 params_file=None, parameter_grid=None, noise_scale_fn=None, batch_size: int = 128,
                 precision: str = "fp64", device=None, **kwargs):
        # the likelihood is evaluated exactly in pixel space; "auto" / None are
        # served by that path, an explicit harmonic basis is not implemented
        if _check_basis(basis) in ("harmonic", "compressed"):
            raise NotImplementedError("PICSLike: harmonic / compressed bases are not implemented; use basis=False")
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
        if X.shape[0] != self.layout.n:
            raise ValueError(f"injected maps have {X.shape[0]} rows, expected {self.layout.n}")
        self._dev_X = X

    def compute_points(self, spectra: list, noise_scale=None):
        """chi2 (B, nsims), ln|C| (B,), lnL (B, nsims) for explicit spectra dicts."""
        L = self.layout
        chi2s, lds, lnls = [], [], []
        for b0 in range(0, len(spectra), self.batch_size):
            part = spectra[b0: b0 + self.batch_size]
            cl = np.stack([L.smoothed_cl_table(c) for c in part])
            sc = None if noise_scale is None else np.asarray(noise_scale[b0: b0 + len(part)], dtype=np.float64)
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

    def run(self):
        self.setup()
        self.compute()

    def compute(self):
        if self.parameter_grid is None:
            raise ValueError("parameter_grid is required (in-memory grid)")
        pts = list(self.parameter_grid.grid_points)
        spectra = [self.parameter_grid.get_spectrum(p) for p in pts]
        scale = None if self.noise_scale_fn is None else [self.noise_scale_fn(p) for p in pts]
        chi2, _, lnl = self.compute_points(spectra, scale)
        chi2 = chi2.cpu().numpy()
        lnl = lnl.cpu().numpy()
        self.simulation_results = [LikelihoodResult(pts, chi2[:, i], lnl[:, i])
                                   for i in range(chi2.shape[1])]
        self.likelihood_result = LikelihoodResult(pts, chi2.mean(axis=1), lnl.mean(axis=1))

    def get_log_likelihood(self):
        return None if self.likelihood_result is None else self.likelihood_result.log_likelihood_values

    def get_chi_squared(self):
        return None if self.likelihood_result is None else self.likelihood_result.chi_squared_values

    def get_best_fit(self):
        return None if self.likelihood_result is None else self.likelihood_result.get_best_fit()
