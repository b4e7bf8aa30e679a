"""Drop-in ``Fisher`` and ``Spectra`` with the reference's constructor and outputs.

Same signatures, seams and result layouts as ``qube.Fisher``
(``qube/fisher.py:141-266, 826-1049``) and ``qube.Spectra``
(``qube/spectra.py:205-395, 1358-1733``): the parameter axis is
spectrum-major, bin-minor in ``spectra_list`` order; power spectra are
(nsims, n_params); ``noise_cov1`` is rebound to C^-1 after ``run()`` and the
injected N stays in ``reduced_noise_cov1``.  The computation runs on the GPU
through ``libcfb200.so``; host copies of the n x n matrices are made only
when those attributes are read.

Supported: the pixel-space estimator (``basis=False`` / ``"pixel"``), the
harmonic basis (``"harmonic"``, see ``harmonic``), the default ``None`` /
``"auto"`` choosing between them by the reference's cost model, SYMMETRIC
spectra, auto-spectra (``do_cross=False``), injected arrays or the
reference's file inputs (``maskfile``, ``covmatfile1`` / ``load_reduced``,
``inputclfile``, ``smoothing_type`` file / gaussian / none with
``beam_file`` / ``fwhmarcmin``, ``inputmapfile1``; ``fileio``), and the
compressed pixel basis (``basis={"method": "pixel", "epsilon": ...}`` or
``"mode_fraction"``; ``harmonic.CompressedPlan``).  Pixel filters raise
``NotImplementedError``.

``precision``: ``"fp64"`` (plain FP64 everywhere) or ``"mixed"`` (BF16x3 /
FP32 tensor-core traces with FP64 refinement, see ``engine_mixed``) on the
pixel-space path; the harmonic basis always runs in FP64.
"""

from __future__ import annotations

import numpy as np
import torch

from . import engine as eng
from . import fileio
from . import layout as lay
from . import params as prm

_LAYOUT_CACHE: dict = {}


def _layout(p: dict, mask, beam) -> lay.Layout:
    """Layouts are pure functions of (geometry params, mask, beam): cache them."""
    mask = np.asarray(mask, dtype=np.float64)
    key = (p["nside"], tuple(p["spins"]), tuple(p["labels"]), p.get("ordering", "RING"),
           p.get("lmin"), p.get("lmax"), p.get("lmax_signal"), p.get("delta_ell"),
           str(p.get("bin_lmins")), str(p.get("bin_lmaxs")), p.get("output_convention"),
           bool(p.get("remove_nb", True)), mask.tobytes().__hash__(),
           None if beam is None else np.asarray(beam, dtype=np.float64).tobytes().__hash__())
    L = _LAYOUT_CACHE.get(key)
    if L is None:
        L = lay.build_layout(p, mask, beam)
        if len(_LAYOUT_CACHE) > 16:
            _LAYOUT_CACHE.clear()
        _LAYOUT_CACHE[key] = L
    L.nsims = int(p.get("nsims") or 1)
    return L


def _check_basis(basis):
    """The basis request as "pixel", "harmonic" or "auto" (cosmocore/core.py:135-160)."""
    if basis is False:
        return "pixel"
    if basis is None:
        return "auto"
    if isinstance(basis, str):
        if basis not in ("auto", "harmonic", "pixel"):
            raise ValueError(f"unknown basis {basis!r}; expected 'auto'/'harmonic'/'pixel', a dict, False or None")
        return basis
    if isinstance(basis, dict):
        method = basis.get("method", "auto")
        if method not in ("auto", "harmonic", "pixel"):
            raise ValueError(f"unknown basis method {method!r}")
        unknown = set(basis) - {"method", "epsilon", "mode_fraction", "compression_target", "C_ell"}
        if unknown:
            raise NotImplementedError(f"basis options {sorted(unknown)} are not implemented")
        if basis.get("epsilon") is not None or basis.get("mode_fraction") is not None:
            # compression intent: the V-based pixel basis (cosmocore/core.py:940-950)
            if method != "pixel":
                raise NotImplementedError(f"basis={basis!r}: compression is implemented for method='pixel' only")
            return "compressed"
        return method
    raise TypeError(f"basis must be None/False/str/dict, got {type(basis).__name__}")


def _compression_of(basis) -> dict:
    if not isinstance(basis, dict):
        return {}
    return dict(epsilon=basis.get("epsilon"), mode_fraction=basis.get("mode_fraction"),
                target=basis.get("compression_target", "noise_weighted"), C_ell=basis.get("C_ell"))


def _resolve_method(req: str, L) -> str:
    """"auto" by the reference's cost model (cosmocore/basis/__init__.py:87-115)."""
    if req != "auto":
        return req
    from .harmonic import auto_method, components

    # layouts the device harmonic basis does not take (more than three
    # components, lmin < 2) are served by the exact pixel path
    if L.lmin < 2 or len(components(L)) > 3:
        return "pixel"
    return auto_method(L)


def _check_kwargs(kwargs):
    for k in ("pixel_filter",):
        if kwargs.get(k) is not None:
            raise NotImplementedError(f"{k} is not supported by the device path")


class _Base:
    def __init__(self, params, params_file, mask, noise_cov1, noise_cov2, cls_data, fiducial_cls,
                 beam, precision, device, kwargs):
        self.params = prm.as_namespace(prm.resolve(params, params_file))
        _check_kwargs(kwargs)
        if self.params.do_cross:
            raise NotImplementedError("do_cross=True (two-map cross spectra) is not supported")
        p = self.params
        ncomp = sum(1 if s == 0 else 2 for s in p.spins)
        if mask is None:  # file adapter of cosmocore/core.py:403-472
            mf = getattr(p, "maskfile", None)
            if not mf:
                raise ValueError("no mask: inject mask= or set params.maskfile")
            mask = fileio.read_mask(str(mf), ncomp, str(getattr(p, "ordering", "RING")))
        if cls_data is None and fiducial_cls is None:
            cf = getattr(p, "inputclfile", None) or getattr(p, "fiducialfile", None)
            if not cf:
                raise ValueError("no spectra: inject cls_data= or set params.inputclfile")
            cls_data = fileio.read_cls(str(cf), self.lmax_signal, getattr(p, "input_convention", "Cl"))
        if beam is None:
            kind = str(getattr(p, "smoothing_type", "none")).lower()
            if kind in ("file", "gaussian"):
                beam = fileio.read_beam(p, self.lmax_signal)
            elif kind != "none":
                raise NotImplementedError(f"smoothing_type={kind!r} without an injected beam")
        if noise_cov1 is None and not getattr(p, "covmatfile1", None):
            raise ValueError("no noise covariance: inject noise_cov1= or set params.covmatfile1")
        self._mask = mask
        self._noise_in = noise_cov1  # None: read from covmatfile1 once the layout is known
        self._cls = cls_data if cls_data is not None else fiducial_cls
        self._fid = fiducial_cls if fiducial_cls is not None else self._cls
        self._beam = beam
        if precision not in ("fp64", "mixed"):
            raise ValueError(f"precision must be 'fp64' or 'mixed', got {precision!r}")
        self.precision = precision
        self.device = torch.device(device) if device is not None else torch.device("cuda")
        self.rank = 0
        self.size = 1

    @property
    def lmax_signal(self) -> int:
        v = getattr(self.params, "lmax_signal", None)
        return 4 * self.params.nside if v is None else int(v)

    def _setup(self):
        p = vars(self.params)
        self.layout = _layout(p, self._mask, self._beam)
        L = self.layout
        n = L.n
        if self._noise_in is None:  # cosmocore/core.py:577-700
            path = str(self.params.covmatfile1)
            if getattr(self.params, "load_reduced", False):
                self._noise_in = fileio.read_covmat_reduced(path, n)
            else:
                ncomp = sum(1 if f.spin == 0 else 2 for f in L.fields)
                self._noise_in = fileio.read_covmat(path, 12 * L.nside ** 2, ncomp, fileio.active_indices(L))
        N = self._noise_in
        if isinstance(N, torch.Tensor):
            if tuple(N.shape) != (n, n):
                raise ValueError(f"injected noise covariance has shape {tuple(N.shape)}, expected ({n}, {n})")
            self._dev_N = N.to(self.device, torch.float64)
        else:
            N = np.asarray(N, dtype=np.float64)
            if N.shape != (n, n):
                raise ValueError(f"injected noise covariance has shape {N.shape}, expected ({n}, {n})")
            self._dev_N = torch.from_numpy(np.ascontiguousarray(N)).to(self.device, non_blocking=True)
        self.npixs = [f.npix for f in L.fields]
        self.spectra_list = L.labels()
        self.beam_smoothing = L.beam_smoothing_vector()
        self.n_params = L.n_params
        self.bins = lay_bins(L)


def _read_maps_file(obj):
    """Maps from params.inputmapfile1 (file adapter of cosmocore/core.py:700-716)."""
    p, L = obj.params, obj.layout
    phys = getattr(p, "physical_labels", None)
    if not phys:
        phys = []
        k = 0
        for f in L.fields:
            if f.spin == 0:
                phys.append(str(p.labels[k]))
                k += 1
            else:
                phys += ["Q", "U"]
                k += 2
    pixact = [f.pixels for f in L.fields for _ in range(1 if f.spin == 0 else 2)]
    nsims = int(getattr(p, "nsims", None) or 1)
    return fileio.read_maps(str(p.inputmapfile1), pixact, list(phys), nsims)


class lay_bins:
    """Read-only view of the bins with the reference's attribute names."""

    def __init__(self, L: lay.Layout):
        self.lmins = np.asarray(L.bin_lmins)
        self.lmaxs = np.asarray(L.bin_lmaxs)
        self.nbins = L.nbins
        self.lmin = int(self.lmins[0])
        self.lmax = int(self.lmaxs[-1])
        self.lmid = (self.lmins + self.lmaxs) / 2.0
        self.dl = self.lmaxs - self.lmins + 1


class Fisher(_Base):
    """Fisher matrix F_ij = 1/2 Tr[C^-1 dC^i C^-1 dC^j] on the GPU."""

    def __init__(self, params=None, basis=None, cache_derivatives: bool = False, symmetry_mode=None,
                 mask=None, noise_cov1=None, noise_cov2=None, cls_data=None, fiducial_cls=None,
                 beam=None, *, params_file=None, precision: str = "fp64", device=None, **kwargs):
        self._basis_req = _check_basis(basis)
        self._compression = _compression_of(basis)
        if symmetry_mode not in (None, "SYMMETRIC", "symmetric") and getattr(
                symmetry_mode, "name", "SYMMETRIC") != "SYMMETRIC":
            raise NotImplementedError("only SymmetryMode.SYMMETRIC is supported")
        super().__init__(params, params_file, mask, noise_cov1, noise_cov2, cls_data, fiducial_cls,
                         beam, precision, device, kwargs)
        self._cache_derivatives = cache_derivatives
        self.fisher = None
        self._dev_S = None
        self._dev_Cinv = None
        self._host = {}
        self.timings = {}

    # -- reference attributes, downloaded lazily --------------------------
    def _host_of(self, key, t):
        if key not in self._host:
            self._host[key] = t.cpu().numpy()
        return self._host[key]

    @property
    def signal_matrix(self):
        return None if self._dev_S is None else self._host_of("S", self._dev_S)

    @property
    def noise_cov1(self):
        if self._dev_Cinv is None:
            return self._noise_in
        return self._host_of("Cinv", self._dev_Cinv)

    @property
    def reduced_noise_cov1(self):
        return self._noise_in if self._dev_Cinv is not None else None

    # -- pipeline ---------------------------------------------------------
    def run(self) -> None:
        self._setup()
        L = self.layout
        self.engine = eng.Engine(L, self.device)
        self._host = {}
        self.method = _resolve_method(self._basis_req, L)
        self._hplan = self._cplan = None
        table = L.smoothed_cl_table(self._cls)
        if self.method in ("harmonic", "compressed"):
            from .harmonic import CompressedPlan, HarmonicPlan

            # S_fixed (multipoles outside the inference window) from the
            # fiducial spectra, the window from cls_data (cosmocore/core.py:950-1010)
            fixed = L.smoothed_cl_table(self._fid)
            self._hplan = HarmonicPlan(self.engine)
            self._dev_S = self._hplan.signal(table, fixed)
            C = self._dev_S + self._dev_N
            if self.method == "compressed":
                self._cplan = CompressedPlan(self._hplan, self._dev_N, fixed, **self._compression)
                self.dim = self._cplan.dim
                C = self._cplan.project(C)
        else:
            self._dev_S = self.engine.signal(table)
            C = self._dev_S + self._dev_N
        self._dev_Cinv = self.engine.spd_inverse(C)
        self.compute()

    def compute(self) -> None:
        self._dev_bias = None
        if self._cplan is not None:
            # compressed basis: the same contractions in the kept subspace
            F, self._dev_bias, _ = self._cplan.fisher_qml(self._dev_Cinv)
        elif self._hplan is not None:
            # harmonic basis (always FP64): F and the noise bias from
            # G = V C^-1 V^T and Z N Z^T; Spectra adds q from z = Z x
            F, self._dev_bias, _ = self._hplan.fisher_qml(self._dev_Cinv, self._dev_N)
        elif self.precision == "mixed":
            from . import engine_mixed

            # the noise bias needs only C^-1, N and dC_b: contract it against
            # the resident A_b slabs now instead of rebuilding dC_b in Spectra
            F, self._dev_bias, _ = engine_mixed.fisher_qml(self.engine, self._dev_Cinv, N=self._dev_N)
        else:
            F, _, _ = self.engine.fisher_qml(self._dev_Cinv)
        self._dev_F = F
        self.fisher = F.cpu().numpy()

    # -- accessors (qube/fisher.py:826-1049) -------------------------------
    def get_fisher_matrix(self):
        return self.fisher

    def get_window_matrix(self):
        return self.get_fisher_matrix()

    def get_error_bars(self, *, as_dict: bool = False):
        if self.fisher is None:
            return None
        Finv = self.engine.spd_inverse(self._dev_F.clone()).cpu().numpy()
        err = np.sqrt(np.diag(Finv))
        return self._to_dict(err) if as_dict else err

    def get_bandpower_slices(self):
        if self.spectra_list is None:
            return None
        return self.layout.bandpower_slices()

    def set_binning(self, bins) -> None:
        """Bins for the next run() (any object with ``lmins`` / ``lmaxs``; CC/core.py:1295-1326)."""
        self.params.bin_lmins = [int(v) for v in bins.lmins]
        self.params.bin_lmaxs = [int(v) for v in bins.lmaxs]
        self._bandpower_window = None

    def _compute_per_ell_fisher(self) -> torch.Tensor:
        """Fisher matrix with one bin per multipole, lmin..lmax, on the same C^-1.

        The reference re-runs its compute phase with Bins.fromdeltal(lmin, lmax, 1)
        (qube/fisher.py:1236-1268); the covariance does not depend on the binning,
        so the resident C^-1 is reused and only the derivatives change.
        """
        p = dict(vars(self.params))
        p.pop("bin_lmins", None)
        p.pop("bin_lmaxs", None)
        p["delta_ell"] = 1
        L1 = _layout(p, self._mask, self._beam)
        E1 = eng.Engine(L1, self.device)
        tables = (E1.deriv_tab, E1.deriv_bin, L1.nbins, L1.n_params)
        if getattr(self, "_cplan", None) is not None:
            return self._cplan.fisher_qml(self._dev_Cinv, with_bias=False, tables=tables)[0]
        if getattr(self, "_hplan", None) is not None:
            return self._hplan.fisher_qml(self._dev_Cinv, tables=tables)[0]
        if self.precision == "mixed":
            from . import engine_mixed

            return engine_mixed.fisher(E1, self._dev_Cinv)
        return E1.fisher_qml(self._dev_Cinv)[0]

    def get_bandpower_window_function(self, per_ell_fisher=None):
        """W = F_b^-1 Q F_perell, (nspectra nbins) x (nspectra n_ell) (qube/fisher.py:1050-1190).

        Q sums the multipoles of each bin; both Fisher matrices are spectrum-major.
        The per-multipole Fisher is computed on demand (and cached) unless given.
        """
        if self.fisher is None:
            raise ValueError("Bandpower window requires a completed Fisher run. Call run() first.")
        if per_ell_fisher is None and getattr(self, "_bandpower_window", None) is not None:
            return self._bandpower_window
        L = self.layout
        lmin, lmax = int(self.params.lmin), int(self.params.lmax)
        n_ell = lmax - lmin + 1
        if per_ell_fisher is None:
            Fpe = self._compute_per_ell_fisher()
        else:
            Fpe = torch.as_tensor(np.asarray(per_ell_fisher, dtype=np.float64), device=self.device)
        Qb = np.zeros((L.nbins, n_ell))
        for b, (lo, hi) in enumerate(zip(L.bin_lmins, L.bin_lmaxs)):
            Qb[b, lo - lmin: hi - lmin + 1] = 1.0
        Q = torch.as_tensor(np.kron(np.eye(L.nspectra), Qb), device=self.device).contiguous()
        E = self.engine
        QF = E.gemm(Q, Fpe.contiguous())
        Finv = E.spd_inverse(self._dev_F.clone())
        W = E.gemm(Finv, QF).cpu().numpy()
        if per_ell_fisher is None:
            self._bandpower_window = W
        return W

    def get_effective_ells(self):
        """Per bin, the window-weighted multipole sum_l W[b,l] l / sum_l W[b,l] (qube/fisher.py:1192-1234)."""
        if self.fisher is None:
            raise ValueError("get_effective_ells requires a completed Fisher run. Call run() first.")
        W = self.get_bandpower_window_function()
        L = self.layout
        lmin = int(self.params.lmin)
        n_ell = int(self.params.lmax) - lmin + 1
        ells = np.arange(lmin, lmin + n_ell, dtype=np.float64)
        nb = L.nbins
        eff = np.empty(L.nspectra * nb)
        for s in range(L.nspectra):
            Wb = W[s * nb:(s + 1) * nb, s * n_ell:(s + 1) * n_ell]
            eff[s * nb:(s + 1) * nb] = (Wb @ ells) / Wb.sum(axis=1)
        return eff

    def get_fisher_block(self, label_i: str, label_j: str | None = None):
        F = self.get_fisher_matrix()
        sl = self.get_bandpower_slices()
        if F is None or sl is None:
            return None
        label_j = label_i if label_j is None else label_j
        for lab in (label_i, label_j):
            if lab not in sl:
                raise KeyError(f"Unknown spectrum label {lab!r}. Legal labels: {list(sl)}")
        return F[sl[label_i], sl[label_j]]

    def _to_dict(self, flat):
        sl = self.layout.bandpower_slices()
        flat = np.asarray(flat)
        return {k: flat[..., v] for k, v in sl.items()}


class Spectra(_Base):
    """QML power spectra C_hat = (q - b) F^-1 on the GPU (qube/spectra.py)."""

    def __init__(self, params=None, fisher: Fisher | None = None, basis=None, mask=None,
                 noise_cov1=None, noise_cov2=None, cls_data=None, fiducial_cls=None, beam=None,
                 maps1=None, maps2=None, *, params_file=None, precision: str | None = None,
                 device=None, **kwargs):
        self._basis = basis
        _check_basis(basis)
        if fisher is not None:
            self.fisher_instance = fisher
            params = params if params is not None else vars(fisher.params)
            mask = fisher._mask if mask is None else mask
            noise_cov1 = fisher._noise_in if noise_cov1 is None else noise_cov1
            cls_data = fisher._cls if cls_data is None else cls_data
            beam = fisher._beam if beam is None else beam
            precision = precision or fisher.precision
            device = device if device is not None else fisher.device
        else:
            self.fisher_instance = None
        super().__init__(params, params_file, mask, noise_cov1, noise_cov2, cls_data, fiducial_cls,
                         beam, precision or "fp64", device, kwargs)
        if maps1 is None and not getattr(self.params, "inputmapfile1", None):
            raise ValueError("no maps: inject maps1= or set params.inputmapfile1")
        self._maps_in = maps1  # None: read from inputmapfile1 once the layout is known
        self.qml_results = None
        self.qml_noise_bias = None
        self.invfisher = None
        self.inv_fisher_sqrt = None

    def _fisher(self) -> Fisher:
        f = self.fisher_instance
        if f is None:
            f = Fisher(vars(self.params), basis=self._basis, mask=self._mask, noise_cov1=self._noise_in,
                       cls_data=self._cls, beam=self._beam, precision=self.precision,
                       device=self.device)
            self.fisher_instance = f
        if f.fisher is None:
            f.run()
        return f

    def setup(self) -> None:
        """Set-up phases of ``run()`` (qube/spectra.py:1220-1280): the Fisher run
        (or reuse), binning, maps, and F^-1 on the device."""
        f = self._fisher()
        self.layout = f.layout
        L = self.layout
        self.spectra_list = f.spectra_list
        self.beam_smoothing = f.beam_smoothing
        self.bins = f.bins
        self.n_params = L.n_params
        if self._maps_in is None:
            self._maps_in = _read_maps_file(self)
        maps = self._maps_in
        if isinstance(maps, torch.Tensor):
            X = maps.to(self.device, torch.float64)
        else:
            X = torch.from_numpy(np.ascontiguousarray(np.asarray(maps, dtype=np.float64)))
            X = X.to(self.device, non_blocking=True)
        nsims = self.params.nsims or X.shape[1]
        if tuple(X.shape) != (L.n, nsims):
            raise ValueError(f"injected maps have shape {tuple(X.shape)}, expected ({L.n}, {nsims})")
        self._dev_X = X
        self._dev_invF = f.engine.spd_inverse(f._dev_F.clone())
        self.invfisher = self._dev_invF.cpu().numpy()
        self.fisher_normalized = f.fisher

    def compute(self) -> None:
        """Raw q, noise bias and C_hat = (q - b) F^-1 (qube/spectra.py:1124-1218);
        runs the set-up first when it has not run."""
        if getattr(self, "_dev_invF", None) is None:
            self.setup()
        f = self.fisher_instance
        L, E, X = self.layout, f.engine, self._dev_X
        if getattr(f, "_cplan", None) is not None:
            _, _, q = f._cplan.fisher_qml(f._dev_Cinv, with_bias=False, maps=X, want_fisher=False)
            bias = f._dev_bias
        elif getattr(f, "_hplan", None) is not None:
            _, _, q = f._hplan.fisher_qml(f._dev_Cinv, None, X, want_fisher=False)
            bias = f._dev_bias
        elif self.precision == "mixed" and getattr(f, "_dev_bias", None) is not None:
            _, _, q = E.fisher_qml(f._dev_Cinv, None, X, want_fisher=False)
            bias = f._dev_bias
        else:
            _, bias, q = E.fisher_qml(f._dev_Cinv, f._dev_N, X, want_fisher=False)
        if L.remove_nb:
            q = q - bias[None, :]
        self._dev_q = q
        self._dev_b = bias
        self._dev_clhat = E.gemm(q, self._dev_invF)
        self._dev_nb = E.gemm(bias[None, :], self._dev_invF)[0]
        self.qml_results = q.cpu().numpy()
        self.qml_noise_bias = bias.cpu().numpy()

    def run(self) -> None:
        self.setup()
        self.compute()

    # -- outputs (qube/spectra.py:1340-1733) -------------------------------
    def _inv_sqrt(self):
        if self.inv_fisher_sqrt is None:
            Fd = self.fisher_instance._dev_F
            w, V = torch.linalg.eigh(Fd)
            thr = w.max() * 1e-12
            inv = torch.where(w > thr, 1.0 / torch.sqrt(torch.clamp(w, min=1e-300)), torch.zeros_like(w))
            self.inv_fisher_sqrt = ((V * inv[None, :]) @ V.T).cpu().numpy()
        return self.inv_fisher_sqrt

    def get_power_spectra(self, mode: str = "deconvolved", *, as_dict: bool = False):
        valid = ("deconvolved", "decorrelated", "convolved")
        if mode not in valid:
            raise ValueError(f"mode must be one of {valid}, got '{mode}'")
        if self.qml_results is None:
            return None
        if mode == "deconvolved":
            res = self._dev_clhat.cpu().numpy()
        elif mode == "decorrelated":
            res = self.qml_results @ self._inv_sqrt()
        else:
            W = self.fisher_instance.fisher

            def convolve(theory):
                if isinstance(theory, dict):
                    theory = np.concatenate([np.asarray(theory[s]) for s in self.spectra_list])
                return W @ np.asarray(theory)

            y = self.qml_results
            if as_dict:
                return self._to_dict(y), W, convolve
            return y, W, convolve
        return self._to_dict(res) if as_dict else res

    def get_noise_bias(self):
        return None if self.qml_noise_bias is None else self._dev_nb.cpu().numpy()

    def get_covariance(self, mode: str = "deconvolved"):
        if mode == "deconvolved":
            return self.invfisher
        if mode == "decorrelated":
            return np.eye(self.n_params)
        if mode == "convolved":
            return self.fisher_instance.fisher
        raise ValueError(f"unknown mode {mode!r}")

    def get_error_bars(self, mode: str = "deconvolved", *, as_dict: bool = False):
        err = np.sqrt(np.diag(self.get_covariance(mode)))
        return self._to_dict(err) if as_dict else err

    def get_effective_ells(self, use_midpoint: bool = False):
        """Window-weighted multipole per bin (delegated to the Fisher run), or the
        bin midpoints with ``use_midpoint`` (qube/spectra.py:1686-1711)."""
        if use_midpoint:
            return self.bins.lmid
        return self._fisher().get_effective_ells()

    def convolve_theory(self, cl_theory):
        """<y> = W C_theory with the window W of the raw estimates (qube/spectra.py:2039-2097);
        ``cl_theory`` is binned, spectrum-major, in the output convention."""
        W = self.fisher_instance.get_window_matrix() if self.fisher_instance is not None else None
        if W is None:
            return None
        return W @ np.asarray(cl_theory)

    def convolve_theory_for_inference(self, cl_theory):
        """Expected deconvolved bandpowers W_bp C_l of a per-multipole theory
        (qube/spectra.py:1735-1878): a dict {label: C_l} or a flat array of
        n_ell (l = lmin..lmax) or lmax + 1 (from l = 0) values per spectrum,
        spectrum-major; unbeamed, in the output convention."""
        f = self.fisher_instance
        if f is None:
            raise ValueError("convolve_theory_for_inference requires an attached Fisher instance. "
                             "Pass fisher=fisher to Spectra() at construction.")
        if getattr(f, "fisher", None) is None:
            raise ValueError("Fisher matrix has not been computed. Call fisher.run() "
                             "(and spectra.run()) before convolve_theory_for_inference().")
        lmin, lmax = int(self.params.lmin), int(self.params.lmax)
        n_ell = lmax - lmin + 1
        labels = list(f.layout.labels()) if getattr(f, "layout", None) is not None else None
        nspectra = len(labels) if labels is not None else 1

        def per_ell(arr, what):
            arr = np.asarray(arr, dtype=np.float64)
            if arr.ndim != 1:
                raise ValueError(f"{what} must be 1D, got shape {arr.shape}")
            if arr.size == n_ell:
                return arr
            if arr.size >= lmax + 1:
                return arr[lmin: lmax + 1]
            raise ValueError(f"{what} length {arr.size} does not match expected {n_ell} "
                             f"(l=lmin..lmax) or {lmax + 1} (l=0..lmax)")

        if isinstance(cl_theory, dict):
            missing = [lab for lab in labels if lab not in cl_theory]
            if missing:
                raise KeyError(f"cl_theory dict missing entries for: {missing}. Expected keys: {labels}")
            vec = np.concatenate([per_ell(cl_theory[lab], lab) for lab in labels])
        else:
            cl = np.asarray(cl_theory, dtype=np.float64)
            if cl.ndim != 1:
                raise ValueError(f"cl_theory must be 1D, got shape {cl.shape}")
            if nspectra > 1:
                if cl.size != nspectra * n_ell:
                    raise ValueError(f"cl_theory length {cl.size} does not match expected {nspectra * n_ell} "
                                     f"(nspectra*n_ell, spectrum-major) for a {nspectra}-spectrum run; "
                                     "or pass a label-keyed dict.")
                vec = cl
            else:
                vec = per_ell(cl, "cl_theory")
        W = f.get_bandpower_window_function()
        return None if W is None else W @ vec

    def write_power_spectra(self, mode: str = "deconvolved", filename: str | None = None,
                            include_errors: bool = True) -> None:
        """Mean spectra over simulations as a (bins x spectra) %.16e table, errors
        beside it; ``convolved`` writes the mean raw y and the window matrix
        (qube/spectra.py:2099-2240)."""
        valid = ("deconvolved", "decorrelated", "convolved")
        if mode not in valid:
            raise ValueError(f"mode must be one of {valid}, got '{mode}'")
        if filename is None:
            out = getattr(self.params, "outclfile", None)
            if out:
                parts = str(out).rsplit(".", 1)
                filename = f"{parts[0]}_{mode}.{parts[1] if len(parts) > 1 else 'dat'}"
            else:
                filename = f"spectra_{mode}.dat"
        parts = filename.rsplit(".", 1)

        def beside(tag):
            return f"{parts[0]}_{tag}.{parts[1]}" if len(parts) > 1 else f"{filename}_{tag}"

        if mode == "convolved":
            res = self.get_power_spectra(mode="convolved")
            if res is None:
                return
            y, W, _ = res
            np.savetxt(filename, np.mean(y, axis=0), header="Raw QML estimates (y vector, mean across simulations)")
            np.savetxt(beside("window"), W, header="Window matrix W: <y> = W @ C_true")
            return
        spectra = self.get_power_spectra(mode=mode)
        if spectra is None:
            return
        nb = self.layout.nbins

        def table(vec):
            return np.asarray(vec).reshape(-1, nb).T  # spectrum-major vector -> (bins, spectra)

        np.savetxt(filename, table(np.mean(spectra, axis=0)), fmt="%.16e")
        if include_errors:
            np.savetxt(beside("errors"), table(self.get_error_bars(mode=mode)), fmt="%.16e")

    def _to_dict(self, flat):
        sl = self.layout.bandpower_slices()
        flat = np.asarray(flat)
        return {k: flat[..., v] for k, v in sl.items()}


def draw_maps(L: lay.Layout, cls: dict, N: torch.Tensor, nsims: int, seed: int = 0,
              device=None) -> torch.Tensor:
    """x ~ N(0, S + N) drawn on the device: x = chol(C) z with z from ``seed``."""
    E = eng.Engine(L, device)
    C = E.signal(L.smoothed_cl_table(cls)) + N
    info = E.potrf(C)
    if int(info.abs().max()) != 0:
        raise ValueError("covariance is not positive definite")
    g = torch.Generator(device=C.device).manual_seed(int(seed))
    z = torch.randn((L.n, nsims), dtype=torch.float64, device=C.device, generator=g)
    return E.gemm(torch.tril(C), z)
