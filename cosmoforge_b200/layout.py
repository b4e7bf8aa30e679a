"""Host-side problem layout: fields, reduced pixel ordering, spectra, bins, weights.

Everything here is small host bookkeeping that turns the reference's params
and in-memory seams into the flat tables the device kernels read.  It
follows the reference's conventions exactly:

* fields and components from ``params.spins`` / ``params.labels``
  (``cosmocore/core.py:474-519``); a spin-2 field occupies ``[Q | U]`` rows;
* active pixels ``mask > 0.5`` per field, reduced vector = concatenated
  components (``cosmocore/geometry.py:94-134``);
* spectrum labels and their order: auto-spectra per field (spin 0: ``LL``;
  spin 2: ``EE, BB, EB``), then cross pairs ``i < j`` (spin 0 x spin 0:
  ``AB``; spin 0 x spin 2: ``TE, TB``) (``cosmocore/spectra_io.py:158-184``,
  ``cosmocore/fields.py:495-680``), which is also the Fisher parameter axis
  under ``SymmetryMode.SYMMETRIC`` (``qube/fisher.py:826-866``);
* beam smoothing ``C_l B_1(l) B_2(l)`` with beams keyed by field-map label
  T / E / B (``cosmocore/beam.py:128-219, 368-388``,
  ``cosmocore/spectra_io.py:446-494``);
* bins ``Bins.fromdeltal`` or explicit ``bin_lmins/bin_lmaxs`` and the
  shape weights ``w_l`` of ``output_convention`` (``cosmocore/bins.py``);
* the binned-derivative weights ``w_l b_l^2`` inside a bin
  (``cosmocore/core.py:1328-1409``, ``cosmocore/basis/pixel.py:850-857``).
"""

from __future__ import annotations

import math
from dataclasses import dataclass, field

import numpy as np

from . import healpix

# Block kinds understood by the device kernels.
KIND_00_AUTO = 0  # spin-0 field with itself
KIND_00_CROSS = 1  # two different spin-0 fields
KIND_22_AUTO = 2  # spin-2 field with itself (EE / BB / EB)
KIND_02 = 3  # spin-0 field (cols) x spin-2 field (rows)

_BEAM_ROW = {"T": 0, "E": 1, "B": 2}


@dataclass
class FieldSpec:
    spin: int
    labels: list  # 1 (spin 0) or 2 (spin 2) map labels
    pixels: np.ndarray  # active HEALPix pixel indices
    vectors: np.ndarray  # (n_pix, 3) unit pointings
    offset: int  # first row in the reduced vector

    @property
    def npix(self) -> int:
        return int(self.pixels.shape[0])

    @property
    def nrows(self) -> int:
        return self.npix * (2 if self.spin == 2 else 1)


@dataclass
class SpectrumSpec:
    label: str
    fi: int
    fj: int
    kind: int
    mode: int  # 22: 0 EE, 1 BB, 2 EB;  02: 0 TE, 1 TB;  00: 0
    map_labels: tuple  # the two field-map labels the label pairs


@dataclass
class BlockSpec:
    """One block of the signal matrix and the spectra feeding it."""

    kind: int
    fa: int  # column field (the lower-offset one)
    fb: int  # row field
    spectra: list  # indices into Layout.spectra, ordered per kind


@dataclass
class Layout:
    nside: int
    ordering: str
    fields: list
    spectra: list
    blocks: list
    lmin: int
    lmax: int
    lmax_signal: int
    bin_lmins: np.ndarray
    bin_lmaxs: np.ndarray
    shape_weights: np.ndarray  # (lmax_signal + 1,) w_l, zero beyond lmax
    beams: dict  # {"T": b_l, "E": b_l, "B": b_l} (lmax_signal + 1)
    remove_nb: bool = True
    nsims: int = 1
    output_convention: str = "Cl"
    extra: dict = field(default_factory=dict)

    # ---- sizes ---------------------------------------------------------
    @property
    def n(self) -> int:
        return int(sum(f.nrows for f in self.fields))

    @property
    def nbins(self) -> int:
        return int(self.bin_lmins.shape[0])

    @property
    def nspectra(self) -> int:
        return len(self.spectra)

    @property
    def n_params(self) -> int:
        return self.nspectra * self.nbins

    # ---- beams and spectra --------------------------------------------
    def smoothing(self, spec: SpectrumSpec) -> np.ndarray:
        """B_1(l) B_2(l) for a spectrum (ones when a beam is missing)."""
        a, b = spec.map_labels
        L = self.lmax_signal
        if a in self.beams and b in self.beams:
            return self.beams[a][: L + 1] * self.beams[b][: L + 1]
        return np.ones(L + 1)

    def beam_smoothing_vector(self) -> np.ndarray:
        """Fisher-row beam factors b_l^2 for l = lmin..lmax, per spectrum."""
        return np.concatenate(
            [self.smoothing(s)[self.lmin: self.lmax + 1] for s in self.spectra]
        ).astype(np.float64)

    def smoothed_cl_table(self, cls: dict) -> np.ndarray:
        """(nspectra, L + 1) beam-smoothed C_l in spectrum order."""
        L = self.lmax_signal
        out = np.zeros((self.nspectra, L + 1))
        for k, s in enumerate(self.spectra):
            if s.label not in cls:
                raise ValueError(f"Missing power spectrum for {s.label}")
            c = np.asarray(cls[s.label], dtype=np.float64)[: L + 1]
            out[k, : c.shape[0]] = c
            out[k] *= self.smoothing(s)
        return out

    def param_weights(self) -> np.ndarray:
        """(n_params, L + 1) per-parameter weights w_l b_l^2 inside each bin."""
        L = self.lmax_signal
        W = np.zeros((self.n_params, L + 1))
        for s_idx, s in enumerate(self.spectra):
            sm = self.smoothing(s)
            for b in range(self.nbins):
                lo, hi = int(self.bin_lmins[b]), int(self.bin_lmaxs[b])
                for ell in range(lo, min(hi, L) + 1):
                    W[s_idx * self.nbins + b, ell] = self.shape_weights[ell] * sm[ell]
        return W

    def param_spectrum(self, p: int) -> SpectrumSpec:
        return self.spectra[p // self.nbins]

    def pointings(self) -> list:
        return [f.vectors for f in self.fields]

    def labels(self) -> list:
        return [s.label for s in self.spectra]

    def bandpower_slices(self) -> dict:
        nb = self.nbins
        return {s.label: slice(k * nb, (k + 1) * nb) for k, s in enumerate(self.spectra)}


def _bins(params: dict, lmin: int, lmax: int):
    lmins = params.get("bin_lmins")
    lmaxs = params.get("bin_lmaxs")
    if lmins is not None and lmaxs is not None:
        lmins = np.asarray(lmins, dtype=int)
        lmaxs = np.asarray(lmaxs, dtype=int)
        floor = 2
    else:
        delta = int(params.get("delta_ell", 1))
        nb = (lmax - lmin + 1) // delta
        lmins = lmin + np.arange(nb) * delta
        lmaxs = lmins + delta - 1
        floor = lmin
    keep = (lmaxs >= floor) & (lmins >= floor)
    lmins, lmaxs = lmins[keep], lmaxs[keep]
    if lmins.size == 0:
        raise ValueError(f"No valid bins (all bins below lmin_floor={floor})")
    if np.any(lmins > lmaxs) or np.any(lmins[1:] <= lmaxs[:-1]):
        raise ValueError("bins must be sorted, non-overlapping, with lmin <= lmax")
    if lmins[0] != lmin:
        raise ValueError(f"bins.lmin={lmins[0]} != params.lmin={lmin}")
    if lmaxs[-1] > lmax:
        raise ValueError(f"bins.lmax={lmaxs[-1]} > params.lmax={lmax}")
    return lmins, lmaxs


def _shape_weights(convention: str, lmax_sig: int, lmin: int) -> np.ndarray:
    key = str(convention).strip().lower()
    if key == "cl":
        return np.ones(lmax_sig + 1)
    if key != "dl":
        raise ValueError(f"Unknown shape convention '{convention}'. Must be 'Cl' or 'Dl'.")
    if lmin == 0:
        raise ValueError("The flat-D_ell shape is undefined at the monopole")
    ell = np.arange(lmax_sig + 1, dtype=np.float64)
    w = np.zeros(lmax_sig + 1)
    w[1:] = 2 * math.pi / (ell[1:] * (ell[1:] + 1))
    return w


def build_layout(params: dict, mask: np.ndarray, beam: np.ndarray | None) -> Layout:
    """Layout of one problem from the reference-style params and seams."""
    nside = int(params["nside"])
    spins = list(params.get("spins", [0, 2]))
    labels = list(params.get("labels", ["T", "E", "B"]))
    ordering = params.get("ordering", "RING")
    lmin = int(params.get("lmin", 2))
    lmax = int(params.get("lmax", 64))
    lmax_sig = params.get("lmax_signal")
    lmax_sig = 4 * nside if lmax_sig is None else int(lmax_sig)

    mask = np.asarray(mask, dtype=np.float64)
    if mask.ndim == 1:
        mask = mask[:, None]
    npix = healpix.nside2npix(nside)
    ncomp = sum(1 if s == 0 else 2 for s in spins)
    if mask.shape[0] != npix:
        raise ValueError(f"mask has npix={mask.shape[0]}, expected {npix} for nside={nside}")
    if mask.shape[1] != ncomp:
        raise ValueError(f"mask has {mask.shape[1]} column(s), expected nfields={ncomp}")

    fields = []
    col = 0
    lab = 0
    off = 0
    for sp in spins:
        if sp == 0:
            flabels = [labels[lab]]
            m = mask[:, col]
            col += 1
            lab += 1
        elif sp == 2:
            a = mask[:, col] > healpix.ACTIVE_THRESHOLD
            b = mask[:, col + 1] > healpix.ACTIVE_THRESHOLD
            if not np.array_equal(a, b):
                raise ValueError(
                    f"mask columns {col} and {col + 1} differ, but they are the two "
                    "components of one spin-2 field and must share a single pixel set")
            flabels = [labels[lab], labels[lab + 1]]
            m = mask[:, col + 1]
            col += 2
            lab += 2
        else:
            raise ValueError(f"unsupported spin {sp}")
        pix = healpix.active_pixels(m)
        vec = healpix.pointings(nside, pix, ordering)
        fs = FieldSpec(spin=sp, labels=flabels, pixels=pix, vectors=vec, offset=off)
        off += fs.nrows
        fields.append(fs)

    spectra = []
    for i, f in enumerate(fields):
        if f.spin == 0:
            u = f.labels[0].upper()
            spectra.append(SpectrumSpec(u + u, i, i, KIND_00_AUTO, 0, (f.labels[0], f.labels[0])))
        else:
            e, b = (x.upper() for x in f.labels)
            spectra.append(SpectrumSpec(e + e, i, i, KIND_22_AUTO, 0, (f.labels[0], f.labels[0])))
            spectra.append(SpectrumSpec(b + b, i, i, KIND_22_AUTO, 1, (f.labels[1], f.labels[1])))
            spectra.append(SpectrumSpec(e + b, i, i, KIND_22_AUTO, 2, (f.labels[0], f.labels[1])))
    for i in range(len(fields)):
        for j in range(i + 1, len(fields)):
            fi, fj = fields[i], fields[j]
            if fi.spin == 0 and fj.spin == 0:
                spectra.append(SpectrumSpec((fi.labels[0] + fj.labels[0]).upper(), i, j,
                                            KIND_00_CROSS, 0, (fi.labels[0], fj.labels[0])))
            elif fi.spin == 0 and fj.spin == 2:
                t = fi.labels[0]
                for mode, pl in enumerate(fj.labels):
                    spectra.append(SpectrumSpec((t + pl).upper(), i, j, KIND_02, mode, (t, pl)))
            else:
                raise NotImplementedError(
                    "only spin-0 x spin-0 and spin-0 (first) x spin-2 cross pairs are supported")

    blocks = []
    for i, f in enumerate(fields):
        idx = [k for k, s in enumerate(spectra) if s.fi == i and s.fj == i]
        blocks.append(BlockSpec(KIND_00_AUTO if f.spin == 0 else KIND_22_AUTO, i, i, idx))
    for i in range(len(fields)):
        for j in range(i + 1, len(fields)):
            idx = [k for k, s in enumerate(spectra) if s.fi == i and s.fj == j]
            kind = KIND_00_CROSS if fields[j].spin == 0 else KIND_02
            blocks.append(BlockSpec(kind, i, j, idx))

    beams = {}
    if beam is not None:
        beam = np.asarray(beam, dtype=np.float64)
        if beam.shape[0] < 3:
            raise ValueError(f"injected beam must have at least 3 rows (T, E, B), got {beam.shape[0]}")
        if beam.shape[1] < lmax_sig + 1:
            raise ValueError(f"beam is too short: expected at least {lmax_sig + 1} multipoles")
        for k, r in _BEAM_ROW.items():
            beams[k] = beam[r, : lmax_sig + 1].copy()
    else:
        for k in _BEAM_ROW:
            beams[k] = np.ones(lmax_sig + 1)

    lmins, lmaxs = _bins(params, lmin, lmax)
    conv = params.get("output_convention", "Cl")
    return Layout(
        nside=nside, ordering=ordering, fields=fields, spectra=spectra, blocks=blocks,
        lmin=lmin, lmax=lmax, lmax_signal=lmax_sig, bin_lmins=lmins, bin_lmaxs=lmaxs,
        shape_weights=_shape_weights(conv, lmax_sig, lmin), beams=beams,
        remove_nb=bool(params.get("remove_nb", True)), nsims=int(params.get("nsims") or 1),
        output_convention=conv,
    )
