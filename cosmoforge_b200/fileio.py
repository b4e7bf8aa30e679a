"""File inputs of the reference's configuration (masks, noise covariances, C_l, beams, maps).

Host-side adapters with the semantics of the reference's readers, used when
an input is not injected through the in-memory seams:

* masks: HEALPix FITS maps, one column per component, RING order
  (``cosmocore/in_out.py:174-207`` ``read_mask``);
* noise covariance: raw FP64 ``.bin``, full sky (``npix*ncomp``)^2 reduced to
  the active pixels, or already reduced with ``load_reduced``
  (``cosmocore/in_out.py:59-145``);
* C_l: text table with a ``#`` header naming the columns, an optional ``ell``
  column, ``Dl`` converted to ``Cl`` (``cosmocore/in_out.py:305-378``);
* beams: ``smoothing_type`` ``file`` (FITS table, columns T, E, B),
  ``gaussian`` (``fwhmarcmin``) or ``none`` (``cosmocore/beam.py:128-215``);
* maps: ``.npy`` (n_fields, n_pix, n_sims), multi-simulation FITS (``SIM_XXX``
  image HDUs with a ``FIELDS`` header) or a simple HEALPix table
  (``cosmocore/in_out.py:439-600``).

FITS is parsed directly (binary tables of ``D`` / ``E`` / ``J`` / ``K``
columns, FP64 / FP32 images); no astropy or healpy is needed.
"""

from __future__ import annotations

import math

import numpy as np

_BLOCK = 2880
_TFORM = {"D": ">f8", "E": ">f4", "J": ">i4", "K": ">i8", "I": ">i2"}
_BITPIX = {-64: ">f8", -32: ">f4", 32: ">i4", 64: ">i8", 16: ">i2"}


def _header(buf: bytes, off: int):
    cards = {}
    while True:
        if off + _BLOCK > len(buf):
            raise ValueError("truncated FITS header")
        block = buf[off:off + _BLOCK].decode("ascii", "replace")
        off += _BLOCK
        for i in range(0, _BLOCK, 80):
            card = block[i:i + 80]
            key = card[:8].strip()
            if key == "END":
                return cards, off
            if card[8:10] == "= ":
                val = card[10:]
                if val.lstrip().startswith("'"):
                    v = val.lstrip()[1:]
                    val = v[:v.find("'")] if "'" in v else v
                else:
                    val = val.split("/")[0]
                cards[key] = val.strip()


def _data_size(hdr) -> int:
    naxis = int(hdr.get("NAXIS", 0))
    if naxis == 0:
        return 0
    size = abs(int(hdr["BITPIX"])) // 8
    for k in range(1, naxis + 1):
        size *= int(hdr[f"NAXIS{k}"])
    pcount = int(hdr.get("PCOUNT", 0))
    return size + pcount


def fits_hdus(path: str):
    """[(header dict, data bytes offset)] of every HDU in the file."""
    buf = open(path, "rb").read()
    out, off = [], 0
    while off < len(buf):
        if not buf[off:off + 80].strip(b" \x00"):
            break
        hdr, off = _header(buf, off)
        out.append((hdr, off))
        off += (_data_size(hdr) + _BLOCK - 1) // _BLOCK * _BLOCK
    return buf, out


def read_bintable(path: str) -> dict:
    """{column name: FP64 array} of the first binary table (vector cells flattened)."""
    buf, hdus = fits_hdus(path)
    for hdr, off in hdus:
        if hdr.get("XTENSION") != "BINTABLE":
            continue
        fields, names = [], []
        for k in range(1, int(hdr["TFIELDS"]) + 1):
            form = hdr[f"TFORM{k}"].strip()
            code = form[-1]
            if code not in _TFORM:
                raise ValueError(f"{path}: unsupported column format {form}")
            rep = int(form[:-1]) if len(form) > 1 else 1
            name = hdr.get(f"TTYPE{k}", f"COL{k}").strip()
            names.append(name)
            fields.append((name, _TFORM[code], (rep,)) if rep > 1 else (name, _TFORM[code]))
        dt = np.dtype(fields)
        if dt.itemsize != int(hdr["NAXIS1"]):
            raise ValueError(f"{path}: row length {hdr['NAXIS1']} != {dt.itemsize}")
        table = np.frombuffer(buf, dtype=dt, count=int(hdr["NAXIS2"]), offset=off)
        cols = {n: np.asarray(table[n], dtype=np.float64).reshape(-1) for n in names}
        cols["__header__"] = hdr
        return cols
    raise ValueError(f"{path}: no binary table")


def read_image_hdus(path: str) -> dict:
    """{EXTNAME: (array, header)} of every image extension."""
    buf, hdus = fits_hdus(path)
    out = {}
    for i, (hdr, off) in enumerate(hdus):
        if i == 0 and int(hdr.get("NAXIS", 0)) == 0:
            continue
        if i > 0 and hdr.get("XTENSION") != "IMAGE":
            continue
        naxis = int(hdr["NAXIS"])
        shape = tuple(int(hdr[f"NAXIS{k}"]) for k in range(naxis, 0, -1))
        dt = np.dtype(_BITPIX[int(hdr["BITPIX"])])
        arr = np.frombuffer(buf, dtype=dt, count=int(np.prod(shape)), offset=off).reshape(shape)
        out[hdr.get("EXTNAME", f"HDU{i}")] = (np.asarray(arr, dtype=np.float64), hdr)
    return out


def _healpix_columns(path: str):
    cols = read_bintable(path)
    hdr = cols.pop("__header__")
    ordering = str(hdr.get("ORDERING", "RING")).upper()
    return [cols[k] for k in cols], ordering


def read_mask(path: str, ncols: int, ordering: str = "RING") -> np.ndarray:
    """(npix, ncols) mask from the first ncols map columns of a HEALPix FITS file."""
    cols, file_ordering = _healpix_columns(path)
    if file_ordering != ordering.upper():
        raise NotImplementedError(f"{path}: mask stored {file_ordering}, analysis ordering {ordering}")
    if len(cols) < ncols:
        raise ValueError(f"{path}: {len(cols)} map column(s), need {ncols}")
    return np.stack(cols[:ncols], axis=1).astype(np.float64)


def active_indices(layout) -> np.ndarray:
    """Flat full-sky indices (component-major) of the reduced vector's rows."""
    npix = 12 * layout.nside ** 2
    idx, comp = [], 0
    for f in layout.fields:
        for _ in range(1 if f.spin == 0 else 2):
            idx.append(np.asarray(f.pixels, dtype=np.int64) + comp * npix)
            comp += 1
    return np.concatenate(idx)


def read_covmat(path: str, npix: int, ncomp: int, active: np.ndarray) -> np.ndarray:
    """Reduced covariance from a full-sky FP64 matrix of order npix*ncomp."""
    full = np.fromfile(path.strip(), dtype=np.float64)
    nfull = npix * ncomp
    if full.size != nfull * nfull:
        raise ValueError(f"{path}: {full.size} values, expected {nfull}^2 for npix={npix}, components={ncomp}")
    full = full.reshape(nfull, nfull)
    a = np.asarray(active, dtype=np.intp)
    return np.ascontiguousarray(full[np.ix_(a, a)])


def read_covmat_reduced(path: str, n: int) -> np.ndarray:
    data = np.fromfile(path.strip(), dtype=np.float64)
    if data.size != n * n:
        raise ValueError(f"{path}: {data.size} values, expected {n * n} for a reduced ({n}, {n}) matrix")
    return data.reshape(n, n)


def read_cls(path: str, lmax: int, input_convention: str = "Cl") -> dict:
    """{label: C_l} (length lmax + 1) from a '#'-headed text table."""
    with open(path.strip()) as f:
        header = f.readline()
        if not header.lstrip().startswith("#"):
            raise ValueError("First line must be a header starting with '#'")
        labels = header.strip().lstrip("#").split()
        arr = np.atleast_2d(np.loadtxt(f, dtype=np.float64))
    ell_col = next((i for i, lab in enumerate(labels) if lab.lower() == "ell"), None)
    out = {}
    if ell_col is not None:
        ells = arr[:, ell_col].astype(int)
        keep = (ells >= 0) & (ells <= lmax)
    else:
        n_fit = max(0, min(arr.shape[0], lmax - 1))
    for i, lab in enumerate(labels):
        if i == ell_col:
            continue
        v = np.zeros(lmax + 1)
        if ell_col is not None:
            v[ells[keep]] = arr[keep, i]
        elif n_fit > 0:
            v[2:2 + n_fit] = arr[:n_fit, i]
        out[lab] = v
    conv = str(input_convention).lower()
    if conv in ("dl", "d_l"):
        ell = np.arange(lmax + 1, dtype=np.float64)
        fac = np.zeros(lmax + 1)
        fac[1:] = 2.0 * math.pi / (ell[1:] * (ell[1:] + 1.0))
        out = {k: v * fac for k, v in out.items()}
    return out


def gaussian_beam_pol(fwhm_arcmin: float, lmax: int) -> np.ndarray:
    """(3, lmax + 1) Gaussian window: T exp(-l(l+1) s^2 / 2), E and B with the spin-2 factor exp(2 s^2)."""
    s2 = (math.radians(fwhm_arcmin / 60.0) / math.sqrt(8.0 * math.log(2.0))) ** 2
    ell = np.arange(lmax + 1, dtype=np.float64)
    g = np.exp(-0.5 * ell * (ell + 1.0) * s2)
    return np.stack([g, g * math.exp(2.0 * s2), g * math.exp(2.0 * s2)])


def read_beam(params, lmax: int) -> np.ndarray:
    """(3, lmax + 1) beam per ``smoothing_type`` (file / gaussian / none)."""
    kind = str(getattr(params, "smoothing_type", "file")).lower()
    if kind == "none":
        return np.ones((3, lmax + 1))
    if kind == "gaussian":
        return gaussian_beam_pol(float(getattr(params, "fwhmarcmin", 440.0)), lmax)
    if kind == "file":
        cols = read_bintable(str(params.beam_file).strip())
        cols.pop("__header__")
        cols = list(cols.values())
        if len(cols) < 3:
            raise ValueError(f"Beam file must have at least 3 columns (T, E, B), got {len(cols)}")
        return np.stack([c[:lmax + 1] for c in cols[:3]])
    raise NotImplementedError(f"smoothing_type={kind!r} is not supported by the file adapter")


def _field_index(hdr, label: str) -> int:
    fields = [s.strip() for s in str(hdr.get("FIELDS", "")).replace(",", " ").split()]
    if label in fields:
        return fields.index(label)
    default = {"T": 0, "Q": 1, "U": 2, "E": 1, "B": 2}
    if label in default:
        return default[label]
    raise ValueError(f"field {label!r} not found in FIELDS={fields}")


def read_maps(path: str, pixact: list, labels: list, nsims: int) -> np.ndarray:
    """(n_active_total, nsims) maps: per component label, its active pixels."""
    n = sum(len(p) for p in pixact)
    out = np.empty((n, nsims))
    if len(labels) != len(pixact):
        raise ValueError(f"{len(labels)} field label(s) for {len(pixact)} component(s)")
    if path.endswith(".npy"):
        data = np.load(path)
        if data.ndim != 3 or data.shape[0] < len(pixact) or data.shape[2] < nsims:
            raise ValueError(f"{path}: expected (n_fields, n_pix, n_sims), got {data.shape}")
        r = 0
        for k, p in enumerate(pixact):
            out[r:r + len(p)] = data[k][np.asarray(p, dtype=np.intp), :nsims]
            r += len(p)
        return out
    images = read_image_hdus(path)
    if "SIM_000" in images:
        hdr0 = images["SIM_000"][1]
        fidx = [_field_index(hdr0, lab) for lab in labels]
        for s in range(nsims):
            data = images[f"SIM_{s:03d}"][0]
            r = 0
            for k, p in enumerate(pixact):
                out[r:r + len(p), s] = data[fidx[k]][np.asarray(p, dtype=np.intp)]
                r += len(p)
        return out
    if nsims != 1:
        raise ValueError(f"Simple HEALPix format only supports nsims=1, got nsims={nsims}")
    cols, _ = _healpix_columns(path)
    default = {"T": 0, "Q": 1, "U": 2, "E": 1, "B": 2}
    r = 0
    for lab, p in zip(labels, pixact):
        out[r:r + len(p), 0] = cols[default[lab]][np.asarray(p, dtype=np.intp)]
        r += len(p)
    return out
