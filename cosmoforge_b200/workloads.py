"""Seeded synthetic problem instances for the QML / Fisher / pixel-likelihood path.

No public dataset is involved: every input is generated here from seeds with
``numpy.random.default_rng``.  Each generator returns a :class:`SkyProblem`
holding exactly what the reference's in-memory seams take (``mask``,
``noise_cov1``, ``cls_data``, ``beam``) plus the params dict, so the same
instance can be handed to the reference classes and to this package.

Maps (``x ~ N(0, S + N)``) need the signal covariance; they are drawn by
:func:`cosmoforge_b200.qube.draw_maps` on the device, or supplied by the
caller.
"""

from __future__ import annotations

import math
from dataclasses import dataclass, field

import numpy as np

from . import healpix

SIN20 = math.sin(math.radians(20.0))
SIN30 = math.sin(math.radians(30.0))


@dataclass
class SkyProblem:
    """One pixel-space problem instance, in the reference's seam formats."""

    name: str
    params: dict
    mask: np.ndarray  # (npix, n_components) float64
    cls: dict  # {label: C_l}, l-indexed, physical, length >= lmax_signal + 1
    beam: np.ndarray  # (3, lmax_signal + 1): T, E, B windows
    noise: np.ndarray | None  # (n, n) reduced noise covariance
    noise_diag: np.ndarray | None = None  # set when N is diagonal
    extra: dict = field(default_factory=dict)

    @property
    def n_active(self) -> int:
        return int((self.mask > healpix.ACTIVE_THRESHOLD).sum())


def fiducial_tt(lmax: int) -> np.ndarray:
    """C_l^TT = 2 pi 1000 / (l (l + 1)) muK^2 for l >= 2, zero below."""
    cl = np.zeros(lmax + 1)
    ell = np.arange(2, lmax + 1, dtype=np.float64)
    cl[2:] = 2.0 * math.pi * 1000.0 / (ell * (ell + 1.0))
    return cl


def reion_bump(lmax: int, centre: float = 5.0, width: float = 3.0) -> np.ndarray:
    ell = np.arange(lmax + 1, dtype=np.float64)
    g = np.exp(-((ell - centre) ** 2) / (2.0 * width * width))
    g[:2] = 0.0
    return g


def tqu_shapes(lmax: int) -> dict:
    """TT, EE, BB, TE shapes with TB = EB = 0.

    EE = 0.04 TT + 0.1 muK^2 exp(-(l-5)^2/18); BB = 0.02 EE;
    TE = 0.3 sqrt(TT EE).
    """
    tt = fiducial_tt(lmax)
    ee = 0.04 * tt + 0.1 * reion_bump(lmax)
    ee[:2] = 0.0
    bb = 0.02 * ee
    te = 0.3 * np.sqrt(tt * ee)
    z = np.zeros(lmax + 1)
    return {"TT": tt, "EE": ee, "BB": bb, "TE": te, "TB": z.copy(), "EB": z.copy()}


def gaussian_beam(fwhm_deg: float, lmax: int) -> np.ndarray:
    sigma = math.radians(fwhm_deg) / math.sqrt(8.0 * math.log(2.0))
    ell = np.arange(lmax + 1, dtype=np.float64)
    return np.exp(-0.5 * ell * (ell + 1.0) * sigma * sigma)


def z_cut_mask(nside: int, zcut: float) -> np.ndarray:
    z = healpix.ring_z(nside)
    return (np.abs(z) > zcut).astype(np.float64)


def _params(nside, spins, labels, lmin, lmax, lmax_signal, nsims, **kw) -> dict:
    p = dict(
        nside=nside,
        spins=list(spins),
        labels=list(labels),
        lmin=lmin,
        lmax=lmax,
        lmax_signal=lmax_signal,
        delta_ell=1,
        ordering="RING",
        nsims=nsims,
        remove_nb=True,
        input_convention="Cl",
        output_convention="Cl",
        smoothing_type="file",
        apply_pixwin=False,
        do_cross=False,
        feedback=0,
    )
    p.update(kw)
    return p


def config0(nsims: int = 1) -> SkyProblem:
    """Plain FP64 spin-0 TT: nside 8, |z| > sin 20 deg (480 px), l = 2..24.

    Beam: Gaussian FWHM 9 deg times the nside-8 pixel window (sub-pixel
    average).  Noise: white, sigma = 2 muK.  lmax_signal = 4 nside = 32.
    """
    nside, L = 8, 32
    mask = z_cut_mask(nside, SIN20)[:, None]
    n = int(mask.sum())
    b = gaussian_beam(9.0, L) * healpix.pixel_window(nside, L)
    beam = np.stack([b, b, b])
    cls = {"TT": fiducial_tt(L)}
    diag = np.full(n, 4.0)
    return SkyProblem(
        name="config0_tt_nside8",
        params=_params(nside, [0], ["T"], 2, 24, L, nsims),
        mask=mask,
        cls=cls,
        beam=beam,
        noise=np.diag(diag),
        noise_diag=diag,
    )


def hit_pattern_variance(nside: int, pixels: np.ndarray) -> np.ndarray:
    """sigma_T^2 = 1 + 3 cos^2(pi z / 2): 4 muK^2 at the equator, 1 at the poles."""
    z = healpix.ring_z(nside)[pixels]
    return 1.0 + 3.0 * np.cos(0.5 * math.pi * z) ** 2


def config1(seed: int = 0, nside: int = 16, lmax: int = 47, lmax_signal: int = 64,
            n_lowrank: int = 32, nsims: int = 1, dense_noise: bool = True) -> SkyProblem:
    """TQU precision-sweep problem: nside 16, |z| > sin 20 deg in T and P.

    1984 px per field, n = 5952; l = 2..47 for the six spectra TT, EE, BB,
    EB, TE, TB (EB = TB = 0), lmax_signal = 64.  Beam: Gaussian 4 deg in T,
    E and B.  Noise: N = D^1/2 (I + U U^T) D^1/2 with sigma_T^2 from
    :func:`hit_pattern_variance`, sigma_Q^2 = sigma_U^2 = 2 sigma_T^2 and
    U (n x 32) ~ N(0, 0.1^2) from ``seed``.
    """
    mask1 = z_cut_mask(nside, SIN20)
    mask = np.stack([mask1, mask1, mask1], axis=1)
    pix = healpix.active_pixels(mask1)
    var_t = hit_pattern_variance(nside, pix)
    d = np.concatenate([var_t, 2.0 * var_t, 2.0 * var_t])
    n = d.shape[0]
    rng = np.random.default_rng(seed)
    U = rng.normal(0.0, 0.1, size=(n, n_lowrank))
    sd = np.sqrt(d)
    W = sd[:, None] * U
    noise = None
    if dense_noise:
        noise = W @ W.T
        noise[np.diag_indices(n)] += d
    b = gaussian_beam(4.0, lmax_signal)
    beam = np.stack([b, b, b])
    return SkyProblem(
        name=f"config1_tqu_nside{nside}",
        params=_params(nside, [0, 2], ["T", "E", "B"], 2, lmax, lmax_signal, nsims),
        mask=mask,
        cls=tqu_shapes(lmax_signal),
        beam=beam,
        noise=noise,
        extra={"noise_d": d, "noise_W": W},
    )


# --- config 3: five-parameter TQU pixel likelihood --------------------------

THETA_NAMES = ("A", "n", "h", "r", "s")
THETA_LO = np.array([0.8, -0.1, 0.0, 0.0, 0.9])
THETA_HI = np.array([1.2, 0.1, 0.3, 0.1, 1.1])
THETA_CENTRE = 0.5 * (THETA_LO + THETA_HI)
PIVOT_ELL = 10.0


def model_cls(theta, lmax: int) -> dict:
    """C_l(theta) of the five-parameter model (A, n, h, r, s).

    t_l = A (l / 10)^n scales the TT / EE / TE shapes of :func:`tqu_shapes`;
    h adds h exp(-(l-5)^2/18) to EE; BB = r EE; TB = EB = 0.  s scales the
    noise and does not enter the spectra.
    """
    A, n_tilt, h, r, _ = (float(v) for v in theta)
    sh = tqu_shapes(lmax)
    ell = np.arange(lmax + 1, dtype=np.float64)
    t = np.zeros(lmax + 1)
    t[2:] = A * (ell[2:] / PIVOT_ELL) ** n_tilt
    ee = t * sh["EE"] + h * reion_bump(lmax)
    ee[:2] = 0.0
    z = np.zeros(lmax + 1)
    return {"TT": t * sh["TT"], "EE": ee, "BB": r * ee, "TE": t * sh["TE"],
            "TB": z.copy(), "EB": z.copy()}


def config3(lmax_signal: int = 23, nsims: int = 1) -> SkyProblem:
    """nside 8 TQU likelihood: T |z| > sin 20 (480 px), Q/U |z| > sin 30 (416 px per field).

    n = 480 + 2 x 416 = 1312, l = 2..23 with lmax_signal = 23.  nside 8 has
    two rings of 32 pixels at z = +-0.5 exactly, and sin 30 deg rounds to
    0.49999999999999994 in FP64, so both pass the strict cut: 352 + 64 = 416
    pixels per field.
    Beam as config 0; white noise sigma_T^2 = 4 muK^2, sigma_Q^2 = sigma_U^2 =
    8 muK^2 (scaled by s).
    """
    nside = 8
    mt = z_cut_mask(nside, SIN20)
    mp = z_cut_mask(nside, SIN30)
    mask = np.stack([mt, mp, mp], axis=1)
    nt, npol = int(mt.sum()), int(mp.sum())
    diag = np.concatenate([np.full(nt, 4.0), np.full(2 * npol, 8.0)])
    L = lmax_signal
    b = gaussian_beam(9.0, L) * healpix.pixel_window(nside, L)
    beam = np.stack([b, b, b])
    return SkyProblem(
        name="config3_tqu_nside8",
        params=_params(nside, [0, 2], ["T", "E", "B"], 2, 23, L, nsims),
        mask=mask,
        cls=model_cls(THETA_CENTRE, L),
        beam=beam,
        noise=np.diag(diag),
        noise_diag=diag,
    )


def sobol_points(n: int, seed: int = 0) -> np.ndarray:
    """n scrambled-Sobol points in the five-parameter box."""
    from scipy.stats import qmc

    u = qmc.Sobol(d=5, scramble=True, seed=seed).random(n)
    return THETA_LO + u * (THETA_HI - THETA_LO)


def patch_problems(n_patches: int = 48, seed: int = 0, nside: int = 16,
                   lmax: int = 47, lmax_signal: int = 64):
    """Config-2 part 2: spherical caps of radius U[10, 40] deg, TT, white noise.

    Returns a list of (mask, sigma) with centres uniform on the sphere and
    sigma ~ U[1, 5] muK.
    """
    rng = np.random.default_rng(seed)
    npix = healpix.nside2npix(nside)
    vec = healpix.pointings(nside, np.arange(npix))
    out = []
    for _ in range(n_patches):
        radius = math.radians(rng.uniform(10.0, 40.0))
        c = rng.normal(size=3)
        c /= np.linalg.norm(c)
        sigma = rng.uniform(1.0, 5.0)
        m = (vec @ c > math.cos(radius)).astype(np.float64)
        out.append((m, sigma))
    return out


def config2_patches(n_patches: int = 48, seed: int = 0, nside: int = 16, lmax: int = 47,
                    lmax_signal: int = 64, delta_ell: int = 5) -> list:
    """Config-2 part 2 as problem instances: TT on each cap of :func:`patch_problems`.

    l = 2..lmax in bins of delta_ell multipoles, fiducial C_l as config 0,
    Gaussian 4 deg beam (as config 1), white noise sigma^2 per patch.  At
    nside 16 a cap of radius 10-40 deg holds about 23-360 pixels: too few to
    separate single multipoles up to l = 47 (the Fisher matrix of 46
    one-multipole bins is numerically singular on every cap), hence bins of
    5 multipoles by default.
    """
    out = []
    b = gaussian_beam(4.0, lmax_signal)
    beam = np.stack([b, b, b])
    for k, (m, sigma) in enumerate(patch_problems(n_patches, seed, nside, lmax, lmax_signal)):
        n = int(m.sum())
        diag = np.full(n, sigma * sigma)
        out.append(SkyProblem(
            name=f"config2_patch{k}",
            params=_params(nside, [0], ["T"], 2, lmax, lmax_signal, 1, delta_ell=delta_ell),
            mask=m[:, None],
            cls={"TT": fiducial_tt(lmax_signal)},
            beam=beam,
            noise=np.diag(diag),
            noise_diag=diag,
        ))
    return out
