"""Minimal stand-in for the parts of ``healpy`` the reference imports.

Test infrastructure only: it lets the reference package import and run in a
container without healpy, so that golden vectors can be generated from it.

Geometry follows the closed-form HEALPix pixelisation of Gorski et al. 2005
(ApJ 622, 759), section 4: RING pixel -> (z, phi) by polar-cap / equatorial
ring formulas, with theta taken from atan2(sin theta, z) near the poles
(|z| > 0.99) and arccos(z) elsewhere, which is how HEALPix C++ evaluates it.
NESTED indices are converted to RING through the face / (x, y) bit
de-interleave of the same paper.
"""

from __future__ import annotations

import math

import numpy as np

UNSEEN = -1.6375e30
__version__ = "0.0-standin"


def nside2npix(nside):
    return 12 * int(nside) * int(nside)


def npix2nside(npix):
    nside = int(round(math.sqrt(int(npix) / 12.0)))
    if 12 * nside * nside != int(npix):
        raise ValueError(f"{npix} is not a valid HEALPix npix")
    return nside


def nside2resol(nside, arcmin=False):
    resol = math.sqrt(4.0 * math.pi / nside2npix(nside))
    return resol * 180.0 * 60.0 / math.pi if arcmin else resol


def mask_bad(m, badval=UNSEEN, rtol=1e-5, atol=1e-8):
    m = np.asarray(m)
    return np.abs(m - badval) <= atol + rtol * abs(badval)


def _isqrt(v):
    r = int(math.isqrt(int(v)))
    return r


def _ring_loc(nside, pix):
    """Return (z, phi, sth or None) for one RING pixel index."""
    npix = 12 * nside * nside
    ncap = 2 * nside * (nside - 1)
    fact2 = 4.0 / npix
    fact1 = (nside << 1) * fact2
    if pix < ncap:
        iring = (1 + _isqrt(1 + 2 * pix)) >> 1
        iphi = (pix + 1) - 2 * iring * (iring - 1)
        tmp = (iring * iring) * fact2
        z = 1.0 - tmp
        sth = math.sqrt(tmp * (2.0 - tmp)) if z > 0.99 else None
        phi = (iphi - 0.5) * (0.5 * math.pi) / iring
    elif pix < npix - ncap:
        nl4 = 4 * nside
        ip = pix - ncap
        tmp = ip // nl4
        iring = tmp + nside
        iphi = ip - nl4 * tmp + 1
        fodd = 1.0 if ((iring + nside) & 1) else 0.5
        z = (2 * nside - iring) * fact1
        sth = None
        phi = (iphi - fodd) * math.pi * 0.75 * fact1
    else:
        ip = npix - pix
        iring = (1 + _isqrt(2 * ip - 1)) >> 1
        iphi = 4 * iring + 1 - (ip - 2 * iring * (iring - 1))
        tmp = (iring * iring) * fact2
        z = tmp - 1.0
        sth = math.sqrt(tmp * (2.0 - tmp)) if z < -0.99 else None
        phi = (iphi - 0.5) * (0.5 * math.pi) / iring
    return z, phi, sth


_JRLL = (2, 2, 2, 2, 3, 3, 3, 3, 4, 4, 4, 4)
_JPLL = (1, 3, 5, 7, 0, 2, 4, 6, 1, 3, 5, 7)


def _compact_bits(v):
    out = 0
    bit = 0
    while v:
        out |= (v & 1) << bit
        v >>= 2
        bit += 1
    return out


def nest2ring(nside, ipnest):
    """Convert one NESTED index to RING (face / x-y de-interleave)."""
    scalar = np.isscalar(ipnest)
    arr = np.atleast_1d(np.asarray(ipnest, dtype=np.int64))
    out = np.empty_like(arr)
    npface = nside * nside
    nl4 = 4 * nside
    npix = 12 * npface
    ncap = 2 * nside * (nside - 1)
    for k, p in enumerate(arr.tolist()):
        face = p // npface
        ipf = p % npface
        ix = _compact_bits(ipf)
        iy = _compact_bits(ipf >> 1)
        jr = _JRLL[face] * nside - ix - iy - 1
        if jr < nside:
            nr = jr
            kshift = 0
            startpix = 2 * nr * (nr - 1)
        elif jr > 3 * nside:
            nr = nl4 - jr
            kshift = 0
            startpix = npix - 2 * (nr + 1) * nr
        else:
            nr = nside
            kshift = (jr - nside) & 1
            startpix = ncap + (jr - nside) * nl4
        jp = (_JPLL[face] * nr + ix - iy + 1 + kshift) // 2
        if jp > nl4:
            jp -= nl4
        if jp < 1:
            jp += nl4
        out[k] = startpix + jp - 1
    return int(out[0]) if scalar else out


def pix2ang(nside, ipix, nest=False, lonlat=False):
    nside = int(nside)
    scalar = np.isscalar(ipix)
    pix = np.atleast_1d(np.asarray(ipix, dtype=np.int64))
    if nest:
        pix = np.atleast_1d(nest2ring(nside, pix))
    theta = np.empty(pix.shape, dtype=np.float64)
    phi = np.empty(pix.shape, dtype=np.float64)
    for k, p in enumerate(pix.tolist()):
        z, ph, sth = _ring_loc(nside, p)
        theta[k] = math.atan2(sth, z) if sth is not None else math.acos(z)
        phi[k] = ph
    if lonlat:
        return np.degrees(phi), 90.0 - np.degrees(theta)
    if scalar:
        return float(theta[0]), float(phi[0])
    return theta, phi


def ang2vec(theta, phi, lonlat=False):
    theta = np.asarray(theta, dtype=np.float64)
    phi = np.asarray(phi, dtype=np.float64)
    st = np.sin(theta)
    return np.stack([st * np.cos(phi), st * np.sin(phi), np.cos(theta)], axis=-1)


def pix2vec(nside, ipix, nest=False):
    theta, phi = pix2ang(nside, ipix, nest=nest)
    v = ang2vec(theta, phi)
    return v[..., 0], v[..., 1], v[..., 2]


def gauss_beam(fwhm, lmax=512, pol=False):
    """Gaussian beam window b_l = exp(-l(l+1) sigma^2 / 2), sigma = fwhm/sqrt(8 ln 2).

    With ``pol=True`` the E/B columns carry the spin-2 factor exp(2 sigma^2)
    and the TE column exp(sigma^2), as HEALPix defines them.
    """
    sigma = fwhm / math.sqrt(8.0 * math.log(2.0))
    ell = np.arange(lmax + 1, dtype=np.float64)
    g = np.exp(-0.5 * ell * (ell + 1) * sigma * sigma)
    if not pol:
        return g
    fac = np.array([1.0, math.exp(2 * sigma * sigma), math.exp(2 * sigma * sigma),
                    math.exp(sigma * sigma)])
    return g[:, None] * fac[None, :]


def read_map(*args, **kwargs):  # pragma: no cover - file paths are not used
    raise NotImplementedError("healpy stand-in: inject arrays instead of reading maps")


def read_cl(*args, **kwargs):  # pragma: no cover - file paths are not used
    raise NotImplementedError("healpy stand-in: inject the beam instead of reading it")
