"""HEALPix geometry needed by the pixel-space path: pixel centres and pointings.

The reference gets pixel centres from ``healpy.pix2ang`` and turns them into
unit vectors with a scalar ``sin``/``cos`` loop
(``cosmocore/signal_kernels.py:113-161``), on purpose not the vectorised
numpy trig, so that pointings are reproducible bit for bit.  This module
evaluates the same closed-form HEALPix ring formulas (Gorski et al. 2005,
ApJ 622, 759, section 4) and the same scalar loop, so the pointings fed to
the device kernels are the ones the reference itself would use.

Also provides the active-pixel selection of ``cosmocore/geometry.py:94-134``
(``mask > 0.5``) and a pixel window computed by sub-pixel averaging (the
HEALPix pixel-window data files are not shipped with this project).
"""

from __future__ import annotations

import math

import numpy as np

ACTIVE_THRESHOLD = 0.5


def nside2npix(nside: int) -> int:
    return 12 * int(nside) * int(nside)


def _ring_z_phi(nside: int, pix: int):
    """(z, phi, sin(theta) or None) of one RING pixel centre."""
    npix = 12 * nside * nside
    ncap = 2 * nside * (nside - 1)
    fact2 = 4.0 / npix
    fact1 = (nside << 1) * fact2
    if pix < ncap:
        iring = (1 + math.isqrt(1 + 2 * pix)) >> 1
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
        iring = (1 + math.isqrt(2 * ip - 1)) >> 1
        iphi = 4 * iring + 1 - (ip - 2 * iring * (iring - 1))
        tmp = (iring * iring) * fact2
        z = tmp - 1.0
        sth = math.sqrt(tmp * (2.0 - tmp)) if z < -0.99 else None
        phi = (iphi - 0.5) * (0.5 * math.pi) / iring
    return z, phi, sth


_JRLL = (2, 2, 2, 2, 3, 3, 3, 3, 4, 4, 4, 4)
_JPLL = (1, 3, 5, 7, 0, 2, 4, 6, 1, 3, 5, 7)


def _compact_bits(v: int) -> int:
    out = 0
    bit = 0
    while v:
        out |= (v & 1) << bit
        v >>= 2
        bit += 1
    return out


def nest2ring(nside: int, ipnest) -> np.ndarray:
    """NESTED -> RING index conversion (face number, x/y bit de-interleave)."""
    arr = np.atleast_1d(np.asarray(ipnest, dtype=np.int64))
    out = np.empty_like(arr)
    npface = nside * nside
    nl4 = 4 * nside
    npix = 12 * npface
    ncap = 2 * nside * (nside - 1)
    for k, p in enumerate(arr.tolist()):
        face, ipf = divmod(p, npface)
        ix = _compact_bits(ipf)
        iy = _compact_bits(ipf >> 1)
        jr = _JRLL[face] * nside - ix - iy - 1
        if jr < nside:
            nr, kshift, startpix = jr, 0, 2 * jr * (jr - 1)
        elif jr > 3 * nside:
            nr = nl4 - jr
            kshift, startpix = 0, npix - 2 * (nr + 1) * nr
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
    return out


def pix2ang(nside: int, pixels, nest: bool = False):
    """Colatitude and longitude of pixel centres (HEALPix convention)."""
    pix = np.atleast_1d(np.asarray(pixels, dtype=np.int64))
    if nest:
        pix = nest2ring(nside, pix)
    theta = np.empty(pix.shape, dtype=np.float64)
    phi = np.empty(pix.shape, dtype=np.float64)
    for k, p in enumerate(pix.tolist()):
        z, ph, sth = _ring_z_phi(int(nside), p)
        theta[k] = math.atan2(sth, z) if sth is not None else math.acos(z)
        phi[k] = ph
    return theta, phi


def unit_vectors(theta: np.ndarray, phi: np.ndarray) -> np.ndarray:
    """(n, 3) unit vectors by the scalar libm loop of the reference."""
    out = np.empty((theta.shape[0], 3), dtype=np.float64)
    for i in range(theta.shape[0]):
        t = float(theta[i])
        p = float(phi[i])
        x = math.sin(t) * math.cos(p)
        y = math.sin(t) * math.sin(p)
        z = math.cos(t)
        norm = math.sqrt(x**2 + y**2 + z**2)
        out[i, 0] = x / norm
        out[i, 1] = y / norm
        out[i, 2] = z / norm
    return out


def pointings(nside: int, pixels, ordering: str = "RING") -> np.ndarray:
    theta, phi = pix2ang(nside, pixels, nest=(ordering == "NESTED"))
    return unit_vectors(theta, phi)


def active_pixels(mask_column: np.ndarray) -> np.ndarray:
    """Indices of active pixels of one mask column (``mask > 0.5``)."""
    return np.flatnonzero(np.asarray(mask_column, dtype=np.float64) > ACTIVE_THRESHOLD)


def ring_z(nside: int) -> np.ndarray:
    """z = cos(theta) of every RING pixel centre."""
    npix = nside2npix(nside)
    return np.array([_ring_z_phi(nside, p)[0] for p in range(npix)])


def pixel_window(nside: int, lmax: int, sub_level: int = 3) -> np.ndarray:
    """Temperature pixel window w_l by averaging over sub-pixels.

    w_l^2 = (1/N_pix) sum_p (1/N_c^2) sum_{c,c' in p} P_l(r_c . r_c'), where
    the N_c = 4^sub_level children of pixel p are the NESTED pixels of
    resolution nside * 2^sub_level that tile it.  This is the beam of a pixel
    average, azimuthally averaged over the sky.
    """
    nside_hi = nside << sub_level
    nc = 4**sub_level
    npix = nside2npix(nside)
    children = np.arange(npix * nc, dtype=np.int64)
    vec = pointings(nside_hi, nest2ring(nside_hi, children)).reshape(npix, nc, 3)
    x = np.einsum("pid,pjd->pij", vec, vec).reshape(-1)
    x = np.clip(x, -1.0, 1.0)
    p_prev = np.ones_like(x)
    p_cur = x.copy()
    w2 = np.zeros(lmax + 1)
    w2[0] = 1.0
    if lmax >= 1:
        w2[1] = p_cur.mean()
    for ell in range(2, lmax + 1):
        p_next = ((2 * ell - 1) * x * p_cur - (ell - 1) * p_prev) / ell
        p_prev, p_cur = p_cur, p_next
        w2[ell] = p_cur.mean()
    return np.sqrt(np.clip(w2, 0.0, None))
