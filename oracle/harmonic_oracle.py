"""CPU oracle for the harmonic-basis path (test infrastructure only).

NumPy restatement of the real harmonic operator V that the reference's
harmonic basis builds (cosmocore/basis/harmonic_basis.py:20-180): spin-0 rows
from fully normalised associated Legendre functions with the Condon-Shortley
phase (cosmocore/basics/legendre.py:153-210), spin-2 E/B rows over [Q | U]
columns from the Wigner small-d functions d^l_{m,+-2}
(cosmocore/basics/wigner.py:12-120), combined as
D+ = d_{m,-2} + d_{m,2}, D- = d_{m,-2} - d_{m,2} with the reference's
cos/sin row pattern.  The small-d values come from the explicit
factorial sum at the first degree and the standard three-term recurrence in
the degree above it (both published formulas, not the reference's code).

Rows are ordered component-major, then by multipole, then m = 0 followed by
the (cos m, sin m) pairs, so the 2l + 1 rows of a multipole are contiguous
(the reference orders by m first; the order does not enter any result).  A
component is a spin-0 field (T) or the E or B part of a spin-2 field.

The addition theorem makes dC/dC_l = t_l V_(u,l)^T V_(v,l) (plus its
transpose for cross spectra), which the tests check against the pixel-space
derivative of the oracle, entry by entry.  Only the tests import this module.
"""

from __future__ import annotations

from math import lgamma

import numpy as np


def components(L):
    """[(field index, 'T' | 'E' | 'B')] in row order."""
    out = []
    for fi, f in enumerate(L.fields):
        if f.spin == 0:
            out.append((fi, "T"))
        else:
            out.extend([(fi, "E"), (fi, "B")])
    return out


def spectrum_components(L, s):
    """(u, v) component indices of spectrum s (u == v for auto spectra)."""
    comps = components(L)
    sp = L.spectra[s]
    fi, fj = sp.fi, sp.fj
    fs = L.fields

    def idx(f, c):
        return comps.index((f, c))

    if fs[fi].spin == 0 and fs[fj].spin == 0:
        return idx(fi, "T"), idx(fj, "T")
    if fs[fi].spin == 2 and fs[fj].spin == 2:
        a, b = {0: ("E", "E"), 1: ("B", "B"), 2: ("E", "B")}[sp.mode]
        return idx(fi, a), idx(fj, b)
    t, p = (fi, fj) if fs[fi].spin == 0 else (fj, fi)
    return idx(t, "T"), idx(p, "E" if sp.mode == 0 else "B")


def plm_normalised(x, s, lmax):
    """sqrt((2l+1)/4pi) sqrt((l-m)!/(l+m)!) P_l^m(x), Condon-Shortley phase; (lmax+1, lmax+1, npix)."""
    x = np.asarray(x, np.float64)
    s = np.asarray(s, np.float64)
    P = np.zeros((lmax + 1, lmax + 1) + x.shape)
    P[0, 0] = 1.0
    if lmax >= 1:
        P[1, 0] = x
    for ell in range(2, lmax + 1):
        P[ell, 0] = ((2 * ell - 1) * x * P[ell - 1, 0] - (ell - 1) * P[ell - 2, 0]) / ell
    for m in range(1, lmax + 1):
        P[m, m] = -s * np.sqrt((2 * m - 1) / (2 * m)) * P[m - 1, m - 1]
        if m < lmax:
            P[m + 1, m] = x * np.sqrt(2 * m + 1) * P[m, m]
        for ell in range(m + 2, lmax + 1):
            d = ell * ell - m * m
            P[ell, m] = ((2 * ell - 1) / np.sqrt(d)) * x * P[ell - 1, m] - np.sqrt(
                ((ell - 1) ** 2 - m * m) / d) * P[ell - 2, m]
    for ell in range(lmax + 1):
        P[ell] *= np.sqrt((2 * ell + 1) / (4 * np.pi))
    return P


def _d_start(j, mp, m, ch, sh):
    """d^j_{mp,m} from the explicit sum (Wigner), arrays ch = cos(b/2), sh = sin(b/2)."""
    out = np.zeros_like(ch)
    lnorm = 0.5 * (lgamma(j + mp + 1) + lgamma(j - mp + 1) + lgamma(j + m + 1) + lgamma(j - m + 1))
    for k in range(0, 2 * j + 1):
        a, b, c, d = j + m - k, k, mp - m + k, j - mp - k
        if min(a, b, c, d) < 0:
            continue
        coef = (-1.0) ** (mp - m + k) * np.exp(lnorm - lgamma(a + 1) - lgamma(b + 1) - lgamma(c + 1)
                                                - lgamma(d + 1))
        out += coef * ch ** (2 * j + m - mp - 2 * k) * sh ** (mp - m + 2 * k)
    return out


def wigner_d(lmax, m, s, cos_t):
    """d^l_{m,s}(theta) for l = 0..lmax (zero below max(|m|, |s|)); (lmax+1, npix)."""
    cos_t = np.asarray(cos_t, np.float64)
    th = np.arccos(np.clip(cos_t, -1.0, 1.0))
    ch, sh = np.cos(0.5 * th), np.sin(0.5 * th)
    out = np.zeros((lmax + 1,) + cos_t.shape)
    j0 = max(abs(m), abs(s))
    if j0 > lmax:
        return out
    out[j0] = _d_start(j0, m, s, ch, sh)
    for j in range(j0 + 1, lmax + 1):
        a = (2 * j - 1) * (j * (j - 1) * cos_t - m * s)
        b = j * np.sqrt(max(((j - 1) ** 2 - m * m) * ((j - 1) ** 2 - s * s), 0))
        c = (j - 1) * np.sqrt((j * j - m * m) * (j * j - s * s))
        prev2 = out[j - 2] if j - 2 >= 0 else 0.0
        out[j] = (a * out[j - 1] - b * prev2) / c
    return out


def mode_offsets(L, lmin, lmax):
    """Row offset of every (component, l) block and the total row count."""
    comps = components(L)
    off = {}
    r = 0
    for ci in range(len(comps)):
        for ell in range(lmin, lmax + 1):
            off[(ci, ell)] = r
            r += 2 * ell + 1
    return off, r


def harmonic_operator(L, lmin, lmax):
    """V: (n_modes, n) FP64 over the reduced pixel vector."""
    comps = components(L)
    off, nm = mode_offsets(L, lmin, lmax)
    V = np.zeros((nm, L.n))
    for ci, (fi, c) in enumerate(comps):
        f = L.fields[fi]
        v = f.vectors
        z = np.clip(v[:, 2], -1.0, 1.0)
        st = np.sqrt(np.maximum(0.0, 1.0 - z * z))
        phi = np.arctan2(v[:, 1], v[:, 0])
        cols = f.offset + np.arange(f.npix)
        if c == "T":
            P = plm_normalised(z, st, lmax)
            for ell in range(lmin, lmax + 1):
                r = off[(ci, ell)]
                V[r, cols] = P[ell, 0]
                for m in range(1, ell + 1):
                    V[r + 2 * m - 1, cols] = np.sqrt(2.0) * P[ell, m] * np.cos(m * phi)
                    V[r + 2 * m, cols] = np.sqrt(2.0) * P[ell, m] * np.sin(m * phi)
            continue
        q_cols, u_cols = cols, cols + f.npix
        is_b = c == "B"
        for m in range(0, lmax + 1):
            dp = wigner_d(lmax, m, 2, z)
            dm = wigner_d(lmax, m, -2, z)
            cm, sm = np.cos(m * phi), np.sin(m * phi)
            for ell in range(max(lmin, m, 2), lmax + 1):
                sc = np.sqrt((2 * ell + 1) / (4 * np.pi)) * 0.5
                Dp = dm[ell] + dp[ell]
                Dm = dm[ell] - dp[ell]
                r = off[(ci, ell)]
                if m == 0:
                    if is_b:
                        V[r, u_cols] = sc * Dp
                    else:
                        V[r, q_cols] = sc * Dp
                    continue
                sc2 = sc * np.sqrt(2.0)
                rc, rs = r + 2 * m - 1, r + 2 * m
                if not is_b:
                    V[rc, q_cols] = sc2 * Dp * cm
                    V[rc, u_cols] = sc2 * Dm * sm
                    V[rs, q_cols] = sc2 * Dp * sm
                    V[rs, u_cols] = -sc2 * Dm * cm
                else:
                    V[rc, q_cols] = -sc2 * Dm * sm
                    V[rc, u_cols] = sc2 * Dp * cm
                    V[rs, q_cols] = sc2 * Dm * cm
                    V[rs, u_cols] = sc2 * Dp * sm
    # the pixel-space 02 kernel (tq = -sum c_TE P^2_l ...) fixes the relative
    # sign of the spin-2 rows against the spin-0 rows: E and B rows enter with
    # the opposite overall sign of the d-function expression above
    for ci, (fi, c) in enumerate(comps):
        if c != "T":
            r0 = off[(ci, lmin)]
            V[r0: r0 + (lmax + 1) ** 2 - lmin ** 2] *= -1.0
    return V


def derivative_from_V(L, V, s, ell, lmin, lmax):
    """t = 1 derivative of spectrum s at multipole l from V (n x n)."""
    off, _ = mode_offsets(L, lmin, lmax)
    u, v = spectrum_components(L, s)
    Vu = V[off[(u, ell)]: off[(u, ell)] + 2 * ell + 1]
    Vv = V[off[(v, ell)]: off[(v, ell)] + 2 * ell + 1]
    D = Vu.T @ Vv
    return D if u == v else D + D.T


def fisher_harmonic(L, Cinv, lmin, lmax, weights=None):
    """Binned Fisher F (P x P) as 1/2 sum t t' <G_vs, G_ut> over the l blocks of
    G = V C^-1 V^T (the harmonic form of 1/2 Tr(C^-1 dC_b C^-1 dC_b'))."""
    V = harmonic_operator(L, lmin, lmax)
    G = V @ Cinv @ V.T
    off, _ = mode_offsets(L, lmin, lmax)
    nc = len(components(L))
    W = L.param_weights() if weights is None else weights
    nb, P = L.nbins, L.n_params
    pairs = []
    for s in range(L.nspectra):
        u, v = spectrum_components(L, s)
        pairs.append([(u, v)] if u == v else [(u, v), (v, u)])
    F = np.zeros((P, P))
    for l1 in range(lmin, lmax + 1):
        for l2 in range(lmin, lmax + 1):
            g = np.stack([G[off[(p, l1)]: off[(p, l1)] + 2 * l1 + 1, off[(q, l2)]: off[(q, l2)] + 2 * l2 + 1].ravel()
                          for p in range(nc) for q in range(nc)])
            K = g @ g.T  # K[(p q), (p' q')] = <G_pq, G_p'q'>
            for p1 in range(P):
                s1 = p1 // nb
                t1 = W[p1, l1]
                if t1 == 0.0:
                    continue
                for p2 in range(P):
                    s2 = p2 // nb
                    t2 = W[p2, l2]
                    if t2 == 0.0:
                        continue
                    acc = sum(K[v * nc + a, u * nc + b] for (u, v) in pairs[s1] for (a, b) in pairs[s2])
                    F[p1, p2] += 0.5 * t1 * t2 * acc
    return F


def signal_harmonic(L, cl_table, lmin, lmax, signal_pixel, fixed_table=None):
    """S as the harmonic basis assembles it (cosmocore/core.py:950-1010):
    V^T Lambda V over the inference window [lmin, lmax] plus the pixel-space
    signal of the multipoles outside it (S_fixed, from fixed_table, the
    fiducial spectra, default cl_table).  Tables: beam-smoothed
    (nspectra, lmax_signal + 1); signal_pixel(table) builds a pixel S."""
    S = signal_pixel(_outside(cl_table if fixed_table is None else fixed_table, lmin, lmax))
    V = harmonic_operator(L, lmin, lmax)
    off, _ = mode_offsets(L, lmin, lmax)
    LV = np.zeros_like(V)
    for s in range(L.nspectra):
        u, v = spectrum_components(L, s)
        for ell in range(lmin, lmax + 1):
            c = cl_table[s, ell]
            ru, rv = off[(u, ell)], off[(v, ell)]
            k = 2 * ell + 1
            LV[ru:ru + k] += c * V[rv:rv + k]
            if u != v:
                LV[rv:rv + k] += c * V[ru:ru + k]
    return S + V.T @ LV


def qml_harmonic(L, Cinv, N, maps, lmin, lmax, weights=None):
    """Raw bias b_p = 1/2 Tr(C^-1 N C^-1 dC_p) and q_p = 1/2 y^T dC_p y
    (y = C^-1 x) through Z = V C^-1: b from the (l, m)-diagonal of Z N Z^T,
    q from z = Z x."""
    V = harmonic_operator(L, lmin, lmax)
    off, _ = mode_offsets(L, lmin, lmax)
    W = L.param_weights() if weights is None else weights
    Z = V @ Cinv
    h = Z @ N @ Z.T
    z = Z @ maps
    nb, P = L.nbins, L.n_params
    bias = np.zeros(P)
    q = np.zeros((maps.shape[1], P))
    for p in range(P):
        s = p // nb
        u, v = spectrum_components(L, s)
        f = 1.0 if u == v else 2.0
        for ell in range(lmin, lmax + 1):
            t = W[p, ell]
            if t == 0.0:
                continue
            k = 2 * ell + 1
            ru, rv = off[(u, ell)], off[(v, ell)]
            bias[p] += 0.5 * f * t * np.trace(h[ru:ru + k, rv:rv + k])
            q[:, p] += 0.5 * f * t * np.sum(z[ru:ru + k] * z[rv:rv + k], axis=0)
    return bias, q


def _fisher_from_G(L, G, lmin, lmax, W):
    off, _ = mode_offsets(L, lmin, lmax)
    nc = len(components(L))
    nb, P = L.nbins, L.n_params
    pairs = []
    for s in range(L.nspectra):
        u, v = spectrum_components(L, s)
        pairs.append([(u, v)] if u == v else [(u, v), (v, u)])
    F = np.zeros((P, P))
    for l1 in range(lmin, lmax + 1):
        for l2 in range(lmin, lmax + 1):
            g = np.stack([G[off[(p, l1)]: off[(p, l1)] + 2 * l1 + 1, off[(q, l2)]: off[(q, l2)] + 2 * l2 + 1].ravel()
                          for p in range(nc) for q in range(nc)])
            K = g @ g.T
            for p1 in range(P):
                t1 = W[p1, l1]
                if t1 == 0.0:
                    continue
                for p2 in range(P):
                    t2 = W[p2, l2]
                    if t2 == 0.0:
                        continue
                    acc = sum(K[v * nc + a, u * nc + b] for (u, v) in pairs[p1 // nb] for (a, b) in pairs[p2 // nb])
                    F[p1, p2] += 0.5 * t1 * t2 * acc
    return F


def _qml_from_Z(L, Z, Nm, xm, lmin, lmax, W):
    off, _ = mode_offsets(L, lmin, lmax)
    h = Z @ Nm @ Z.T
    z = Z @ xm
    nb, P = L.nbins, L.n_params
    bias = np.zeros(P)
    q = np.zeros((xm.shape[1], P))
    for p in range(P):
        u, v = spectrum_components(L, p // nb)
        f = 1.0 if u == v else 2.0
        for ell in range(lmin, lmax + 1):
            t = W[p, ell]
            if t == 0.0:
                continue
            k = 2 * ell + 1
            ru, rv = off[(u, ell)], off[(v, ell)]
            bias[p] += 0.5 * f * t * np.trace(h[ru:ru + k, rv:rv + k])
            q[:, p] += 0.5 * f * t * np.sum(z[ru:ru + k] * z[rv:rv + k], axis=0)
    return bias, q


def keep_modes(evals, epsilon=None, mode_fraction=None):
    """Indices of the kept eigenvectors, eigenvalues sorted descending
    (cosmocore/basis/pixel.py:265-311)."""
    order = np.argsort(evals)[::-1]
    ev = evals[order]
    amax = np.max(np.abs(ev))
    if mode_fraction is not None:
        n_sig = int(np.sum(ev > 1e-10 * amax))
        keep = np.zeros(ev.size, bool)
        keep[:max(1, int(np.ceil(mode_fraction * n_sig)))] = True
    elif epsilon is not None:
        keep = np.abs(ev) > epsilon * amax
    else:
        keep = np.abs(ev) > 1e-10 * amax
    return order[keep]


def _sym_sqrt(S):
    """S^1/2 by eigendecomposition, eigenvalues clipped at 1e-30 (cosmocore/basis/pixel.py:339-348)."""
    w, Q = np.linalg.eigh(S)
    return (Q * np.sqrt(np.maximum(w, 1e-30))) @ Q.T


def compression_basis(L, V, N_eff, lmin, lmax, epsilon=None, mode_fraction=None, target="noise_weighted",
                      C_ell=None):
    """Block-diagonal U (n x dim): per field, the kept eigenvectors of the
    compression matrix of the field's rows of V (cosmocore/basis/pixel.py:
    265-557, 965-1055, 1493-1612):
    "harmonic" P_f = V_f^T V_f; "noise_weighted" P_f (N_eff^-1)_ff P_f;
    "total_covariance" P_f ((N_eff)_ff + V_f^T Lam V_f)^-1 P_f; "snr"
    S_f^1/2 (N_eff^-1)_ff S_f^1/2 with S_f = V_f^T Lam V_f, Lam = C_l at each
    row's multipole (C_ell an array or the first value of a dict).  A spin-2
    field with an (E, B) threshold pair builds the E rows' and the B rows'
    matrices apart (Lam from C_ell["EE"] / ["BB"]), keeps each by its own
    threshold, and orthogonalises the union by an economy SVD (singular
    values above 1e-10 of the largest)."""
    comps = components(L)
    nrow = (lmax + 1) ** 2 - lmin ** 2
    ell_row = np.concatenate([np.repeat(np.arange(lmin, lmax + 1), 2 * np.arange(lmin, lmax + 1) + 1)] * len(comps))
    Ninv = np.linalg.inv(N_eff)

    def lam(rows, cl):
        c = np.asarray(cl, dtype=np.float64)
        e = ell_row[rows]
        return np.where(e < c.size, c[np.minimum(e, c.size - 1)], 0.0)

    def comp_matrix(Vs, cols, cl):
        P = Vs.T @ Vs
        if target == "harmonic":
            return P
        if target == "noise_weighted":
            return P @ Ninv[np.ix_(cols, cols)] @ P
        S = Vs.T @ (Vs * cl[:, None])
        if target == "total_covariance":
            return P @ np.linalg.inv(N_eff[np.ix_(cols, cols)] + S) @ P
        Sq = _sym_sqrt(S)
        return Sq @ Ninv[np.ix_(cols, cols)] @ Sq

    def kept(M, e, m):
        ev, vec = np.linalg.eigh(0.5 * (M + M.T))
        return vec[:, keep_modes(ev, e, m)]

    def per_field(x, fi):
        return x[fi] if isinstance(x, list) else x

    blocks = []
    for fi, f in enumerate(L.fields):
        cols = np.arange(f.offset, f.offset + f.nrows)
        cis = [ci for ci, (g, _) in enumerate(comps) if g == fi]
        rows = np.concatenate([np.arange(ci * nrow, (ci + 1) * nrow) for ci in cis])
        e_f, m_f = per_field(epsilon, fi), per_field(mode_fraction, fi)
        if e_f is None and m_f is None and epsilon is None and mode_fraction is None:
            e_f = 1e-6
        if f.spin == 2 and (isinstance(e_f, tuple) or isinstance(m_f, tuple)):
            parts = []
            for j, (ci, lab) in enumerate(zip(cis, ("EE", "BB"))):
                r = np.arange(ci * nrow, (ci + 1) * nrow)
                cl = lam(r, C_ell[lab]) if target in ("total_covariance", "snr") else None
                parts.append(kept(comp_matrix(V[np.ix_(r, cols)], cols, cl),
                                  e_f[j] if isinstance(e_f, tuple) else None,
                                  m_f[j] if isinstance(m_f, tuple) else None))
            Q, sv, _ = np.linalg.svd(np.hstack(parts), full_matrices=False)
            blocks.append((cols, Q[:, sv > 1e-10 * sv[0]]))
        else:
            cl = None
            if target in ("total_covariance", "snr"):
                cl = lam(rows, next(iter(C_ell.values())) if isinstance(C_ell, dict) else C_ell)
            e_s = e_f[0] if isinstance(e_f, tuple) else e_f
            m_s = None if isinstance(m_f, tuple) else m_f
            blocks.append((cols, kept(comp_matrix(V[np.ix_(rows, cols)], cols, cl), e_s, m_s)))
    dim = sum(b.shape[1] for _, b in blocks)
    U = np.zeros((L.n, dim))
    c = 0
    for cols, b in blocks:
        U[cols, c:c + b.shape[1]] = b
        c += b.shape[1]
    return U


def compressed_estimator(L, N, tab, tab_fixed, maps, signal_pixel, epsilon=None, mode_fraction=None,
                         target="noise_weighted", weights=None, C_ell=None):
    """F, raw bias, raw q of the compressed pixel basis: C_c = U^T C U with C
    the harmonic-basis covariance, derivatives (V U)^T E_l (V U), bias with
    U^T N U, maps U^T x (cosmocore/basis/pixel.py:1614-1996)."""
    lmin, lmax = L.lmin, L.lmax
    W = L.param_weights() if weights is None else weights
    V = harmonic_operator(L, lmin, lmax)
    S = signal_harmonic(L, tab, lmin, lmax, signal_pixel, tab_fixed)
    S_fixed = signal_pixel(_outside(tab_fixed, lmin, lmax))
    switch = lmax < L.lmax_signal or lmin > 2
    N_eff = N + S_fixed if switch else N
    U = compression_basis(L, V, N_eff, lmin, lmax, epsilon, mode_fraction, target, C_ell)
    Cc = U.T @ (N + S) @ U
    Cc_inv = np.linalg.inv(Cc)
    VU = V @ U
    G = VU @ Cc_inv @ VU.T
    F = _fisher_from_G(L, G, lmin, lmax, W)
    Z = VU @ Cc_inv
    bias, q = _qml_from_Z(L, Z, U.T @ N @ U, U.T @ maps, lmin, lmax, W)
    return F, bias, q, U.shape[1]


def _outside(tab, lmin, lmax):
    out = np.array(tab, dtype=np.float64, copy=True)
    out[:, lmin:lmax + 1] = 0.0
    return out
