"""Harmonic-basis estimator on the device (the reference's ``basis="harmonic"``).

The reference's harmonic basis (cosmocore/basis/harmonic.py:191-1252,
harmonic_basis.py:20-180, qube/fisher.py:416-500, 575-583) writes the
covariance over the inference window [lmin, lmax] as V^T Lambda V with V the
real spherical harmonics of the active pixels (spin 0: T; spin 2: E and B
over [Q | U]), adds the pixel-space signal of the multipoles outside the
window (S_fixed), and exploits dC/dC_l = t_l V_l^T V_l: every Fisher trace,
noise bias and quadratic form becomes a contraction over (l, m) modes.

Here:
* ``V`` (n_modes x n, FP64) is built once per layout by ``cf_harmonic_operator``;
* ``signal`` = S_fixed (the pixel builder on the C_l table with the window
  zeroed) + V^T (Lambda V) on the DMMA GEMM;
* C^-1 comes from the dense Jacobi-scaled Cholesky inverse of the engine (the
  reference uses Sherman-Morrison-Woodbury; both are the exact inverse of the
  same C);
* ``fisher_qml``: Z = V C^-1, G = Z V^T, F from G by ``cf_harmonic_fisher``,
  the bias from Z N against Z and q from z = Z x by ``cf_harmonic_pair``.

For the config-1 problem (n = 5952, three components, l = 2..47) this is four
n_modes x n x n-class GEMMs (~2e12 FLOP) instead of 276 A_b = C^-1 dC_b
products.  Always FP64.
"""

from __future__ import annotations

import numpy as np
import torch

from ._lib import check, stream
from .engine import Engine

F64 = torch.float64


def components(L):
    """[(field index, 'T' | 'E' | 'B')] in row order of V."""
    out = []
    for fi, f in enumerate(L.fields):
        if f.spin == 0:
            out.append((fi, "T"))
        else:
            out.extend([(fi, "E"), (fi, "B")])
    return out


def spectrum_components(L, comps, s):
    """(u, v) component indices of spectrum s (u == v for auto spectra)."""
    sp = L.spectra[s]
    fi, fj = sp.fi, sp.fj
    fs = L.fields
    if fs[fi].spin == 0 and fs[fj].spin == 0:
        return comps.index((fi, "T")), comps.index((fj, "T"))
    if fs[fi].spin == 2 and fs[fj].spin == 2:
        a, b = {0: ("E", "E"), 1: ("B", "B"), 2: ("E", "B")}[sp.mode]
        return comps.index((fi, a)), comps.index((fj, b))
    t, p = (fi, fj) if fs[fi].spin == 0 else (fj, fi)
    return comps.index((t, "T")), comps.index((p, "E" if sp.mode == 0 else "B"))


def n_modes_reference(L) -> int:
    """Mode count the reference's basis selector uses (basis/__init__.py:48-84)."""
    base = (L.lmax + 1) ** 2 - 4
    return sum(2 * base if f.spin == 2 else base for f in L.fields)


def auto_method(L) -> str:
    """The reference's leading-order cost model (basis/__init__.py:87-115):
    harmonic when n_modes^3 <= (n_bins + 1) n_pix^3, else pixel."""
    return "harmonic" if float(n_modes_reference(L)) ** 3 <= float(L.nbins + 1) * float(L.n) ** 3 else "pixel"


class HarmonicPlan:
    """V and its index tables for one layout, on the engine's device."""

    def __init__(self, E: Engine):
        L = E.L
        if L.lmin < 2:
            raise ValueError(f"the harmonic basis needs lmin >= 2, got {L.lmin}")
        self.E, self.L = E, L
        self.comps = components(L)
        nc = len(self.comps)
        if nc > 3:
            raise NotImplementedError(f"harmonic basis: at most 3 components (T, E, B), got {nc}")
        self.nc = nc
        self.lmin, self.lmax = L.lmin, L.lmax
        self.Lp = L.lmax_signal + 1
        if self.lmax >= self.Lp:
            raise ValueError("inference lmax above lmax_signal")
        nrow = (self.lmax + 1) ** 2 - self.lmin ** 2
        self.nrow, self.nm = nrow, nc * nrow
        off = np.zeros((nc, self.Lp), dtype=np.int64)
        rowinfo = np.zeros((self.nm, 2), dtype=np.int32)
        for c in range(nc):
            for ell in range(self.lmin, self.lmax + 1):
                r0 = c * nrow + ell * ell - self.lmin ** 2
                off[c, ell] = r0
                rowinfo[r0:r0 + 2 * ell + 1] = (c, ell)
        dev = E.dev
        self.off = torch.from_numpy(off).to(dev)
        self.rowinfo = torch.from_numpy(rowinfo).to(dev)
        pairs = [spectrum_components(L, self.comps, s) for s in range(L.nspectra)]
        self.pairs = pairs
        self.su = torch.tensor([p[0] for p in pairs], dtype=torch.int32, device=dev)
        self.sv = torch.tensor([p[1] for p in pairs], dtype=torch.int32, device=dev)
        self.V = torch.zeros((self.nm, L.n), dtype=F64, device=dev)
        lib = E.lib
        for c, (fi, kind) in enumerate(self.comps):
            f = L.fields[fi]
            check(lib.cf_harmonic_operator(f.spin, int(kind == "B"), f.npix, E.vec[fi].data_ptr(), self.lmin,
                                           self.lmax, self.V.data_ptr(), L.n, c * nrow, f.offset, stream()),
                  "cf_harmonic_operator")

    # ------------------------------------------------------------------
    def signal(self, cl_table) -> torch.Tensor:
        """S = S_fixed + V^T Lambda V from a beam-smoothed (nspectra, L+1) table."""
        E, L = self.E, self.L
        tab = torch.as_tensor(cl_table, dtype=F64, device=E.dev).contiguous()
        fixed = tab.clone()
        fixed[:, self.lmin:self.lmax + 1] = 0.0
        S = E.signal(fixed)
        lam = torch.zeros((self.nc, self.nc, self.Lp), dtype=F64, device=E.dev)
        for s, (u, v) in enumerate(self.pairs):
            lam[u, v, self.lmin:self.lmax + 1] = tab[s, self.lmin:self.lmax + 1]
            lam[v, u, self.lmin:self.lmax + 1] = tab[s, self.lmin:self.lmax + 1]
        LV = torch.empty_like(self.V)
        check(E.lib.cf_harmonic_lambda(self.nm, L.n, self.nc, self.lmin, self.rowinfo.data_ptr(),
                                       self.off.data_ptr(), lam.data_ptr(), self.Lp, self.V.data_ptr(), L.n,
                                       LV.data_ptr(), L.n, stream()), "cf_harmonic_lambda")
        E.gemm(self.V, LV, C=S, beta=1.0, transa=True)
        return S

    def fisher_qml(self, Cinv: torch.Tensor, N: torch.Tensor | None = None, maps: torch.Tensor | None = None,
                   want_fisher: bool = True):
        """F (P x P), raw bias (P,) and raw q (nsims x P), same convention as Engine.fisher_qml."""
        E, L = self.E, self.L
        P, nb, n = L.n_params, L.nbins, L.n
        dev = E.dev
        Z = E.gemm(self.V, Cinv)
        F = torch.zeros((P, P), dtype=F64, device=dev)
        lib = E.lib
        if want_fisher:
            G = E.gemm(Z, self.V, transb=True)
            check(lib.cf_harmonic_fisher(self.nc, self.lmin, self.lmax, self.Lp, G.data_ptr(), self.nm,
                                         self.off.data_ptr(), L.nspectra, self.su.data_ptr(), self.sv.data_ptr(),
                                         E.deriv_tab.data_ptr(), E.deriv_bin.data_ptr(), nb, F.data_ptr(), P,
                                         stream()), "cf_harmonic_fisher")
            del G
        bias = q = None
        if N is not None:
            ZN = E.gemm(Z, N.to(dev, F64).contiguous())
            bias = torch.zeros(P, dtype=F64, device=dev)
            check(lib.cf_harmonic_pair(self.lmin, self.lmax, self.Lp, ZN.data_ptr(), n, Z.data_ptr(), n, n, 0,
                                       self.off.data_ptr(), L.nspectra, self.su.data_ptr(), self.sv.data_ptr(),
                                       E.deriv_tab.data_ptr(), E.deriv_bin.data_ptr(), nb, bias.data_ptr(), 0,
                                       stream()), "cf_harmonic_pair")
            del ZN
        if maps is not None:
            X = maps.to(dev, F64).contiguous()
            ns = X.shape[1]
            zx = E.gemm(Z, X)
            q = torch.zeros((ns, P), dtype=F64, device=dev)
            check(lib.cf_harmonic_pair(self.lmin, self.lmax, self.Lp, zx.data_ptr(), ns, zx.data_ptr(), ns, ns, 1,
                                       self.off.data_ptr(), L.nspectra, self.su.data_ptr(), self.sv.data_ptr(),
                                       E.deriv_tab.data_ptr(), E.deriv_bin.data_ptr(), nb, q.data_ptr(), P,
                                       stream()), "cf_harmonic_pair")
        return F, bias, q


def qml_solve(E: Engine, cls: dict, N: torch.Tensor, maps: torch.Tensor, plan: HarmonicPlan | None = None):
    """S, C^-1, F, q, bias, F^-1, C_hat of the harmonic-basis estimator (FP64)."""
    plan = plan or HarmonicPlan(E)
    L = E.L
    S = plan.signal(L.smoothed_cl_table(cls))
    Cinv = E.spd_inverse(S + N)
    F, bias, q = plan.fisher_qml(Cinv, N, maps)
    if L.remove_nb:
        q = q - bias[None, :]
    Finv = E.spd_inverse(F.clone())
    return dict(S=S, Cinv=Cinv, fisher=F, q=q, bias=bias, invfisher=Finv, clhat=E.gemm(q, Finv),
                noise_bias=E.gemm(bias[None, :], Finv)[0])
