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

``CompressedPlan`` is the reference's eigen-truncated pixel basis on top of
the same contractions (V -> V U in the kept subspace U).
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
    def outside(self, cl_table) -> torch.Tensor:
        """The table with the inference window [lmin, lmax] zeroed (the S_fixed spectra)."""
        t = torch.as_tensor(cl_table, dtype=F64, device=self.E.dev).clone()
        t[:, self.lmin:self.lmax + 1] = 0.0
        return t

    def signal(self, cl_table, fixed_table=None) -> torch.Tensor:
        """S = S_fixed + V^T Lambda V from beam-smoothed (nspectra, L+1) tables:
        the window from cl_table, S_fixed from fixed_table (the fiducial
        spectra; default cl_table)."""
        E, L = self.E, self.L
        tab = torch.as_tensor(cl_table, dtype=F64, device=E.dev).contiguous()
        S = E.signal(self.outside(tab if fixed_table is None else fixed_table))
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
                   want_fisher: bool = True, V: torch.Tensor | None = None, tables=None):
        """F (P x P), raw bias (P,) and raw q (nsims x P), same convention as Engine.fisher_qml.

        V: the operator whose columns span the space of Cinv / N / maps
        (default the pixel-space V; a compressed basis passes V U).
        tables: (deriv_tab, deriv_bin, nbins, n_params) of another binning."""
        E, L = self.E, self.L
        V = self.V if V is None else V
        tab_t, bin_t, nb, P = tables if tables is not None else (E.deriv_tab, E.deriv_bin, L.nbins, L.n_params)
        n = V.shape[1]
        dev = E.dev
        Z = E.gemm(V, Cinv)
        F = torch.zeros((P, P), dtype=F64, device=dev)
        lib = E.lib
        if want_fisher:
            G = E.gemm(Z, V, transb=True)
            check(lib.cf_harmonic_fisher(self.nc, self.lmin, self.lmax, self.Lp, G.data_ptr(), self.nm,
                                         self.off.data_ptr(), L.nspectra, self.su.data_ptr(), self.sv.data_ptr(),
                                         tab_t.data_ptr(), bin_t.data_ptr(), nb, F.data_ptr(), P,
                                         stream()), "cf_harmonic_fisher")
            del G
        bias = q = None
        if N is not None:
            ZN = E.gemm(Z, N.to(dev, F64).contiguous())
            bias = torch.zeros(P, dtype=F64, device=dev)
            check(lib.cf_harmonic_pair(self.lmin, self.lmax, self.Lp, ZN.data_ptr(), n, Z.data_ptr(), n, n, 0,
                                       self.off.data_ptr(), L.nspectra, self.su.data_ptr(), self.sv.data_ptr(),
                                       tab_t.data_ptr(), bin_t.data_ptr(), nb, bias.data_ptr(), 0,
                                       stream()), "cf_harmonic_pair")
            del ZN
        if maps is not None:
            X = maps.to(dev, F64).contiguous()
            ns = X.shape[1]
            zx = E.gemm(Z, X)
            q = torch.zeros((ns, P), dtype=F64, device=dev)
            check(lib.cf_harmonic_pair(self.lmin, self.lmax, self.Lp, zx.data_ptr(), ns, zx.data_ptr(), ns, ns, 1,
                                       self.off.data_ptr(), L.nspectra, self.su.data_ptr(), self.sv.data_ptr(),
                                       tab_t.data_ptr(), bin_t.data_ptr(), nb, q.data_ptr(), P,
                                       stream()), "cf_harmonic_pair")
        return F, bias, q


def keep_modes(evals: np.ndarray, epsilon=None, mode_fraction=None) -> np.ndarray:
    """Indices of the kept eigenvectors, by descending eigenvalue
    (cosmocore/basis/pixel.py:265-311): |lambda| > epsilon max |lambda|, or the
    leading ceil(mode_fraction n_significant), or everything above 1e-10 max."""
    order = np.argsort(evals)[::-1]
    ev = evals[order]
    amax = float(np.max(np.abs(ev)))
    if mode_fraction is not None:
        n_sig = int(np.sum(ev > 1e-10 * amax))
        keep = np.zeros(ev.size, bool)
        keep[:max(1, int(np.ceil(mode_fraction * n_sig)))] = True
    elif epsilon is not None:
        keep = np.abs(ev) > epsilon * amax
    else:
        keep = np.abs(ev) > 1e-10 * amax
    return order[keep]


def _per_field(x, nf, what):
    """A scalar or a per-field list of thresholds as one value per field; an
    entry may be an (E, B) pair for a spin-2 field."""
    if x is None or isinstance(x, (int, float)):
        return [x] * nf
    if isinstance(x, tuple) and len(x) == 2 and nf == 1:
        return [x]
    x = list(x)
    if len(x) != nf:
        raise ValueError(f"{what} needs one value per field ({nf}), got {len(x)}")
    return [tuple(v) if isinstance(v, (tuple, list)) else v for v in x]


def _sym_sqrt(S: torch.Tensor) -> torch.Tensor:
    """S^1/2 of a symmetric positive semi-definite matrix from its
    eigendecomposition, eigenvalues clipped at 1e-30 (cosmocore/basis/pixel.py:
    339-348)."""
    w, Q = torch.linalg.eigh(S)
    return (Q * torch.sqrt(torch.clamp(w, min=1e-30))[None, :]) @ Q.T


class CompressedPlan:
    """Eigen-truncated pixel basis (the reference's PixelBasis with epsilon /
    mode_fraction, cosmocore/basis/pixel.py:265-557, 965-1055, 1493-1996).

    Per field f, the kept eigenvectors U_f of the compression matrix of the
    field's rows of V (V_f, n_f columns) and its block of the effective noise
    N_eff = N + S_fixed (N itself when the inference window covers the signal
    band):

    * "harmonic":         P_f = V_f^T V_f
    * "noise_weighted":   P_f (N_eff^-1)_ff P_f  (the default)
    * "total_covariance": P_f C_f^-1 P_f, C_f = (N_eff)_ff + V_f^T Lambda V_f
    * "snr":              S_f^1/2 (N_eff^-1)_ff S_f^1/2, S_f = V_f^T Lambda V_f

    Lambda holds C_l at each row's multipole (the ``C_ell`` array, or the first
    entry of a ``C_ell`` dict).  A spin-2 field given an (E, B) pair of
    thresholds is split: the E rows and the B rows each get their own matrix
    (Lambda from ``C_ell["EE"]`` / ``["BB"]``) and threshold, and the two sets
    of kept vectors are orthogonalised together by an SVD (singular values
    above 1e-10 of the largest).  U = diag(U_f) (n x dim).  The estimator then
    runs in the kept subspace: C_c = U^T C U, derivatives (V U)^T E_l (V U),
    noise U^T N U, maps U^T x, through the same harmonic contractions.  The
    symmetric eigendecompositions and the SVD are cuSOLVER's
    (torch.linalg.eigh / svd, once per basis).
    """

    TARGETS = ("harmonic", "noise_weighted", "total_covariance", "snr")

    def __init__(self, hp: HarmonicPlan, N: torch.Tensor, fixed_table, epsilon=None, mode_fraction=None,
                 target: str = "noise_weighted", C_ell=None):
        if epsilon is not None and mode_fraction is not None:
            raise ValueError("epsilon and mode_fraction are mutually exclusive")
        if target not in self.TARGETS:
            raise ValueError(f"Unknown compression target '{target}'. Available: {list(self.TARGETS)}")
        if target in ("total_covariance", "snr") and C_ell is None:
            raise ValueError(f"C_ell is required for '{target}' compression_target")
        E, L = hp.E, hp.L
        nf = len(L.fields)
        eps = _per_field(epsilon, nf, "epsilon")
        mfs = _per_field(mode_fraction, nf, "mode_fraction")
        for mf in mfs:
            for v in (mf if isinstance(mf, tuple) else (mf,)):
                if v is not None and not (0 < v <= 1):
                    raise ValueError(f"mode_fraction must be in (0, 1], got {v}")
        if epsilon is None and mode_fraction is None:
            eps = [1e-6] * nf
        self.hp, self.E, self.L = hp, E, L
        N = N.to(E.dev, F64).contiguous()
        switch = hp.lmax < L.lmax_signal or hp.lmin > 2
        N_eff = N + E.signal(hp.outside(fixed_table)) if switch else N.clone()
        Ninv = E.spd_inverse(N_eff.clone()) if target in ("noise_weighted", "snr") else None
        ell_of_row = hp.rowinfo[:, 1].to(torch.long)

        def lam_rows(rows, cl):
            c = torch.as_tensor(np.asarray(cl, dtype=np.float64), device=E.dev)
            ell = ell_of_row[rows]
            return torch.where(ell < c.numel(), c[torch.clamp(ell, max=c.numel() - 1)], torch.zeros_like(c[:1]))

        def comp_matrix(Vs, cols, cl):
            P = E.gemm(Vs, Vs, transa=True)
            if target == "harmonic":
                return P
            if target == "noise_weighted":
                return E.gemm(E.gemm(P, Ninv[cols, cols].contiguous()), P)
            S = E.gemm(Vs, Vs * cl[:, None], transa=True)
            if target == "total_covariance":
                Cinv = E.spd_inverse(N_eff[cols, cols] + S)
                return E.gemm(E.gemm(P, Cinv), P)
            Sq = _sym_sqrt(0.5 * (S + S.T))
            return E.gemm(E.gemm(Sq, Ninv[cols, cols].contiguous()), Sq)

        def kept(M, e, mf):
            M = 0.5 * (M + M.T)
            ev, vec = torch.linalg.eigh(M)
            keep = keep_modes(ev.cpu().numpy(), e, mf)
            return vec[:, torch.from_numpy(keep.copy()).to(E.dev)]

        def first_cl():
            return next(iter(C_ell.values())) if isinstance(C_ell, dict) else C_ell

        blocks = []
        for fi, f in enumerate(L.fields):
            cols = slice(f.offset, f.offset + f.nrows)
            cs = [c for c, (g, _) in enumerate(hp.comps) if g == fi]
            rows = torch.arange(cs[0] * hp.nrow, (cs[-1] + 1) * hp.nrow, device=E.dev)
            e_f, m_f = eps[fi], mfs[fi]
            split = f.spin == 2 and (isinstance(e_f, tuple) or isinstance(m_f, tuple))
            if split:
                parts = []
                for j, (c, lab) in enumerate(zip(cs, ("EE", "BB"))):
                    r = torch.arange(c * hp.nrow, (c + 1) * hp.nrow, device=E.dev)
                    Vs = hp.V[r, cols].contiguous()
                    cl = None
                    if target in ("total_covariance", "snr"):
                        src = C_ell.get(lab) if isinstance(C_ell, dict) else None
                        if src is None:
                            raise ValueError(f"C_ell[{lab!r}] is required for '{target}' with separate E / B "
                                             "thresholds")
                        cl = lam_rows(r, src)
                    parts.append(kept(comp_matrix(Vs, cols, cl), e_f[j] if isinstance(e_f, tuple) else None,
                                      m_f[j] if isinstance(m_f, tuple) else None))
                Ucat = torch.cat(parts, dim=1)
                Q, sv, _ = torch.linalg.svd(Ucat, full_matrices=False)
                blocks.append((cols, Q[:, sv > 1e-10 * sv[0]]))
            else:
                Vf = hp.V[rows, cols].contiguous()
                cl = lam_rows(rows, first_cl()) if target in ("total_covariance", "snr") else None
                e_s = e_f[0] if isinstance(e_f, tuple) else e_f
                m_s = None if isinstance(m_f, tuple) else m_f
                blocks.append((cols, kept(comp_matrix(Vf, cols, cl), e_s, m_s)))
        self.dim = sum(b.shape[1] for _, b in blocks)
        self.dims = [b.shape[1] for _, b in blocks]
        self.U = torch.zeros((L.n, self.dim), dtype=F64, device=E.dev)
        c = 0
        for cols, b in blocks:
            self.U[cols, c:c + b.shape[1]] = b
            c += b.shape[1]
        self.VU = E.gemm(hp.V, self.U)
        self.Nc = E.gemm(E.gemm(self.U, N, transa=True), self.U)

    def project(self, C: torch.Tensor) -> torch.Tensor:
        """U^T C U."""
        return self.E.gemm(self.E.gemm(self.U, C, transa=True), self.U)

    def fisher_qml(self, Cc_inv, with_bias: bool = True, maps=None, want_fisher: bool = True, tables=None):
        """F, raw bias, raw q in the kept subspace (maps in pixel space)."""
        xc = self.E.gemm(self.U, maps.to(self.E.dev, F64).contiguous(), transa=True) if maps is not None else None
        return self.hp.fisher_qml(Cc_inv, self.Nc if with_bias else None, xc, want_fisher=want_fisher, V=self.VU,
                                  tables=tables)


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
