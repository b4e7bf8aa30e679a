"""Device pipeline for one problem layout: S, C^-1, Fisher, QML, lnL.

The host code here only sequences device kernels from ``libcfb200.so`` on a
CUDA stream; device memory comes from PyTorch.  Stages (reference
counterparts in brackets):

* ``signal``       S = sum_l C~_l kernels  [cosmocore/signal_kernels.py:390-537]
* ``spd_inverse``  C^-1 by the Jacobi-scaled Cholesky inverse
                   [cosmocore/basics/linalg.py:152-219]
* ``fisher_qml``   per spectrum: derivative blocks dC_b of all its bins in one
                   pass, A_b = C^-1 dC_b (and A_b^T) on the DMMA GEMM, Fisher
                   traces as dense contractions against every earlier
                   spectrum, noise bias and quadratic forms from the same
                   derivative blocks  [qube/fisher.py:501-607,
                   qube/spectra.py:1124-1186]
* ``lnl``          batched S(theta) + s N, Cholesky, chi2 and ln|C| from the
                   factor  [picslike/picslike.py:568-664]

Memory layout in HBM: all matrices row-major FP64.  A_b is kept per column
segment (one field's rows) as n x (nbins * m) slabs for every spectrum seen
so far; A_b^T slabs only for the spectrum being processed.
"""

from __future__ import annotations

import ctypes

import numpy as np
import torch

from . import layout as lay
from ._lib import CF_ERR_TIMEOUT, check, lib, ptr, stream

F64 = torch.float64


def _off(t: torch.Tensor, elems: int) -> int:
    return t.data_ptr() + int(elems) * t.element_size()


# BF16x6 product list (plane pairs (0,0), (0,1), (1,0), (0,2), (1,1), (2,0)) as
# host int arrays for the tensor-core GEMMs; the arrays live as long as the module
_X6_ARRAYS = tuple((ctypes.c_int * 6)(*t) for t in ((0, 0, 1, 0, 1, 2), (0, 1, 0, 2, 1, 0)))
_X6_TERMS = tuple(ctypes.cast(a, ctypes.c_void_p) for a in _X6_ARRAYS)


class Engine:
    """Device-resident tables of one layout and the kernels that use them."""

    def __init__(self, L: lay.Layout, device=None):
        self.L = L
        self.dev = torch.device(device) if device is not None else torch.device("cuda")
        self.lib = lib()
        self.vec = [torch.from_numpy(np.ascontiguousarray(f.vectors.T)).to(self.dev, F64)
                    for f in L.fields]
        W = L.param_weights()
        nb, Lmax = L.nbins, L.lmax_signal
        tabs, bins = [], []
        for s in range(L.nspectra):
            t = np.zeros(Lmax + 1)
            b = np.full(Lmax + 1, -1, dtype=np.int32)
            for k in range(nb):
                lo, hi = int(L.bin_lmins[k]), min(int(L.bin_lmaxs[k]), Lmax)
                if lo <= hi:
                    b[lo: hi + 1] = k
                    t[lo: hi + 1] = W[s * nb + k, lo: hi + 1]
            tabs.append(t)
            bins.append(b)
        self.deriv_tab = torch.from_numpy(np.stack(tabs)).to(self.dev, F64)
        self.deriv_bin = torch.from_numpy(np.stack(bins)).to(self.dev, torch.int32)
        self.probe = None  # {tag: [(start_event, end_event, work)]} when timing kernels
        self.block_of_spec = {}
        for bi, blk in enumerate(L.blocks):
            for s in blk.spectra:
                self.block_of_spec[s] = bi

    # ------------------------------------------------------------------
    def _launch_block(self, blk, mode, tabs, bin_of, out, ld, row_off, col_off, bin_stride,
                      outT, ldT, rowT_off, colT_off, binT_stride, batch=1, tstride=0, ostride=0):
        L = self.L
        fa, fb = L.fields[blk.fa], L.fields[blk.fb]
        va, vb = self.vec[blk.fa], self.vec[blk.fb]
        t0, t1, t2 = (tabs + [None, None, None])[:3]
        rc = self.lib.cf_build_block(
            blk.kind, mode, fa.npix, va.data_ptr(), fb.npix, vb.data_ptr(), L.lmax_signal,
            t0, t1, t2, bin_of, out, ld, row_off, col_off, bin_stride, outT, ldT, rowT_off,
            colT_off, binT_stride, batch, tstride, ostride, stream())
        check(rc, "cf_build_block")

    def signal(self, cl_table, out: torch.Tensor | None = None) -> torch.Tensor:
        """S (n x n) or a batch (B x n x n) from beam-smoothed C_l tables.

        ``cl_table``: (nspectra, L+1) or (B, nspectra, L+1) in spectrum order.
        """
        L = self.L
        cl = torch.as_tensor(cl_table, dtype=F64, device=self.dev).contiguous()
        batched = cl.dim() == 3
        B = cl.shape[0] if batched else 1
        n, Lp = L.n, L.lmax_signal + 1
        if out is None:
            out = torch.zeros((B, n, n) if batched else (n, n), dtype=F64, device=self.dev)
        tstride = L.nspectra * Lp
        for blk in L.blocks:
            fa, fb = L.fields[blk.fa], L.fields[blk.fb]
            by_mode = {L.spectra[k].mode: k for k in blk.spectra}
            if blk.kind in (lay.KIND_00_AUTO, lay.KIND_00_CROSS):
                order = [blk.spectra[0]]
            elif blk.kind == lay.KIND_22_AUTO:
                order = [by_mode.get(0), by_mode.get(1), by_mode.get(2)]
            else:
                order = [by_mode.get(0), by_mode.get(1)]
            tabs = [None if k is None else _off(cl, k * Lp) for k in order]
            if tabs[0] is None:
                continue
            self._launch_block(blk, -1, tabs, None, out.data_ptr(), n, fb.offset, fa.offset, 0,
                               out.data_ptr(), n, fa.offset, fb.offset, 0, batch=B,
                               tstride=tstride, ostride=n * n)
        return out

    # ------------------------------------------------------------------
    def spd_inverse(self, A: torch.Tensor) -> torch.Tensor:
        """In place Jacobi-scaled Cholesky inverse of one SPD matrix or a batch."""
        n = A.shape[-1]
        B = A.shape[0] if A.dim() == 3 else 1
        ws = self.lib.cf_spd_inverse_workspace(n, B)
        work = torch.empty(ws // 8 + 1, dtype=F64, device=A.device)
        info = torch.zeros(B, dtype=torch.int32, device=A.device)
        ev = self._probe_begin("spd_inverse")
        check(self.lib.cf_spd_inverse(n, A.data_ptr(), n, n * n, B, work.data_ptr(), info.data_ptr(),
                                      stream()), "cf_spd_inverse")
        self._probe_end("spd_inverse", ev, 0)
        bad = info.cpu()
        if int(bad.abs().max()) != 0:
            raise ValueError(f"dpotrf failed with info={int(bad[bad != 0][0])}")
        return A

    def _probe_begin(self, tag):
        if self.probe is None:
            return None
        ev = (torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True))
        ev[0].record()
        return ev

    def _probe_end(self, tag, ev, work):
        if ev is not None:
            ev[1].record()
            self.probe.setdefault(tag, []).append((ev[0], ev[1], float(work)))

    def gemm(self, A, B, C=None, alpha=1.0, beta=0.0, transa=False, transb=False, CT=None, tag=None):
        M = A.shape[1] if transa else A.shape[0]
        K = A.shape[0] if transa else A.shape[1]
        N = B.shape[0] if transb else B.shape[1]
        if C is None:
            C = torch.empty((M, N), dtype=F64, device=A.device)
        ev = self._probe_begin(tag) if tag else None
        if tag:
            torch.cuda.nvtx.range_push(tag)
        check(self.lib.cf_dgemm(int(transa), int(transb), M, N, K, alpha, A.data_ptr(), A.stride(0), 0,
                                B.data_ptr(), B.stride(0), 0, beta, C.data_ptr(), C.stride(0), 0,
                                ptr(CT), CT.stride(0) if CT is not None else 0, 0, 1, 0, stream()),
              "cf_dgemm")
        if tag:
            torch.cuda.nvtx.range_pop()
            self._probe_end(tag, ev, 2.0 * M * N * K)
        return C

    # ------------------------------------------------------------------
    def _deriv_blocks(self, s: int):
        """Derivative blocks of every bin of spectrum s, in one build pass."""
        L = self.L
        blk = L.blocks[self.block_of_spec[s]]
        fa, fb = L.fields[blk.fa], L.fields[blk.fb]
        nb, Lp = L.nbins, L.lmax_signal + 1
        mode = L.spectra[s].mode
        tab = [_off(self.deriv_tab, s * Lp)]
        bins = _off(self.deriv_bin, s * Lp)
        if blk.kind in (lay.KIND_00_AUTO, lay.KIND_22_AUTO):
            m = fa.nrows
            D = torch.zeros((m, nb * m), dtype=F64, device=self.dev)
            self._launch_block(blk, mode, tab, bins, D.data_ptr(), nb * m, 0, 0, m,
                               D.data_ptr(), nb * m, 0, 0, m)
            return blk, {"auto": D}
        R, Cc = fb.nrows, fa.nrows
        Dba = torch.zeros((R, nb * Cc), dtype=F64, device=self.dev)
        Dab = torch.zeros((Cc, nb * R), dtype=F64, device=self.dev)
        self._launch_block(blk, mode, tab, bins, Dba.data_ptr(), nb * Cc, 0, 0, Cc,
                           Dab.data_ptr(), nb * R, 0, 0, R)
        return blk, {"ba": Dba, "ab": Dab}

    def derivative_dense(self, p: int) -> torch.Tensor:
        """Full n x n dC_p (test helper; the Fisher path never forms it)."""
        L = self.L
        s, b = divmod(p, L.nbins)
        blk, D = self._deriv_blocks(s)
        fa, fb = L.fields[blk.fa], L.fields[blk.fb]
        out = torch.zeros((L.n, L.n), dtype=F64, device=self.dev)
        if "auto" in D:
            m = fa.nrows
            out[fa.offset: fa.offset + m, fa.offset: fa.offset + m] = D["auto"][:, b * m:(b + 1) * m]
        else:
            R, Cc = fb.nrows, fa.nrows
            blkba = D["ba"][:, b * Cc:(b + 1) * Cc]
            out[fb.offset: fb.offset + R, fa.offset: fa.offset + Cc] = blkba
            out[fa.offset: fa.offset + Cc, fb.offset: fb.offset + R] = D["ab"][:, b * R:(b + 1) * R]
        return out

    def qml_reduce(self, M: torch.Tensor | None = None, Y: torch.Tensor | None = None):
        """Raw bias b_p = 1/2 Tr(M dC_p) (M = C^-1 N C^-1) and q_p = 1/2 y^T dC_p y
        for the columns y of Y = C^-1 X, building every dC_p entry in registers
        and reducing it at once (no derivative matrix in HBM)."""
        L = self.L
        n, nb, P, Lp = L.n, L.nbins, L.n_params, L.lmax_signal + 1
        bias = torch.zeros(P, dtype=F64, device=self.dev) if M is not None else None
        nsims = 0 if Y is None else Y.shape[1]
        q = torch.zeros((nsims, P), dtype=F64, device=self.dev) if nsims else None
        if M is not None:
            M = M.contiguous()
        for s in range(L.nspectra):
            blk = L.blocks[self.block_of_spec[s]]
            fa, fb = L.fields[blk.fa], L.fields[blk.fb]
            mode = L.spectra[s].mode
            tab = _off(self.deriv_tab, s * Lp)
            bins = _off(self.deriv_bin, s * Lp)
            va, vb = self.vec[blk.fa], self.vec[blk.fb]
            for m0 in range(0, max(nsims, 1), 4):
                nv = min(4, nsims - m0) if nsims else 0
                Yc = Y[:, m0:m0 + nv].contiguous() if nv else None
                with_bias = M is not None and m0 == 0
                if not with_bias and nv == 0:
                    continue
                check(self.lib.cf_build_block_reduce(
                    blk.kind, mode, fa.npix, va.data_ptr(), fb.npix, vb.data_ptr(), L.lmax_signal,
                    tab, None, None, bins, nb, ptr(M) if with_bias else None, n,
                    ptr(Yc), nv, nv, fb.offset, fa.offset, 0.5,
                    _off(bias, s * nb) if with_bias else None, _off(q, m0 * P + s * nb) if nv else None, P,
                    stream()), "cf_build_block_reduce")
        return bias, q

    def fisher_qml(self, Cinv: torch.Tensor, N: torch.Tensor | None = None,
                   maps: torch.Tensor | None = None, want_fisher: bool = True, fused_reduce: bool = True):
        """F (P x P), raw bias (P,), raw q (nsims x P) by per-spectrum passes.

        Without the Fisher matrix (want_fisher False) and with fused_reduce,
        bias and q come from qml_reduce (derivative entries reduced where they
        are built); otherwise from the derivative blocks the Fisher pass
        builds anyway."""
        L = self.L
        n, nb, P = L.n, L.nbins, L.n_params
        dev = self.dev
        if not want_fisher and fused_reduce and nb <= 128 and (N is not None or maps is not None):
            Y = self.gemm(Cinv, maps.to(dev, F64).contiguous()) if maps is not None else None
            M = self.gemm(Cinv, self.gemm(N, Cinv)) if N is not None else None
            bias, q = self.qml_reduce(M, Y)
            return torch.zeros((P, P), dtype=F64, device=dev), bias, q
        F = torch.zeros((P, P), dtype=F64, device=dev)
        bias = torch.zeros(P, dtype=F64, device=dev) if N is not None else None
        Y = None
        nsims = 0
        if maps is not None:
            X = maps.to(dev, F64).contiguous()
            nsims = X.shape[1]
            Y = self.gemm(Cinv, X)
            q = torch.zeros((nsims, P), dtype=F64, device=dev)
        else:
            q = None
        M = None
        if N is not None:
            M = self.gemm(Cinv, self.gemm(N, Cinv))
        X_slabs = {}
        seg = {i: (f.offset, f.nrows) for i, f in enumerate(L.fields)}
        cols_of = {}
        for s2 in range(L.nspectra):
            blk, D = self._deriv_blocks(s2)
            fa, fb = L.fields[blk.fa], L.fields[blk.fb]
            # ---- noise bias and quadratic forms from the derivative blocks
            if M is not None or Y is not None:
                if "auto" in D:
                    args = (D["auto"], fa.nrows, fa.nrows, fa.offset, fa.offset, 0.5)
                else:
                    args = (D["ba"], fb.nrows, fa.nrows, fb.offset, fa.offset, 1.0)
                Dm, R, Cc, ro, co, scale = args
                for m0 in range(0, max(nsims, 1), 4):
                    use_y = Y is not None and m0 < nsims
                    check(self.lib.cf_qml_reduce_f64(
                        nb, R, Cc, Dm.data_ptr(), Dm.stride(0), Cc,
                        ptr(M) if m0 == 0 else None, n, ro, co,
                        _off(Y, m0) if use_y else None, nsims, min(4, nsims - m0) if use_y else 0,
                        ro, co, scale, _off(bias, s2 * nb) if (bias is not None and m0 == 0) else None,
                        _off(q, m0 * P + s2 * nb) if use_y else None, P, stream()), "cf_qml_reduce_f64")
            if not want_fisher:
                continue
            # ---- A_b slabs (and their transposes) for this spectrum
            XT = {}
            if "auto" in D:
                sa = blk.fa
                off, m = seg[sa]
                Xs = torch.empty((n, nb * m), dtype=F64, device=dev)
                XTs = torch.empty((nb * m, n), dtype=F64, device=dev)
                self.gemm(Cinv[:, off:off + m], D["auto"], C=Xs, CT=XTs, tag="a_gemm")
                X_slabs[(s2, sa)] = Xs
                XT[sa] = XTs
                cols_of[s2] = [sa]
            else:
                (oa, ma), (ob, mb) = seg[blk.fa], seg[blk.fb]
                Xa = torch.empty((n, nb * ma), dtype=F64, device=dev)
                XTa = torch.empty((nb * ma, n), dtype=F64, device=dev)
                self.gemm(Cinv[:, ob:ob + mb], D["ba"], C=Xa, CT=XTa, tag="a_gemm")
                Xb = torch.empty((n, nb * mb), dtype=F64, device=dev)
                XTb = torch.empty((nb * mb, n), dtype=F64, device=dev)
                self.gemm(Cinv[:, oa:oa + ma], D["ab"], C=Xb, CT=XTb, tag="a_gemm")
                X_slabs[(s2, blk.fa)] = Xa
                X_slabs[(s2, blk.fb)] = Xb
                XT[blk.fa] = XTa
                XT[blk.fb] = XTb
                cols_of[s2] = [blk.fa, blk.fb]
            del D
            # ---- Fisher traces of this spectrum against every spectrum so far
            for s1 in range(s2 + 1):
                for ss in cols_of[s1]:
                    s_off, m_s = seg[ss]
                    Xs = X_slabs[(s1, ss)]
                    for tt in cols_of[s2]:
                        t_off, m_t = seg[tt]
                        Yt = XT[tt]
                        check(self.lib.cf_trace_contract_f64(
                            nb, nb, m_t, m_s, _off(Xs, t_off * Xs.stride(0)), m_s, Xs.stride(0),
                            _off(Yt, s_off), m_t * n, n, 0.5, F.data_ptr(), P, s1 * nb, s2 * nb,
                            int(s1 != s2), 0, stream()), "cf_trace_contract_f64")
            del XT
        del X_slabs
        return F, bias, q

    # ------------------------------------------------------------------
    def potrf(self, A: torch.Tensor, keep_work: bool = False):
        """In-place lower Cholesky factor(s); info (and the workspace with the
        diagonal-block inverses when keep_work)."""
        n = A.shape[-1]
        B = A.shape[0] if A.dim() == 3 else 1
        info = torch.zeros(B, dtype=torch.int32, device=A.device)
        work = torch.empty(self.lib.cf_potrf_workspace(n, B) // 8 + 1, dtype=F64, device=A.device)
        check(self.lib.cf_potrf(n, A.data_ptr(), n, n * n, B, work.data_ptr(), info.data_ptr(), stream()),
              "cf_potrf")
        return (info, work) if keep_work else info

    def signal_basis(self, N: torch.Tensor) -> "SignalBasis":
        """The per-multipole basis of C(theta) for this layout and noise (cached on N)."""
        key = (N.data_ptr(), tuple(N.shape))
        if getattr(self, "_basis_key", None) != key:
            self._basis = None
            self._basis = SignalBasis(self, N)
            self._basis_key = key
        return self._basis

    def lnl(self, cl_tables, N: torch.Tensor, maps: torch.Tensor, noise_scale=None, precision: str = "fp64",
            build: str = "auto"):
        """chi2 (B x nsims), ln|C| (B,), lnL (B x nsims), info (B,) for a batch of points.

        precision "fp64": FP64 Cholesky, chi2 = |L^-1 x|^2, ln|C| from its
        diagonal.  "mixed": FP32 Cholesky of C, chi2 from one FP64 refinement
        step against C (second-order in the factor's error), ln|C| from the
        FP32 factor's diagonal summed in FP64.

        build "basis" forms the lower triangle of C(theta) = S(theta) + s N
        from the per-multipole basis (one FP64 GEMM per block region, see
        SignalBasis; for "mixed" the same epilogue writes the FP32 copy to
        factor), "direct" runs the pair kernel per point, "auto" takes the
        basis for batches of 64 or more points when it fits in 4 GB.
        "basis_tc" (mixed only) forms C in FP32 with BF16x6 split products on
        the tensor cores and refines against that FP32 C: the fastest form,
        but chi2 is then the FP32 C's (first order in its rounding: ~1e-7
        relative for maps drawn from C, up to ~1e-5 for maps far from it)
        instead of second order in the factor's error (1e-8).
        """
        if precision not in ("fp64", "mixed"):
            raise ValueError(f"precision must be 'fp64' or 'mixed', got {precision!r}")
        cl = torch.as_tensor(cl_tables, dtype=F64, device=self.dev)
        if cl.dim() == 2:
            cl = cl[None]
        B = cl.shape[0]
        n = self.L.n
        sc = None
        if noise_scale is not None:
            sc = torch.as_tensor(noise_scale, dtype=F64, device=self.dev).reshape(B).contiguous()
        if build == "auto":
            build = "basis" if B >= 64 and SignalBasis.bytes_needed(self.L) <= 4 << 30 else "direct"
        if build not in ("basis", "direct", "basis_tc"):
            raise ValueError(f"build must be 'auto', 'basis', 'direct' or 'basis_tc', got {build!r}")
        if build == "basis_tc":
            if precision != "mixed":
                raise ValueError("build 'basis_tc' forms C in FP32: it serves precision 'mixed' only")
            return self._lnl_mixed_basis_tc(self.signal_basis(N), cl, maps, sc)
        if build == "basis":
            # lower triangles only: the factors and the chi2 kernels read nothing else
            if precision == "mixed":
                C32 = torch.empty((B, n, n), dtype=torch.float32, device=self.dev)
                C = self.signal_basis(N).covariance(cl, sc, lower=True, out32=C32)
                return self._lnl_mixed(C, N, maps, sc, C32=C32)
            C = self.signal_basis(N).covariance(cl, sc, lower=True)
        else:
            C = self.signal(cl)
            if precision == "mixed":
                return self._lnl_mixed(C, N, maps, sc)
            check(self.lib.cf_axpby(n * n, 1.0, C.data_ptr(), n * n, 1.0, ptr(sc), N.data_ptr(), 0,
                                    C.data_ptr(), n * n, B, stream()), "cf_axpby")
        info, work = self.potrf(C, keep_work=True)
        X = maps.to(self.dev, F64).contiguous()
        nsims = X.shape[1]
        chi2 = torch.empty((B, nsims), dtype=F64, device=self.dev)
        logdet = torch.empty(B, dtype=F64, device=self.dev)
        if n <= 24576 - 64:
            # 64-row blocks solved with the factor's diagonal-block inverses
            check(self.lib.cf_chi2_logdet_dinv(n, C.data_ptr(), n, n * n, work.data_ptr(),
                                               self.lib.cf_potrf_dinv_stride(n), B, X.data_ptr(), nsims, 0, nsims,
                                               chi2.data_ptr(), logdet.data_ptr(), stream()), "cf_chi2_logdet_dinv")
        else:
            z = torch.empty((B * nsims, n), dtype=F64, device=self.dev)
            check(self.lib.cf_chi2_logdet(n, C.data_ptr(), n, n * n, B, X.data_ptr(), nsims, 0, nsims,
                                          z.data_ptr(), chi2.data_ptr(), logdet.data_ptr(), stream()),
                  "cf_chi2_logdet")
        return chi2, logdet, -0.5 * (chi2 + logdet[:, None]), info

    def _lnl_mixed_basis_tc(self, basis: "SignalBasis", cl: torch.Tensor, maps: torch.Tensor, sc):
        """Mixed likelihood with C(theta) built in FP32 on the tensor cores: two
        copies from one pass (one is factored in place, the other feeds the
        FP64 refinement arithmetic), FP32 Cholesky, refined chi2 and ln|C|."""
        B, n = cl.shape[0], self.L.n
        C32 = torch.empty((B, n, n), dtype=torch.float32, device=self.dev)
        L32 = torch.empty_like(C32)
        err = basis.covariance_f32(cl, sc, C32, L32)
        info = torch.zeros(B, dtype=torch.int32, device=self.dev)
        work = torch.empty(self.lib.cf_potrf_f32_workspace(n, B) // 4 + 1, dtype=torch.float32, device=self.dev)
        check(self.lib.cf_potrf_f32(n, L32.data_ptr(), n, n * n, B, work.data_ptr(), info.data_ptr(), stream()),
              "cf_potrf_f32")
        X = maps.to(self.dev, F64).contiguous()
        nsims = X.shape[1]
        chi2 = torch.empty((B, nsims), dtype=F64, device=self.dev)
        logdet = torch.empty(B, dtype=F64, device=self.dev)
        check(self.lib.cf_chi2_logdet_mixed_c32_dinv(n, L32.data_ptr(), n, n * n, work.data_ptr(),
                                                     self.lib.cf_potrf_f32_dinv_stride(n), C32.data_ptr(), n, n * n,
                                                     B, X.data_ptr(), nsims, 0, nsims, chi2.data_ptr(),
                                                     logdet.data_ptr(), stream()), "cf_chi2_logdet_mixed_c32_dinv")
        # a tensor-core wait that ran out marks every point of the batch (no host sync: capturable)
        info = torch.where(err[0] != 0, torch.full_like(info, CF_ERR_TIMEOUT), info)
        return chi2, logdet, -0.5 * (chi2 + logdet[:, None]), info

    def _lnl_mixed(self, C: torch.Tensor, N: torch.Tensor, maps: torch.Tensor, sc, C32: torch.Tensor | None = None):
        """C holds S (C32 None: the noise is added here, with the FP32 copy) or
        S + s N with its FP32 copy already in C32."""
        B, n = C.shape[0], self.L.n
        if C32 is None:
            C32 = torch.empty((B, n, n), dtype=torch.float32, device=self.dev)
            check(self.lib.cf_axpby_f32(n * n, 1.0, C.data_ptr(), n * n, 1.0, ptr(sc), N.data_ptr(), 0,
                                        C.data_ptr(), n * n, C32.data_ptr(), n * n, B, stream()), "cf_axpby_f32")
        info = torch.zeros(B, dtype=torch.int32, device=self.dev)
        work = torch.empty(self.lib.cf_potrf_f32_workspace(n, B) // 4 + 1, dtype=torch.float32, device=self.dev)
        check(self.lib.cf_potrf_f32(n, C32.data_ptr(), n, n * n, B, work.data_ptr(), info.data_ptr(), stream()),
              "cf_potrf_f32")
        X = maps.to(self.dev, F64).contiguous()
        nsims = X.shape[1]
        chi2 = torch.empty((B, nsims), dtype=F64, device=self.dev)
        logdet = torch.empty(B, dtype=F64, device=self.dev)
        check(self.lib.cf_chi2_logdet_mixed_dinv(n, C32.data_ptr(), n, n * n, work.data_ptr(),
                                                 self.lib.cf_potrf_f32_dinv_stride(n), C.data_ptr(), n, n * n, B,
                                                 X.data_ptr(), nsims, 0, nsims, chi2.data_ptr(), logdet.data_ptr(),
                                                 stream()), "cf_chi2_logdet_mixed_dinv")
        return chi2, logdet, -0.5 * (chi2 + logdet[:, None]), info


class SignalBasis:
    """C(theta) = S(theta) + s(theta) N for many points as one FP64 GEMM per block region.

    The pair kernels (Legendre / spin-2 recurrences, rotation angles) do not
    depend on the spectra: S = sum_{k, l} C~_{k,l} K_{k,l}, with K_{k,l} the
    signal matrix of a unit table at (spectrum k, multipole l)
    (``cosmocore/signal_kernels.py:164-502`` evaluated once per basis entry by
    the pair kernel).  Each block region of C (a field pair and its mirror) is
    then (points x kdim) . (kdim x region entries): the rows of the basis are
    the region of N (weighted by the point's noise scale) followed by the
    K_{k,l} of the region's spectra, spectrum-major.  Trailing spectra whose
    tables are zero for every point of a batch (TB, EB in a model without
    them) are left out of the product.  Rounding differs from the direct build
    only in the order of the l sum.
    """

    def __init__(self, E: "Engine", N: torch.Tensor):
        L = E.L
        n, Lp = L.n, L.lmax_signal + 1
        self.E, self.n, self.Lp = E, n, Lp
        self.regions = []
        covered = 0
        for blk in L.blocks:
            fa, fb = L.fields[blk.fa], L.fields[blk.fb]
            by_mode = {L.spectra[k].mode: k for k in blk.spectra}
            if blk.kind in (lay.KIND_00_AUTO, lay.KIND_00_CROSS):
                sp = [blk.spectra[0]]
            elif blk.kind == lay.KIND_22_AUTO:
                sp = [by_mode[m] for m in (0, 1, 2) if m in by_mode]
            else:
                sp = [by_mode[m] for m in (0, 1) if m in by_mode]
            spans = [(fb.offset, fa.offset, fb.nrows, fa.nrows)]
            if blk.fa != blk.fb:
                spans.append((fa.offset, fb.offset, fa.nrows, fb.nrows))
            Ks = [torch.empty((1 + len(sp) * Lp, R, Cc), dtype=F64, device=E.dev) for (_, _, R, Cc) in spans]
            for (r0, c0, R, Cc), K in zip(spans, Ks):
                K[0] = N[r0:r0 + R, c0:c0 + Cc]
            for j, k in enumerate(sp):
                tab = torch.zeros((Lp, L.nspectra, Lp), dtype=F64, device=E.dev)
                tab[torch.arange(Lp), k, torch.arange(Lp)] = 1.0
                Sk = E.signal(tab)
                for (r0, c0, R, Cc), K in zip(spans, Ks):
                    K[1 + j * Lp: 1 + (j + 1) * Lp] = Sk[:, r0:r0 + R, c0:c0 + Cc]
                del Sk
            sp_dev = torch.tensor(sp, dtype=torch.long, device=E.dev)
            for (r0, c0, R, Cc), K in zip(spans, Ks):
                self.regions.append((r0, c0, R, Cc, sp, sp_dev, K))
                covered += R * Cc
        if covered != n * n:
            raise ValueError("the blocks of this layout do not cover the covariance matrix")
        self._kplanes = None

    @staticmethod
    def bytes_needed(L) -> int:
        Lp = L.lmax_signal + 1
        tot = 0
        for blk in L.blocks:
            fa, fb = L.fields[blk.fa], L.fields[blk.fb]
            k = 1 + len(blk.spectra) * Lp
            tot += k * fa.nrows * fb.nrows * (1 if blk.fa == blk.fb else 2)
        return 8 * tot

    def covariance(self, cl: torch.Tensor, scale: torch.Tensor | None = None, out=None, lower: bool = False,
                   out32: torch.Tensor | None = None) -> torch.Tensor:
        """C (B x n x n, FP64) for beam-smoothed tables cl (B, nspectra, L+1).

        lower: only the lower triangle is formed (the mirror span of each
        off-diagonal block is left out, the diagonal blocks skip the tiles
        right of their rows; entries above the diagonal are left unset or
        partly filled).  out32: an FP32 copy written by the same GEMM
        epilogue."""
        E, n, Lp = self.E, self.n, self.Lp
        B = cl.shape[0]
        if out is None:
            out = torch.empty((B, n, n), dtype=F64, device=E.dev)
        s = torch.ones(B, dtype=F64, device=E.dev) if scale is None else scale.reshape(B).to(F64)
        # leaving out the trailing all-zero spectra drops exact zeros from every
        # sum (same bits); while a CUDA graph is being captured the host cannot
        # read the tables, so every spectrum stays in
        used = None
        if not torch.cuda.is_current_stream_capturing():
            used = (cl.abs().amax(dim=(0, 2)) > 0).cpu().numpy()
        for r0, c0, R, Cc, sp, sp_dev, K in self.regions:
            if lower and r0 < c0:
                continue  # the mirror span of an off-diagonal block lies above the diagonal
            keep = len(sp)
            while used is not None and keep > 0 and not used[sp[keep - 1]]:
                keep -= 1
            kd = 1 + keep * Lp
            # spectra picked with a device index (no host-to-device copy: capturable)
            ctab = torch.cat([s[:, None], cl.index_select(1, sp_dev[:keep]).reshape(B, keep * Lp)],
                             dim=1).contiguous()
            # batch entry = region row; bit 3 skips the tiles right of the row on a diagonal block
            lo = 8 if (lower and r0 == c0) else 0
            off = r0 * n + c0
            if out32 is None:
                check(self.E.lib.cf_dgemm(0, 0, B, Cc, kd, 1.0, ctab.data_ptr(), kd, 0, K.data_ptr(), R * Cc, Cc,
                                          0.0, _off(out, off), n * n, n, None, 0, 0, R, lo, stream()), "cf_dgemm")
            else:
                check(self.E.lib.cf_dgemm_f32copy(0, 0, B, Cc, kd, 1.0, ctab.data_ptr(), kd, 0, K.data_ptr(), R * Cc,
                                                  Cc, 0.0, _off(out, off), n * n, n, _off(out32, off), n * n, n, R,
                                                  lo, stream()), "cf_dgemm_f32copy")
        return out

    def _planes(self):
        """BF16x3 split planes of every region's basis, entries x kdim (K
        contiguous, padded to a multiple of 8), built on first use."""
        if self._kplanes is None:
            E = self.E
            out = []
            for r0, c0, R, Cc, sp, sp_dev, K in self.regions:
                kd = K.shape[0]
                kp = (kd + 7) // 8 * 8
                Kt = K.reshape(kd, R * Cc).t().contiguous()
                P = torch.zeros((3, R * Cc, kp), dtype=torch.bfloat16, device=E.dev)
                check(E.lib.cf_split_bf16(R * Cc, kd, Kt.data_ptr(), kd, 3, P.data_ptr(), kp, R * Cc * kp,
                                          stream()), "cf_split_bf16")
                del Kt
                out.append((P, kp))
            self._kplanes = out
        return self._kplanes

    def covariance_f32(self, cl: torch.Tensor, scale: torch.Tensor | None, out: torch.Tensor,
                       out2: torch.Tensor | None = None) -> torch.Tensor:
        """C (B x n x n) in FP32 into `out` (and `out2`) from BF16x6 split
        products on the tensor cores: per region, (region entries x kdim) times
        (points x kdim)^T, written transposed into the points' matrices
        (cf_umma_gemm_bf16_scatter).  Returns the device error flag of the
        launches (non-zero: a bounded wait ran out)."""
        E, n, Lp = self.E, self.n, self.Lp
        B = cl.shape[0]
        s = torch.ones(B, dtype=F64, device=E.dev) if scale is None else scale.reshape(B).to(F64)
        used = None
        if not torch.cuda.is_current_stream_capturing():
            used = (cl.abs().amax(dim=(0, 2)) > 0).cpu().numpy()
        err = torch.zeros(1, dtype=torch.int32, device=E.dev)
        ta, tb = _X6_TERMS
        for (r0, c0, R, Cc, sp, sp_dev, K), (P, kp) in zip(self.regions, self._planes()):
            keep = len(sp)
            while used is not None and keep > 0 and not used[sp[keep - 1]]:
                keep -= 1
            kd = 1 + keep * Lp
            ctab = torch.zeros((B, kp), dtype=F64, device=E.dev)
            ctab[:, 0] = s
            ctab[:, 1:kd] = cl.index_select(1, sp_dev[:keep]).reshape(B, keep * Lp)
            cp = torch.empty((3, B, kp), dtype=torch.bfloat16, device=E.dev)
            check(E.lib.cf_split_bf16(B, kp, ctab.data_ptr(), kp, 3, cp.data_ptr(), kp, B * kp, stream()),
                  "cf_split_bf16")
            off = r0 * n + c0
            check(E.lib.cf_umma_gemm_bf16_scatter(R * Cc, B, kd, 6, ta, tb, P.data_ptr(), kp, R * Cc * kp, 3,
                                                  cp.data_ptr(), kp, B * kp, 3, _off(out, off),
                                                  _off(out2, off) if out2 is not None else None, n * n, Cc, n,
                                                  err.data_ptr(), stream()), "cf_umma_gemm_bf16_scatter")
        return err


class LnlGraph:
    """The likelihood of a batch of B points as one CUDA graph replay.

    Static device buffers hold the points' beam-smoothed tables and noise
    scales; the graph records Engine.lnl on them once (C(theta) from the
    per-multipole basis or the pair kernel, the Cholesky factor, chi2 and
    ln|C|), and every later batch is a copy of its tables into the buffers
    and one replay (picslike/picslike.py:479-546 run as one launch per batch).
    A batch smaller than B fills the tail of the buffers with copies of its
    first point and drops their results.
    """

    def __init__(self, E: Engine, N: torch.Tensor, X: torch.Tensor, B: int, precision: str = "fp64",
                 build: str = "auto"):
        L = E.L
        self.E, self.B = E, int(B)
        self.cl = torch.zeros((self.B, L.nspectra, L.lmax_signal + 1), dtype=F64, device=E.dev)
        self.sc = torch.ones(self.B, dtype=F64, device=E.dev)
        self.N = N
        self.X = X.to(E.dev, F64).contiguous()
        self.precision = precision
        self.build = "basis" if (build == "auto" and self.B >= 64
                                 and SignalBasis.bytes_needed(L) <= 4 << 30) else ("direct" if build == "auto"
                                                                                     else build)
        # eager warm-up (kernel attributes, the basis, library module loads), then the capture
        E.lnl(self.cl, N, self.X, noise_scale=self.sc, precision=precision, build=self.build)
        torch.cuda.synchronize(E.dev)
        self.graph = torch.cuda.CUDAGraph()
        with torch.cuda.graph(self.graph):
            self.out = E.lnl(self.cl, N, self.X, noise_scale=self.sc, precision=precision, build=self.build)

    def __call__(self, cl, noise_scale=None):
        """chi2 (b, nsims), ln|C| (b,), lnL (b, nsims), info (b,) for b <= B points."""
        cl = torch.as_tensor(cl, dtype=F64, device=self.E.dev)
        b = cl.shape[0]
        if b > self.B:
            raise ValueError(f"batch of {b} points exceeds the graph's {self.B}")
        self.cl[:b].copy_(cl)
        if b < self.B:
            self.cl[b:].copy_(cl[:1].expand(self.B - b, -1, -1))
        if noise_scale is None:
            self.sc.fill_(1.0)
        else:
            sc = torch.as_tensor(noise_scale, dtype=F64, device=self.E.dev).reshape(b)
            self.sc[:b].copy_(sc)
            self.sc[b:].copy_(sc[:1].expand(self.B - b))
        self.graph.replay()
        chi2, logdet, lnl, info = self.out
        return chi2[:b].clone(), logdet[:b].clone(), lnl[:b].clone(), info[:b].clone()


def qml_solve(E: Engine, cls: dict, N: torch.Tensor, maps: torch.Tensor):
    """S, C^-1, F, q, bias, F^-1, C_hat on the device (plain FP64)."""
    L = E.L
    S = E.signal(L.smoothed_cl_table(cls))
    Cinv = S + N
    E.spd_inverse(Cinv)
    F, bias, q = E.fisher_qml(Cinv, N, maps)
    Finv = E.spd_inverse(F.clone())
    if L.remove_nb:
        q = q - bias[None, :]
    return dict(S=S, Cinv=Cinv, fisher=F, q=q, bias=bias, invfisher=Finv,
                clhat=E.gemm(q, Finv), noise_bias=E.gemm(bias[None, :], Finv)[0])
