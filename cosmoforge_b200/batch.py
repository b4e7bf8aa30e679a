"""Batched QML: many maps against one covariance, many small problems at once.

* :func:`map_solves` - raw quadratic forms q_b(m) = 1/2 y_m^T dC_b y_m,
  y = C^-1 x_m, for thousands of maps given one C^-1 (qube/spectra.py:
  1124-1186 with nsims large).  Per spectrum one GEMM W = D^T Y against the
  stacked derivative blocks of all its bins, then a per-(bin, map) reduction
  (``cf_qform_reduce_*``).  ``precision="mixed"`` runs every product on the
  BF16 split-product tensor-core kernel (CTA-pair form): Y = C^-1 X first,
  whose epilogue writes Y in FP32 for the reductions and the split planes of
  Y^T for the per-spectrum GEMMs, then W against the derivative planes
  emitted by the pair builder (q within 1e-5 of max |q| of the FP64 path).
* :class:`PatchBatch` - many independent spin-0 QML problems of uneven size
  (sky patches) solved together: the problems are grouped by size into
  buckets, every problem of a bucket is padded to the bucket's order with an
  identity noise block (zero signal, zero derivatives, zero map entries, so F,
  q and the bias are unchanged), then the factorisations, the A_b products,
  the Fisher contractions and the quadratic forms run as batched device
  kernels, and the whole pipeline replays from one CUDA graph.
"""

from __future__ import annotations

import numpy as np
import torch

from . import engine as eng
from . import layout as lay
from ._lib import check, lib, stream
from .engine import _off
from .engine_mixed import MixedPlan, _build_planes, _r8

F64 = torch.float64


def _ptr(t, off=0):
    return t.data_ptr() + off * t.element_size()


def _ptr16(t: torch.Tensor, elems: int) -> int:
    return t.data_ptr() + int(elems) * t.element_size()


def map_solves(E: eng.Engine, Cinv: torch.Tensor, X: torch.Tensor, precision: str = "fp64",
               scheme: str = "bf16x6") -> torch.Tensor:
    """Raw q (nmaps x P) for the maps in the columns of X (n x nmaps), no bias removed."""
    L = E.L
    n, nb, P = L.n, L.nbins, L.n_params
    X = X.to(E.dev, F64).contiguous()
    m = X.shape[1]
    q = torch.zeros((m, P), dtype=F64, device=E.dev)
    st = stream()
    if precision == "fp64":
        Y = E.gemm(Cinv, X)
        for s in range(L.nspectra):
            blk, D = E._deriv_blocks(s)
            fa, fb = L.fields[blk.fa], L.fields[blk.fb]
            if "auto" in D:
                mm = fa.nrows
                W = E.gemm(D["auto"], Y[fa.offset: fa.offset + mm], transa=True)
                check(E.lib.cf_qform_reduce_f64(nb, mm, mm, W.data_ptr(), m, Y.data_ptr(), m, fa.offset, m, 0.5,
                                                q.data_ptr(), P, s * nb, st), "cf_qform_reduce_f64")
            else:
                R, Cc = fb.nrows, fa.nrows
                W = E.gemm(D["ba"], Y[fb.offset: fb.offset + R], transa=True)
                check(E.lib.cf_qform_reduce_f64(nb, Cc, Cc, W.data_ptr(), m, Y.data_ptr(), m, fa.offset, m, 1.0,
                                                q.data_ptr(), P, s * nb, st), "cf_qform_reduce_f64")
            del D
        return q
    if precision != "mixed":
        raise ValueError(f"precision must be 'fp64' or 'mixed', got {precision!r}")
    plan = MixedPlan(E, scheme)
    Pl, npd = plan.planes, plan.n_pad
    # Y = C^-1 X as a split-product GEMM too (fields padded to multiples of 8):
    # its epilogue writes Y in FP32 (for the reductions) and the split planes of
    # Y^T that the per-spectrum GEMMs read, so no FP64 GEMM, transpose or split
    Cp = plan.split_cinv(Cinv)
    Xt = plan.pad_rows(X).t().contiguous()  # m x npd
    Xtp = torch.zeros((Pl, m, npd), dtype=torch.bfloat16, device=E.dev)
    check(E.lib.cf_split_bf16(m, npd, Xt.data_ptr(), npd, Pl, Xtp.data_ptr(), npd, m * npd, st), "cf_split_bf16")
    del Xt
    YTp = torch.zeros((Pl, m, npd), dtype=torch.bfloat16, device=E.dev)
    Y32 = torch.empty((npd, m), dtype=torch.float32, device=E.dev)
    # all planes per stage on CTA pairs (the split-product GEMM's fastest form here)
    prev_form = E.lib.cf_umma_set_all_planes(2)
    try:
        check(E.lib.cf_umma_gemm_bf16(npd, m, npd, plan.nterms, plan.ta, plan.tb, Cp.data_ptr(), npd, npd * npd, Pl,
                                      Xtp.data_ptr(), npd, m * npd, Pl, None, 0, 0, Pl, YTp.data_ptr(), npd, m * npd,
                                      Y32.data_ptr(), m, plan.err.data_ptr(), st), "cf_umma_gemm_bf16")
        del Cp, Xtp
        Ypad = Y32.double()
        del Y32
        Ytp = {fi: (_ptr16(YTp, plan.po[fi]), npd, m * npd) for fi in range(len(L.fields))}
        _map_solve_spectra(E, L, plan, Ytp, Ypad, q, m, nb, P, st)
    finally:
        E.lib.cf_umma_set_all_planes(prev_form)
    check(E.lib.cf_umma_status(plan.err.data_ptr(), stream()), "tensor-core kernel")
    return q


def _map_solve_spectra(E, L, plan, Ytp, Y, q, m, nb, P, st):
    """q_b += 1/2 y^T dC_b y for every bin: per spectrum and column segment, the
    split-product GEMM W = dC_b-planes . Y^T-planes and the q reduction (Y in
    the plan's padded field layout; Ytp[field] = (pointer, row stride, plane
    stride) of that field's columns of the Y^T planes)."""
    Pl = plan.planes
    for s in range(L.nspectra):
        blk, ops = _build_planes(plan, s)
        for seg, (B, K, kseg) in ops.items():
            M, ld = B.shape[1], B.shape[2]
            rpb = M // nb
            W = torch.empty((M, m), dtype=torch.float32, device=E.dev)
            yk, ldk, psk = Ytp[kseg]
            check(E.lib.cf_umma_gemm_bf16(M, m, K, plan.nterms, plan.ta, plan.tb, B.data_ptr(), ld, M * ld, Pl,
                                          yk, ldk, psk, Pl, None, 0, 0, 0, None, 0,
                                          0, W.data_ptr(), m, plan.err.data_ptr(), st), "cf_umma_gemm_bf16")
            f = L.fields[seg]
            # Y rows in the padded field layout of the plan
            check(E.lib.cf_qform_reduce_f32(nb, f.nrows, rpb, W.data_ptr(), m, Y.data_ptr(), m, plan.po[seg], m,
                                            0.5, q.data_ptr(), P, s * nb, st), "cf_qform_reduce_f32")
            del W
        del ops


class _PatchGroup:
    """Spin-0 QML problems padded to the largest of them and solved as one batch."""

    def __init__(self, problems, device=None):
        self.dev = torch.device(device or "cuda")
        self.lib = lib()
        self.P = len(problems)
        self.layouts = [lay.build_layout(p["params"], p["mask"], p["beam"]) for p in problems]
        for L in self.layouts:
            if L.nspectra != 1 or L.blocks[0].kind != lay.KIND_00_AUTO:
                raise NotImplementedError("PatchBatch handles single-field spin-0 (TT) problems")
        self.engines = [eng.Engine(L, self.dev) for L in self.layouts]
        self.nb = self.layouts[0].nbins
        if any(L.nbins != self.nb for L in self.layouts):
            raise ValueError("all problems must share the same bins")
        self.ns = [L.n for L in self.layouts]
        self.n_pad = _r8(max(self.ns))
        self.nsims = int(problems[0]["maps"].shape[1])
        if self.nsims > 4 or any(int(p["maps"].shape[1]) != self.nsims for p in problems):
            raise ValueError("every problem needs the same number of maps, at most 4")
        P, nb, npd, ms = self.P, self.nb, self.n_pad, self.nsims
        z = lambda *s: torch.zeros(s, dtype=F64, device=self.dev)  # noqa: E731
        self.tables = [torch.as_tensor(L.smoothed_cl_table(p["cls"]), dtype=F64, device=self.dev).contiguous()
                       for L, p in zip(self.layouts, problems)]
        Nfull = np.zeros((P, npd, npd))
        Xfull = np.zeros((P, npd, ms))
        for k, (L, p) in enumerate(zip(self.layouts, problems)):
            n = L.n
            Nfull[k, :n, :n] = np.asarray(p["noise"], np.float64)
            Nfull[k, n:, n:] = np.eye(npd - n)
            Xfull[k, :n] = np.asarray(p["maps"], np.float64)
        self.N = torch.from_numpy(Nfull).to(self.dev)
        self.X = torch.from_numpy(Xfull).to(self.dev)
        self.C = z(P, npd, npd)
        self.dC = z(P, nb, npd, npd)
        self.A = z(P, nb, npd, npd)
        self.AT = z(P, nb, npd, npd)
        self.T = z(P, npd, npd)
        self.M = z(P, npd, npd)
        self.Y = z(P, npd, ms)
        self.F = z(P, nb, nb)
        self.Finv = z(P, nb, nb)
        self.q = z(P, ms, nb)
        self.bias = z(P, nb)
        self.qmb = z(P, ms, nb)
        self.clhat = z(P, ms, nb)
        self.info_c = torch.zeros(P, dtype=torch.int32, device=self.dev)
        self.info_f = torch.zeros(P, dtype=torch.int32, device=self.dev)
        self.work_c = torch.empty(self.lib.cf_spd_inverse_workspace(npd, P) // 8 + 1, dtype=F64, device=self.dev)
        self.work_f = torch.empty(self.lib.cf_spd_inverse_workspace(nb, P) // 8 + 1, dtype=F64, device=self.dev)
        self._graph = None

    def _dgemm(self, ta, tb, M, N, K, A, lda, sA, B, ldb, sB, C, ldc, sC, batch, beta=0.0, CT=None, ldct=0,
               sCT=0):
        check(self.lib.cf_dgemm(ta, tb, M, N, K, 1.0, A, lda, sA, B, ldb, sB, beta, C, ldc, sC, CT, ldct, sCT,
                                batch, 0, stream()), "cf_dgemm")

    def _pipeline(self):
        P, nb, npd, ms = self.P, self.nb, self.n_pad, self.nsims
        st = stream()
        lib = self.lib
        nn = npd * npd
        self.C.zero_()
        self.dC.zero_()
        for k, (E, L) in enumerate(zip(self.engines, self.layouts)):
            blk = L.blocks[0]
            Cp = _ptr(self.C, k * nn)
            E._launch_block(blk, -1, [self.tables[k].data_ptr()], None, Cp, npd, 0, 0, 0, Cp, npd, 0, 0, 0)
            Dp = _ptr(self.dC, k * nb * nn)
            E._launch_block(blk, L.spectra[0].mode, [_off(E.deriv_tab, 0)], _off(E.deriv_bin, 0), Dp, npd, 0, 0,
                            nn, Dp, npd, 0, 0, nn)
        check(lib.cf_axpby(nn, 1.0, self.C.data_ptr(), nn, 1.0, None, self.N.data_ptr(), nn, self.C.data_ptr(), nn,
                           P, st), "cf_axpby")
        self.info_c.zero_()
        check(lib.cf_spd_inverse(npd, self.C.data_ptr(), npd, nn, P, self.work_c.data_ptr(), self.info_c.data_ptr(),
                                 st), "cf_spd_inverse")
        Ci = self.C  # now C^-1 (identity block in the padding)
        # M = C^-1 N C^-1, Y = C^-1 X (batched over problems)
        self._dgemm(0, 0, npd, npd, npd, self.N.data_ptr(), npd, nn, Ci.data_ptr(), npd, nn, self.T.data_ptr(),
                    npd, nn, P)
        self._dgemm(0, 0, npd, npd, npd, Ci.data_ptr(), npd, nn, self.T.data_ptr(), npd, nn, self.M.data_ptr(),
                    npd, nn, P)
        self._dgemm(0, 0, npd, ms, npd, Ci.data_ptr(), npd, nn, self.X.data_ptr(), ms, npd * ms,
                    self.Y.data_ptr(), ms, npd * ms, P)
        self.F.zero_()
        self.q.zero_()
        self.bias.zero_()
        for k, n in enumerate(self.ns):
            # A_b = C^-1 dC_b and A_b^T for every bin of problem k
            self._dgemm(0, 0, n, n, n, _ptr(Ci, k * nn), npd, 0, _ptr(self.dC, k * nb * nn), npd, nn,
                        _ptr(self.A, k * nb * nn), npd, nn, nb, CT=_ptr(self.AT, k * nb * nn), ldct=npd, sCT=nn)
            check(lib.cf_trace_contract_f64(nb, nb, n, n, _ptr(self.A, k * nb * nn), nn, npd,
                                            _ptr(self.AT, k * nb * nn), nn, npd, 0.5, _ptr(self.F, k * nb * nb), nb,
                                            0, 0, 0, 0, st), "cf_trace_contract_f64")
            check(lib.cf_qml_reduce_f64(nb, n, n, _ptr(self.dC, k * nb * nn), npd, nn, _ptr(self.M, k * nn), npd,
                                        0, 0, _ptr(self.Y, k * npd * ms), ms, ms, 0, 0, 0.5,
                                        _ptr(self.bias, k * nb), _ptr(self.q, k * ms * nb), nb, st),
                  "cf_qml_reduce_f64")
        # C_hat = (q - b) F^-1
        self.Finv.copy_(self.F)
        self.info_f.zero_()
        check(lib.cf_spd_inverse(nb, self.Finv.data_ptr(), nb, nb * nb, P, self.work_f.data_ptr(),
                                 self.info_f.data_ptr(), st), "cf_spd_inverse")
        for j in range(ms):
            check(lib.cf_axpby(nb, 1.0, _ptr(self.q, j * nb), ms * nb, -1.0, None, self.bias.data_ptr(), nb,
                               _ptr(self.qmb, j * nb), ms * nb, P, st), "cf_axpby")
        self._dgemm(0, 0, ms, nb, nb, self.qmb.data_ptr(), nb, ms * nb, self.Finv.data_ptr(), nb, nb * nb,
                    self.clhat.data_ptr(), nb, ms * nb, P)

    def results(self):
        """Per-problem dict of numpy arrays: fisher, q (raw), bias, clhat, info flags."""
        F, q, b, ch = (t.cpu().numpy() for t in (self.F, self.q, self.bias, self.clhat))
        ic, jf = self.info_c.cpu().numpy(), self.info_f.cpu().numpy()
        out = []
        for k in range(self.P):
            out.append(dict(fisher=F[k], q=q[k], bias=b[k], clhat=ch[k], n=self.ns[k], info_cov=int(ic[k]),
                            info_fisher=int(jf[k])))
        return out


def bucket_bounds(ns, buckets: int) -> list:
    """Split problems sorted by size into at most `buckets` contiguous groups
    minimising the padded work sum_g |g| max_g(n)^3 (exact, by dynamic
    programming over the sorted sizes); returns the groups' end indices."""
    ns = sorted(int(n) for n in ns)
    P = len(ns)
    k = max(1, min(int(buckets), P))
    INF = float("inf")
    best = [[INF] * (P + 1) for _ in range(k + 1)]
    cut = [[0] * (P + 1) for _ in range(k + 1)]
    best[0][0] = 0.0
    for g in range(1, k + 1):
        for j in range(1, P + 1):
            for i in range(g - 1, j):
                c = best[g - 1][i] + (j - i) * float(ns[j - 1]) ** 3
                if c < best[g][j]:
                    best[g][j], cut[g][j] = c, i
    g = min(range(1, k + 1), key=lambda q: best[q][P])
    ends, j = [], P
    while g > 0:
        ends.append(j)
        j = cut[g][j]
        g -= 1
    return sorted(ends)


class PatchBatch:
    """Independent spin-0 QML problems of uneven size (sky patches) solved together.

    problems: list of dicts with ``params``, ``mask`` (npix x 1), ``beam``,
    ``cls`` ({"TT": C_l}), ``noise`` (n x n reduced noise covariance) and
    ``maps`` (n x nsims, nsims <= 4).  All problems must share lmin / lmax /
    lmax_signal (the same bins).  The problems are sorted by size and split
    into ``buckets`` groups (boundaries minimising the padded n^3 work), each
    padded to its own largest problem; every group's pipeline runs as batched
    kernels and all of them replay from one CUDA graph.  ``buckets=None``
    takes the count the autotuner picked for this set of sizes (cached), or 1.
    """

    def __init__(self, problems, device=None, buckets: int | None = None):
        self.dev = torch.device(device or "cuda")
        sizes = [int((np.asarray(p["mask"]) > 0.5).sum()) for p in problems]
        if buckets is None:
            from .autotune import patch_buckets_for

            buckets = patch_buckets_for(sizes, self.dev)
        order = sorted(range(len(problems)), key=lambda k: sizes[k])
        ends = bucket_bounds(sizes, buckets)
        self.groups, self.members = [], []
        start = 0
        for e in ends:
            idx = order[start:e]
            self.groups.append(_PatchGroup([problems[k] for k in idx], self.dev))
            self.members.append(idx)
            start = e
        self.buckets = len(self.groups)
        self.P = len(problems)
        self.nb = self.groups[0].nb
        if any(g.nb != self.nb for g in self.groups):
            raise ValueError("all problems must share the same bins")
        self.ns = [0] * self.P
        for g, idx in zip(self.groups, self.members):
            for k, n in zip(idx, g.ns):
                self.ns[k] = n
        self._graph = None

    @property
    def info_f(self) -> torch.Tensor:
        out = torch.zeros(self.P, dtype=torch.int32, device=self.dev)
        for g, idx in zip(self.groups, self.members):
            out[torch.as_tensor(idx, device=self.dev)] = g.info_f
        return out

    def _pipeline(self):
        for g in self.groups:
            g._pipeline()

    def run(self, graph: bool = True):
        """Solve every problem (replays one captured pipeline after the first call)."""
        if self._graph is not None:
            self._graph.replay()
        else:
            self._pipeline()
            if graph:
                g = torch.cuda.CUDAGraph()
                with torch.cuda.graph(g):
                    self._pipeline()
                self._graph = g
        return self

    def results(self):
        """Per-problem dict of numpy arrays (input order): fisher, q (raw), bias, clhat, info flags."""
        out = [None] * self.P
        for g, idx in zip(self.groups, self.members):
            for k, r in zip(idx, g.results()):
                out[k] = r
        return out
