"""Mixed-precision Fisher on the tensor cores (tcgen05 BF16 split products).

Same algebra as ``engine.Engine.fisher_qml`` (``qube/fisher.py:501-607``), with
the two O(P n^3) / O(P^2 n^2) stages moved to the 5th-generation tensor
cores:

* C^-1 (FP64, from the Jacobi-scaled Cholesky inverse) is split into BF16
  planes c = c_0 + c_1 (+ c_2); the derivative blocks of one spectrum are
  emitted by the pair builder directly as BF16 planes (FP64 recurrences,
  split at the store);
* A_b = C^-1 dC_b runs as the split-product GEMM ``cf_umma_gemm_bf16``
  (FP32 accumulation in TMEM) whose epilogue writes A_b, and A_b^T, as two
  BF16 planes (16 significant bits);
* the traces F_pq = 1/2 sum_{k,l} A_p[k,l] A_q[l,k] run as the tensor-core
  contraction ``cf_umma_trace_bf16`` over the flattened (k, l) plane with the
  products (0,0), (0,1), (1,0), (1,1) of those planes, partial sums added
  into an FP64 F.

Schemes: ``bf16x3`` = planes {(0,0), (0,1), (1,0)} (~16 bits per product),
``bf16x6`` adds {(0,2), (1,1), (2,0)} (~24 bits).  The noise bias and the
quadratic forms come out of the same traces: C^-1 N and (C^-1 x) x^T are
appended to the A_b slabs as extra parameters (``_extra_slabs``).

Field segments are placed at 8-element-aligned offsets of a padded index
space (zero rows / columns in the gaps) so every TMA box starts 16-byte
aligned whatever the pixel counts.
"""

from __future__ import annotations

import ctypes

import torch

from . import layout as lay
from ._lib import check, stream
from .engine import Engine, _off

BF16 = torch.bfloat16
SCHEMES = {
    "bf16x3": (2, (0, 0, 1), (0, 1, 0)),
    "bf16x6": (3, (0, 0, 1, 0, 1, 2), (0, 1, 0, 2, 1, 0)),
}
# How A_b is stored and traced: (planes, ta, tb).  The traces sum ~n^2 products
# per entry of F, so the rounding of A_b to two planes (16 significant bits,
# unbiased) averages out; (1,1) is kept because on the diagonal it is the
# square of the second planes, a bias if left out (measured on the TQU
# nside-16 problem: |dF_bb|/F_bb 4.1e-6 with two planes and four terms,
# 3.8e-6 with three planes and six).
TRACE = {
    "bf16x3": (2, (0, 0, 1), (0, 1, 0)),
    "bf16x6": (2, (0, 0, 1, 1), (0, 1, 0, 1)),
}


def _r8(x: int) -> int:
    return (int(x) + 7) // 8 * 8


class MixedPlan:
    """Padded segment layout and plane buffers for one layout and scheme."""

    def __init__(self, E: Engine, scheme: str):
        if scheme not in SCHEMES:
            raise ValueError(f"unknown scheme {scheme!r}; expected one of {list(SCHEMES)}")
        self.E = E
        self.planes, ta, tb = SCHEMES[scheme]
        self.nterms = len(ta)
        self._ta = (ctypes.c_int * len(ta))(*ta)
        self._tb = (ctypes.c_int * len(tb))(*tb)
        # planes of the stored A_b slabs, and the product terms of their traces
        self.out_planes, qa, qb = TRACE[scheme]
        self.trace = (self.out_planes, len(qa), (ctypes.c_int * len(qa))(*qa), (ctypes.c_int * len(qb))(*qb))
        L = E.L
        self.po = []  # padded offset of each field segment
        off = 0
        for f in L.fields:
            self.po.append(off)
            off = _r8(off + f.nrows)
        self.n_pad = off
        self.segments = list(range(len(L.fields)))
        self.err = torch.zeros(1, dtype=torch.int32, device=E.dev)

    @property
    def ta(self):
        return ctypes.cast(self._ta, ctypes.c_void_p)

    @property
    def tb(self):
        return ctypes.cast(self._tb, ctypes.c_void_p)

    def split_cinv(self, Cinv: torch.Tensor) -> torch.Tensor:
        """BF16 planes of an n x n FP64 matrix in the padded index space."""
        L, E = self.E.L, self.E
        npd = self.n_pad
        Cp = torch.zeros((self.planes, npd, npd), dtype=BF16, device=E.dev)
        for fi, f in enumerate(L.fields):
            for gi, g in enumerate(L.fields):
                src = _off(Cinv, f.offset * L.n + g.offset)
                dst = _off(Cp, self.po[fi] * npd + self.po[gi])
                check(E.lib.cf_split_bf16(f.nrows, g.nrows, src, L.n, self.planes, dst, npd, npd * npd,
                                          stream()), "cf_split_bf16")
        return Cp

    def pad_rows(self, V: torch.Tensor) -> torch.Tensor:
        """Rows of an n x k FP64 array moved to their padded positions (zeros in gaps)."""
        L = self.E.L
        out = torch.zeros((self.n_pad, V.shape[1]), dtype=V.dtype, device=V.device)
        for fi, f in enumerate(L.fields):
            out[self.po[fi]: self.po[fi] + f.nrows] = V[f.offset: f.offset + f.nrows]
        return out


def _build_planes(plan: MixedPlan, s: int):
    """BF16 planes of the derivative blocks of spectrum s as GEMM B operands.

    Returns {segment: (B planes tensor, K, k_seg)}: B rows are (bin, j) for
    output columns j in `segment` (each bin padded to a multiple of 8 rows,
    the padding rows zero), the K index runs over segment `k_seg`.
    """
    E, L = plan.E, plan.E.L
    blk = L.blocks[E.block_of_spec[s]]
    fa, fb = L.fields[blk.fa], L.fields[blk.fb]
    nb, Lp = L.nbins, L.lmax_signal + 1
    mode = L.spectra[s].mode
    t0 = _off(E.deriv_tab, s * Lp)
    bins = _off(E.deriv_bin, s * Lp)
    P = plan.planes
    va, vb = E.vec[blk.fa], E.vec[blk.fb]
    def alloc(rows_per_bin, rows_pad, ld):
        mk = torch.empty if rows_pad == rows_per_bin else torch.zeros
        return mk((P, nb * rows_pad, ld), dtype=BF16, device=E.dev)

    if blk.kind in (lay.KIND_00_AUTO, lay.KIND_22_AUTO):
        m = fa.nrows
        mp = ldm = _r8(m)
        D = alloc(m, mp, ldm)
        ps = nb * mp * ldm
        check(E.lib.cf_build_block_planes(
            blk.kind, mode, fa.npix, va.data_ptr(), fb.npix, vb.data_ptr(), L.lmax_signal, t0, None, None,
            bins, D.data_ptr(), ldm, 0, 0, mp * ldm, D.data_ptr(), ldm, 0, 0, mp * ldm, 1, 0, 0, P, ps, ps,
            1, stream()), "cf_build_block_planes")
        return blk, {blk.fa: (D, m, blk.fa)}
    R, Cc = fb.nrows, fa.nrows
    Rp = ldR = _r8(R)
    Cp_ = ldC = _r8(Cc)
    Dba = alloc(R, Rp, ldC)  # [b][r in fb (padded)][c in fa]
    Dab = alloc(Cc, Cp_, ldR)  # [b][c in fa (padded)][r in fb]
    for flags in (1, 2):  # Dba (coalesced rows of fb), then Dab by the transposed walk
        check(E.lib.cf_build_block_planes(
            blk.kind, mode, fa.npix, va.data_ptr(), fb.npix, vb.data_ptr(), L.lmax_signal, t0, None, None,
            bins, Dba.data_ptr(), ldC, 0, 0, Rp * ldC, Dab.data_ptr(), ldR, 0, 0, Cp_ * ldR, 1, 0, 0, P,
            nb * Rp * ldC, nb * Cp_ * ldR, flags, stream()), "cf_build_block_planes")
    # output columns in fa: K over fb with B[b][j in fa][k in fb] = Dab;
    # output columns in fb: K over fa with B[b][j in fb][k in fa] = Dba
    return blk, {blk.fa: (Dab, R, blk.fb), blk.fb: (Dba, Cc, blk.fa)}


def default_gemm_forms(L) -> dict:
    """Per-spectrum form of the A_b GEMM: {spectrum: (all_planes, promotion_kc)}.

    The all-planes form (every plane of a k-slice per pipeline stage, the
    leading product in its own TMEM accumulator, the five corrections sharing
    a second one) is the faster one, and faster again on CTA pairs (form 2:
    256-row tiles, each CTA holding half of B; the same arithmetic per output
    entry).  On blocks that involve a spin-0 field its errors correlate with
    the transposed entries of A_b at the lowest multipoles (measured on the
    TQU nside-16 problem: |dF_bb|/F_bb 1.2e-5 for TT l=2 against 4e-6 term by
    term), so those spectra run term by term.
    """
    forms = {}
    for s, sp in enumerate(L.spectra):
        spin0 = any(L.fields[f].spin == 0 for f in (sp.fi, sp.fj))
        forms[s] = (0, 16) if spin0 else (2, 16)
    return forms


def fisher(E: Engine, Cinv: torch.Tensor, scheme: str = "bf16x6", forms: dict | None = None) -> torch.Tensor:
    """F (P x P, FP64) on the tensor cores (see _fisher_core)."""
    return _fisher_core(E, Cinv, scheme, forms=forms)[0]


def _fisher_core(E: Engine, Cinv: torch.Tensor, scheme: str = "bf16x6", N=None, maps=None, forms=None):
    """F (P x P, FP64), and the noise bias and quadratic forms when N / maps are
    given, with the A_b GEMMs and the traces on the tensor cores.

    A_b is kept for every parameter in one buffer per column segment (field):
    ``X[f]`` holds, for every spectrum whose derivative touches columns of
    field f, its bins' column slabs side by side (n_pad x sum nb * m_f), and
    ``XT[f]`` their transposes.  After all spectra, each ordered segment pair
    (s, t) is one tensor-core contraction of all parameters touching s against
    all parameters touching t, scattered into F through parameter-index maps.

    The noise bias and the quadratic forms are the same contraction against
    other matrices (qube/spectra.py:1124-1186):
    b_p = 1/2 Tr(A_p C^-1 N) and q_p = 1/2 y^T dC_p y = 1/2 Tr(A_p y x^T),
    y = C^-1 x.  So C^-1 N and each y x^T are appended to every segment's slabs
    as extra parameters, and the one pass of traces that forms F also forms
    F[p, extra] = b_p and q_p, reading every A_b slab once for all three.
    """
    plan = MixedPlan(E, scheme)
    L = E.L
    nb, P = L.nbins, L.n_params
    npd = plan.n_pad
    Pl, Po = plan.planes, plan.out_planes
    ev = E._probe_begin("split_cinv")
    Cp = plan.split_cinv(Cinv)
    E._probe_end("split_cinv", ev, 0)
    nsims = 0 if maps is None else maps.shape[1]
    nx = (1 if N is not None else 0) + nsims  # extra parameters: C^-1 N, then y_q x_q^T
    segrows = {i: f.nrows for i, f in enumerate(L.fields)}
    segpad = {i: _r8(f.nrows) for i, f in enumerate(L.fields)}
    cols_of = {}
    for s in range(L.nspectra):
        blk = L.blocks[E.block_of_spec[s]]
        cols_of[s] = [blk.fa] if blk.fa == blk.fb else [blk.fa, blk.fb]
    seg_specs = {f: [s for s in range(L.nspectra) if f in cols_of[s]] for f in range(len(L.fields))}
    X, XT, pmap, ldseg, xcol = {}, {}, {}, {}, {}
    for f, specs in seg_specs.items():
        if not specs and not nx:
            continue
        xcol[f] = len(specs) * nb * segpad[f]  # first column of the extra parameters
        ncols = xcol[f] + nx * segpad[f]
        ldseg[f] = _r8(ncols)
        X[f] = torch.empty((Po, npd, ldseg[f]), dtype=BF16, device=E.dev)
        XT[f] = torch.empty((Po, ncols, npd), dtype=BF16, device=E.dev)
        pmap[f] = torch.tensor([s * nb + b for s in specs for b in range(nb)] + [P + q for q in range(nx)],
                               dtype=torch.int32, device=E.dev)
    if forms is None:
        from .autotune import forms_for

        forms = forms_for(E, Cinv, scheme)
    prev_ap = E.lib.cf_umma_set_all_planes(1)
    prev_kc = E.lib.cf_umma_set_promotion(16)
    prev_gm = E.lib.cf_umma_set_group(16)
    for s in range(L.nspectra):
        form = tuple(forms.get(s, (1, 16)))
        ap, kc = form[0], form[1]
        E.lib.cf_umma_set_all_planes(ap)
        E.lib.cf_umma_set_promotion(kc)
        E.lib.cf_umma_set_group(form[2] if len(form) > 2 else 16)
        ev = E._probe_begin("build_planes")
        blk, ops = _build_planes(plan, s)
        E._probe_end("build_planes", ev, 0)
        for seg, (B, K, kseg) in ops.items():
            ncol = nb * segpad[seg]
            col0 = seg_specs[seg].index(s) * ncol
            Xs, XTs = X[seg], XT[seg]
            ev = E._probe_begin("a_gemm_mixed")
            torch.cuda.nvtx.range_push("a_gemm_mixed")
            check(E.lib.cf_umma_gemm_bf16(
                npd, ncol, K, plan.nterms, plan.ta, plan.tb, _off(Cp, plan.po[kseg]), npd, npd * npd, Pl,
                B.data_ptr(), B.shape[2], B.shape[1] * B.shape[2], Pl,
                _off(Xs, col0), ldseg[seg], npd * ldseg[seg], Po,
                _off(XTs, col0 * npd), npd, XTs.shape[1] * npd, None, 0,
                plan.err.data_ptr(), stream()), "cf_umma_gemm_bf16")
            torch.cuda.nvtx.range_pop()
            E._probe_end("a_gemm_mixed", ev, 2.0 * npd * ncol * K * plan.nterms)
        del ops
    E.lib.cf_umma_set_all_planes(prev_ap)
    E.lib.cf_umma_set_promotion(prev_kc)
    E.lib.cf_umma_set_group(prev_gm)
    if nx:
        ev = E._probe_begin("qml_mixed")
        _extra_slabs(plan, Cp, Cinv, N, maps, X, XT, ldseg, xcol, segpad)
        E._probe_end("qml_mixed", ev, 0)
    Pt = P + nx
    Fx = torch.zeros((Pt, Pt), dtype=torch.float64, device=E.dev)
    segs = list(X)
    for a, ss in enumerate(segs):
        # (s, t) and (t, s) give transposed blocks of F: compute s <= t, mirror s < t
        for tt in segs[a:]:
            P1, P2 = pmap[ss].numel(), pmap[tt].numel()
            m_s, m_t = segrows[ss], segrows[tt]
            ev = E._probe_begin("trace_mixed")
            torch.cuda.nvtx.range_push("trace_mixed")
            tpl, tnt, tta, ttb = plan.trace
            check(E.lib.cf_umma_trace_bf16_mapped(
                P1, P2, m_t, m_s, tnt, ctypes.cast(tta, ctypes.c_void_p), ctypes.cast(ttb, ctypes.c_void_p),
                _off(X[ss], plan.po[tt] * ldseg[ss]), segpad[ss], ldseg[ss], npd * ldseg[ss], tpl,
                _off(XT[tt], plan.po[ss]), segpad[tt] * npd, npd, XT[tt].shape[1] * npd, tpl,
                0.5, Fx.data_ptr(), Pt, pmap[ss].data_ptr(), pmap[tt].data_ptr(), int(ss != tt), 0,
                plan.err.data_ptr(), stream()), "cf_umma_trace_bf16_mapped")
            torch.cuda.nvtx.range_pop()
            E._probe_end("trace_mixed", ev, 2.0 * P1 * P2 * m_t * m_s * tnt)
    del X, XT
    check(E.lib.cf_umma_status(plan.err.data_ptr(), stream()), "tensor-core kernel")
    if not nx:
        return Fx, None
    F = Fx[:P, :P].contiguous()
    bias = Fx[:P, P].contiguous() if N is not None else None
    q = Fx[:P, Pt - nsims:].T.contiguous() if nsims else None
    return F, (bias, q)


def _extra_slabs(plan, Cp, Cinv, N, maps, X, XT, ldseg, xcol, segpad):
    """Column slabs (and transposes) of the extra contraction partners C^-1 N
    and y_q x_q^T, written after each segment's A_b slabs.

    With A~ appended as a parameter, the trace gives 1/2 Tr(A_p A~); the bias
    needs A~ = (N C^-1)^T = C^-1 N and the quadratic form of map q needs
    A~ = (x y^T)^T = y x^T.
    """
    E = plan.E
    npd, Pl, Po = plan.n_pad, plan.planes, plan.out_planes
    j = 0
    if N is not None:
        Np = plan.split_cinv(N)
        for f in X:
            # X[f][:, c] = (C^-1 N)[:, po_f + c] = C^-1 (row po_f + c of N)^T
            check(E.lib.cf_umma_gemm_bf16(
                npd, segpad[f], npd, plan.nterms, plan.ta, plan.tb, Cp.data_ptr(), npd, npd * npd, Pl,
                _off(Np, plan.po[f] * npd), npd, npd * npd, Pl,
                _off(X[f], xcol[f]), ldseg[f], npd * ldseg[f], plan.out_planes,
                _off(XT[f], xcol[f] * npd), npd, XT[f].shape[1] * npd, None, 0,
                plan.err.data_ptr(), stream()), "cf_umma_gemm_bf16")
        del Np
        j = 1
    if maps is not None:
        nsims = maps.shape[1]
        Xm = maps.to(E.dev, torch.float64).contiguous()
        Ym = E.gemm(Cinv, Xm)
        xp, yp = plan.pad_rows(Xm), plan.pad_rows(Ym)
        for f in X:
            sp, c0 = segpad[f], xcol[f] + j * segpad[f]
            xs = _off(xp, plan.po[f] * nsims)
            # X[f][k, c0 + q sp + c] = y_q[k] x_q[po_f + c]
            check(E.lib.cf_outer_planes_rect(npd, sp, nsims, yp.data_ptr(), xs, nsims, Po, _off(X[f], c0),
                                             ldseg[f], sp, npd * ldseg[f], stream()), "cf_outer_planes_rect")
            # XT[f][c0 + q sp + c, k] = x_q[po_f + c] y_q[k]
            check(E.lib.cf_outer_planes_rect(sp, npd, nsims, xs, yp.data_ptr(), nsims, Po, _off(XT[f], c0 * npd),
                                             npd, sp * npd, XT[f].shape[1] * npd, stream()), "cf_outer_planes_rect")


def fisher_qml(E: Engine, Cinv: torch.Tensor, N: torch.Tensor | None = None,
               maps: torch.Tensor | None = None, scheme: str = "bf16x6", forms: dict | None = None):
    """Mixed F, FP64 bias and q (same return convention as Engine.fisher_qml)."""
    F, qml = _fisher_core(E, Cinv, scheme, N, maps, forms=forms)
    bias, q = qml if qml is not None else (None, None)
    if q is not None and N is None:
        bias = None
    return F, bias, q
