"""CPU oracle for the QML / Fisher / pixel-likelihood path (test infrastructure).

This module is the checker, never the thing measured or shipped: only the
tests, ``__graft_entry__.smoke()`` and the CPU-baseline leg of ``bench.py``
may import it.  It restates the reference algorithm:

* signal and binned-derivative matrices through the C restatement in
  ``signal_oracle.c`` (``cosmocore/signal_kernels.py:164-537``,
  ``cosmocore/basis/pixel.py:802-950``);
* ``matrix_inverse_symm``: Jacobi scaling D M D, LAPACK ``dpotrf`` +
  ``dpotri``, mirror, unscale (``cosmocore/basics/linalg.py:152-219``);
* Fisher F_ij = 1/2 Tr(C^-1 dC_i C^-1 dC_j) from A_i = C^-1 dC_i
  (``qube/fisher.py:501-607``);
* QML y = C^-1 x, q_b = 1/2 y^T dC_b y, bias_b = 1/2 Tr(C^-1 N C^-1 dC_b),
  q -= bias, C_hat = q F^-1 (``qube/spectra.py:1124-1186, 1340-1356,
  1713-1733``);
* PICSLike chi2 = x^T C^-1 x, ln|C| = 2 sum ln L_ii, lnL = -(chi2 + ln|C|)/2
  (``picslike/picslike.py:568-664``, ``cosmocore/basics/linalg.py:430-474``).

Parity of this oracle is pinned against the reference's own outputs and
the Fortran known answers in ``tests/golden/*.npz``.
"""

from __future__ import annotations

import ctypes
import os
import subprocess
from pathlib import Path

import numpy as np
from scipy.linalg import lapack

from cosmoforge_b200 import layout as lay

HERE = Path(__file__).resolve().parent
LIB_PATH = HERE / "_build" / "liborc.so"

_lib = None


def build(force: bool = False) -> Path:
    """Compile ``signal_oracle.c`` into ``oracle/_build/liborc.so``."""
    src = HERE / "signal_oracle.c"
    if LIB_PATH.exists() and not force and LIB_PATH.stat().st_mtime >= src.stat().st_mtime:
        return LIB_PATH
    LIB_PATH.parent.mkdir(exist_ok=True)
    tmp = LIB_PATH.with_suffix(f".{os.getpid()}.tmp")
    subprocess.run(
        ["gcc", "-O2", "-fopenmp", "-ffp-contract=off", "-fno-fast-math", "-fPIC",
         "-shared", str(src), "-o", str(tmp), "-lm"],
        check=True,
    )
    os.replace(tmp, LIB_PATH)
    return LIB_PATH


def _load():
    global _lib
    if _lib is None:
        build()
        lib = ctypes.CDLL(str(LIB_PATH))
        dp = ctypes.POINTER(ctypes.c_double)
        lib.orc_block_00_auto.argtypes = [ctypes.c_int, dp, ctypes.c_int, dp, dp, ctypes.c_long, ctypes.c_long]
        lib.orc_block_00_cross.argtypes = [ctypes.c_int, dp, ctypes.c_int, dp, ctypes.c_int, dp, dp,
                                           ctypes.c_long, ctypes.c_long, ctypes.c_long]
        lib.orc_block_22_auto.argtypes = [ctypes.c_int, dp, ctypes.c_int, dp, dp, dp, dp,
                                          ctypes.c_long, ctypes.c_long]
        lib.orc_block_02.argtypes = [ctypes.c_int, dp, ctypes.c_int, dp, ctypes.c_int, dp, dp, dp,
                                     ctypes.c_long, ctypes.c_long, ctypes.c_long]
        lib.orc_mirror_lower.argtypes = [ctypes.c_long, dp, ctypes.c_long]
        lib.orc_rotation_angle.argtypes = [dp, dp, dp]
        lib.orc_legendre.argtypes = [ctypes.c_int, ctypes.c_double, ctypes.c_int, dp]
        _lib = lib
    return _lib


def _p(a: np.ndarray):
    assert a.dtype == np.float64 and a.flags.c_contiguous
    return a.ctypes.data_as(ctypes.POINTER(ctypes.c_double))


def rotation_angle(r1, r2):
    out = np.zeros(2)
    _load().orc_rotation_angle(_p(np.ascontiguousarray(r1, dtype=np.float64)),
                               _p(np.ascontiguousarray(r2, dtype=np.float64)), _p(out))
    return float(out[0]), float(out[1])


def legendre(kind: int, x: float, lmax: int) -> np.ndarray:
    out = np.zeros(3 * (lmax + 1))
    _load().orc_legendre(kind, float(x), lmax, _p(out))
    return out if kind == 22 else out[: lmax + 1]


def _fill_block(lib, L: lay.Layout, blk: lay.BlockSpec, tables: np.ndarray, S: np.ndarray):
    """Fill one block's lower-triangle entries using per-spectrum l tables."""
    zero = np.zeros(L.lmax_signal + 1)
    fa, fb = L.fields[blk.fa], L.fields[blk.fb]
    n = S.shape[0]

    def tab(k):
        return np.ascontiguousarray(tables[k]) if k is not None else zero

    if blk.kind == lay.KIND_00_AUTO:
        lib.orc_block_00_auto(fa.npix, _p(fa.vectors), L.lmax_signal, _p(tab(blk.spectra[0])),
                              _p(S), n, fa.offset)
    elif blk.kind == lay.KIND_00_CROSS:
        lib.orc_block_00_cross(fa.npix, _p(fa.vectors), fb.npix, _p(fb.vectors), L.lmax_signal,
                               _p(tab(blk.spectra[0])), _p(S), n, fa.offset, fb.offset)
    elif blk.kind == lay.KIND_22_AUTO:
        by_mode = {L.spectra[k].mode: k for k in blk.spectra}
        lib.orc_block_22_auto(fa.npix, _p(fa.vectors), L.lmax_signal, _p(tab(by_mode.get(0))),
                              _p(tab(by_mode.get(1))), _p(tab(by_mode.get(2))), _p(S), n, fa.offset)
    elif blk.kind == lay.KIND_02:
        by_mode = {L.spectra[k].mode: k for k in blk.spectra}
        lib.orc_block_02(fa.npix, _p(fa.vectors), fb.npix, _p(fb.vectors), L.lmax_signal,
                         _p(tab(by_mode.get(0))), _p(tab(by_mode.get(1))), _p(S), n,
                         fa.offset, fb.offset)


def signal_matrix(L: lay.Layout, cl_table: np.ndarray) -> np.ndarray:
    """S = sum_l C~_l x kernels, every block, mirrored (signal_kernels.py:390-537)."""
    lib = _load()
    S = np.zeros((L.n, L.n))
    tables = np.ascontiguousarray(cl_table, dtype=np.float64)
    for blk in L.blocks:
        _fill_block(lib, L, blk, tables, S)
    lib.orc_mirror_lower(L.n, _p(S), L.n)
    return S


def binned_derivative(L: lay.Layout, p: int, weights: np.ndarray | None = None) -> np.ndarray:
    """dC_p for Fisher parameter p = spectrum * nbins + bin (pixel.py:802-950)."""
    lib = _load()
    W = L.param_weights() if weights is None else weights
    spec_idx = p // L.nbins
    tables = np.zeros((L.nspectra, L.lmax_signal + 1))
    tables[spec_idx] = W[p]
    blk = next(b for b in L.blocks if spec_idx in b.spectra)
    sub = lay.BlockSpec(blk.kind, blk.fa, blk.fb, [spec_idx])
    if blk.kind in (lay.KIND_22_AUTO, lay.KIND_02):
        sub = blk
    S = np.zeros((L.n, L.n))
    _fill_block(lib, L, sub, tables, S)
    lib.orc_mirror_lower(L.n, _p(S), L.n)
    return S


def matrix_inverse_symm(M: np.ndarray) -> np.ndarray:
    """Jacobi-scaled Cholesky inverse, as cosmocore/basics/linalg.py:152-219."""
    M = np.asfortranarray(M.copy())
    d = np.abs(np.diag(M).copy())
    d[d == 0.0] = 1.0
    dinv = 1.0 / np.sqrt(d)
    np.multiply(M, dinv[None, :], out=M)
    np.multiply(M, dinv[:, None], out=M)
    Lc, info = lapack.dpotrf(M, lower=True, overwrite_a=True, clean=True)
    if info != 0:
        raise ValueError(f"dpotrf failed with info={info}")
    inv, info = lapack.dpotri(Lc, lower=True, overwrite_c=True)
    if info != 0:
        raise ValueError(f"dpotri failed with info={info}")
    il = np.tril_indices(inv.shape[0], -1)
    inv[il[1], il[0]] = inv[il]
    np.multiply(inv, dinv[None, :], out=inv)
    np.multiply(inv, dinv[:, None], out=inv)
    return np.ascontiguousarray(inv)


def logdet_chol(C: np.ndarray) -> float:
    """ln|C| = 2 sum ln L_ii from dpotrf (linalg.py:430-474)."""
    Lc, info = lapack.dpotrf(np.asfortranarray(C), lower=True, overwrite_a=False, clean=True)
    if info != 0:
        raise ValueError(f"dpotrf failed with info={info}")
    return 2.0 * float(np.sum(np.log(np.diag(Lc))))


def trace_product(A: np.ndarray, B: np.ndarray, BT: np.ndarray | None = None) -> float:
    """Tr(A B) = sum_ij A_ij B_ji (linalg.py:66-98); pass BT = B^T if already formed."""
    if BT is None:
        BT = np.ascontiguousarray(B.T)
    return float(np.vdot(A.ravel(), BT.ravel()))


def fisher(L: lay.Layout, Cinv: np.ndarray, params=None) -> np.ndarray:
    """F_ij = 1/2 Tr(A_i A_j), A_i = C^-1 dC_i, for the listed parameters."""
    P = L.n_params if params is None else len(params)
    idx = list(range(L.n_params)) if params is None else list(params)
    W = L.param_weights()
    A = [Cinv @ binned_derivative(L, p, W) for p in idx]
    AT = [np.ascontiguousarray(a.T) for a in A]
    F = np.zeros((P, P))
    for a in range(P):
        for b in range(a, P):
            F[a, b] = F[b, a] = 0.5 * trace_product(A[a], A[b], AT[b])
    return F


def qml(L: lay.Layout, Cinv: np.ndarray, N: np.ndarray, maps: np.ndarray):
    """Raw q (nsims, P) with bias removed if remove_nb, and raw bias (P,)."""
    Y = Cinv @ maps
    M = Cinv @ (N @ Cinv)
    W = L.param_weights()
    q = np.zeros((maps.shape[1], L.n_params))
    b = np.zeros(L.n_params)
    for p in range(L.n_params):
        dC = binned_derivative(L, p, W)
        b[p] = 0.5 * trace_product(M, dC)
        qv = 0.5 * np.sum(Y * (dC @ Y), axis=0)
        if L.remove_nb:
            qv = qv - b[p]
        q[:, p] = qv
    return q, b


def qml_solve(L: lay.Layout, cls: dict, N: np.ndarray, maps: np.ndarray):
    """Full traditional pipeline: S, C^-1, F, q, bias, F^-1, C_hat."""
    S = signal_matrix(L, L.smoothed_cl_table(cls))
    Cinv = matrix_inverse_symm(N + S)
    F = fisher(L, Cinv)
    q, b = qml(L, Cinv, N, maps)
    Finv = matrix_inverse_symm(F)
    return dict(S=S, Cinv=Cinv, fisher=F, q=q, bias=b, invfisher=Finv,
                clhat=q @ Finv, noise_bias=b @ Finv)


def lnl_point(L: lay.Layout, cls: dict, N: np.ndarray, maps: np.ndarray, noise_scale=1.0):
    """(chi2 per sim, logdet, lnL per sim) at one parameter point."""
    S = signal_matrix(L, L.smoothed_cl_table(cls))
    C = S + noise_scale * N
    Cinv = matrix_inverse_symm(C)
    chi2 = np.einsum("in,ij,jn->n", maps, Cinv, maps)
    ld = logdet_chol(C)
    return chi2, ld, -0.5 * (chi2 + ld)
