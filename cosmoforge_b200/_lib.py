"""ctypes binding of the device library ``libcfb200.so``.

The library is the only compute path: when it is missing or no CUDA device
is present, every entry point here raises instead of falling back to CPU.
"""

from __future__ import annotations

import ctypes as C
from pathlib import Path

import torch

LIB_PATH = Path(__file__).resolve().parent / "libcfb200.so"

CF_OK = 0
CF_ERR_ARG = -1
CF_ERR_CUDA = -2
CF_ERR_TIMEOUT = -3
CF_ERR_UNSUPPORTED = -4
CF_ERR_TOO_LARGE = -5

_i, _l, _d, _p, _sz = C.c_int, C.c_long, C.c_double, C.c_void_p, C.c_size_t
_f = C.c_float

SIGNATURES = {
    "cf_version": (_i, []),
    "cf_launch_count": (C.c_ulonglong, []),
    "cf_build_block": (_i, [_i, _i, _i, _p, _i, _p, _i, _p, _p, _p, _p, _p, _l, _l, _l, _l, _p, _l,
                            _l, _l, _l, _i, _l, _l, _p]),
    "cf_build_block_planes": (_i, [_i, _i, _i, _p, _i, _p, _i, _p, _p, _p, _p, _p, _l, _l, _l, _l, _p,
                                   _l, _l, _l, _l, _i, _l, _l, _i, _l, _l, _i, _p]),
    "cf_harmonic_operator": (_i, [_i, _i, _i, _p, _i, _i, _p, _l, _l, _l, _p]),
    "cf_harmonic_lambda": (_i, [_l, _l, _i, _i, _p, _p, _p, _i, _p, _l, _p, _l, _p]),
    "cf_harmonic_fisher": (_i, [_i, _i, _i, _i, _p, _l, _p, _i, _p, _p, _p, _p, _i, _p, _l, _p]),
    "cf_harmonic_pair": (_i, [_i, _i, _i, _p, _l, _p, _l, _l, _i, _p, _i, _p, _p, _p, _p, _i, _p, _l, _p]),
    "cf_build_block_reduce": (_i, [_i, _i, _i, _p, _i, _p, _i, _p, _p, _p, _p, _i, _p, _l, _p, _l, _i, _l, _l,
                                   _d, _p, _p, _l, _p]),
    "cf_dgemm": (_i, [_i, _i, _i, _i, _i, _d, _p, _l, _l, _p, _l, _l, _d, _p, _l, _l, _p, _l, _l,
                      _i, _i, _p]),
    "cf_dgemm_f32copy": (_i, [_i, _i, _i, _i, _i, _d, _p, _l, _l, _p, _l, _l, _d, _p, _l, _l, _p, _l, _l, _i, _i,
                              _p]),
    "cf_potrf_workspace": (_sz, [_i, _i]),
    "cf_potrf": (_i, [_i, _p, _l, _l, _i, _p, _p, _p]),
    "cf_trtri_lower": (_i, [_i, _p, _l, _l, _p, _l, _l, _i, _p, _p]),
    "cf_spd_inverse_workspace": (_sz, [_i, _i]),
    "cf_spd_inverse": (_i, [_i, _p, _l, _l, _i, _p, _p, _p]),
    "cf_spd_inverse_static_max_n": (_i, []),
    "cf_spd_inverse_static": (_i, [_i, _p, _l, _p, _p]),
    "cf_trace_contract_f64": (_i, [_i, _i, _i, _i, _p, _l, _l, _p, _l, _l, _d, _p, _l, _l, _l, _i, _i,
                                   _p]),
    "cf_qml_reduce_f64": (_i, [_i, _i, _i, _p, _l, _l, _p, _l, _l, _l, _p, _l, _i, _l, _l, _d, _p,
                               _p, _l, _p]),
    "cf_chi2_logdet": (_i, [_i, _p, _l, _l, _i, _p, _l, _l, _i, _p, _p, _p, _p]),
    "cf_chi2_logdet_dinv": (_i, [_i, _p, _l, _l, _p, _l, _i, _p, _l, _l, _i, _p, _p, _p]),
    "cf_potrf_dinv_stride": (_sz, [_i]),
    "cf_axpby": (_i, [_l, _d, _p, _l, _d, _p, _p, _l, _p, _l, _i, _p]),
    "cf_transpose": (_i, [_i, _i, _p, _l, _p, _l, _p]),
    "cf_umma_trace_bf16": (_i, [_i, _i, _i, _i, _i, _p, _p, _p, _l, _l, _l, _i, _p, _l, _l, _l, _i, _d,
                                _p, _l, _l, _l, _i, _i, _p, _p]),
    "cf_umma_set_promotion": (_i, [_i]),
    "cf_umma_set_trace_pairs": (_i, [_i]),
    "cf_umma_set_wait_limit": (C.c_longlong, [C.c_longlong]),
    "cf_umma_status": (_i, [_p, _p]),
    "cf_umma_set_all_planes": (_i, [_i]),
    "cf_umma_set_group": (_i, [_i]),
    "cf_umma_trace_bf16_mapped": (_i, [_i, _i, _i, _i, _i, _p, _p, _p, _l, _l, _l, _i, _p, _l, _l, _l, _i,
                                       _d, _p, _l, _p, _p, _i, _i, _p, _p]),
    "cf_outer_planes": (_i, [_i, _i, _p, _p, _l, _i, _p, _l, _l, _l, _p]),
    "cf_outer_planes_rect": (_i, [_i, _i, _i, _p, _p, _l, _i, _p, _l, _l, _l, _p]),
    "cf_split_bf16": (_i, [_i, _i, _p, _l, _i, _p, _l, _l, _p]),
    "cf_umma_gemm_bf16": (_i, [_i, _i, _i, _i, _p, _p, _p, _l, _l, _i, _p, _l, _l, _i, _p, _l, _l, _i,
                               _p, _l, _l, _p, _l, _p, _p]),
    "cf_umma_gemm_bf16_scatter": (_i, [_i, _i, _i, _i, _p, _p, _p, _l, _l, _i, _p, _l, _l, _i, _p, _p, _l, _i,
                                       _l, _p, _p]),
    "cf_potrf_f32_workspace": (_sz, [_i, _i]),
    "cf_potrf_f32": (_i, [_i, _p, _l, _l, _i, _p, _p, _p]),
    "cf_sgemm_bf16x6": (_i, [_i, _i, _i, _f, _p, _l, _l, _p, _l, _l, _f, _p, _l, _l, _i, _i, _p, _p]),
    "cf_sgemm_bf16x6_set_wait_limit": (C.c_longlong, [C.c_longlong]),
    "cf_sgemm_bf16x6_set_stages": (_i, [_i]),
    "cf_potrf_f32_set_tensor": (_i, [_i]),
    "cf_potrf_f32_set_group": (_i, [_i]),
    "cf_axpby_f32": (_i, [_l, _d, _p, _l, _d, _p, _p, _l, _p, _l, _p, _l, _i, _p]),
    "cf_chi2_logdet_mixed": (_i, [_i, _p, _l, _l, _p, _l, _l, _i, _p, _l, _l, _i, _p, _p, _p]),
    "cf_chi2_logdet_mixed_c32": (_i, [_i, _p, _l, _l, _p, _l, _l, _i, _p, _l, _l, _i, _p, _p, _p]),
    "cf_chi2_logdet_mixed_dinv": (_i, [_i, _p, _l, _l, _p, _l, _p, _l, _l, _i, _p, _l, _l, _i, _p, _p, _p]),
    "cf_chi2_logdet_mixed_c32_dinv": (_i, [_i, _p, _l, _l, _p, _l, _p, _l, _l, _i, _p, _l, _l, _i, _p, _p, _p]),
    "cf_potrf_f32_dinv_stride": (_sz, [_i]),
    "cf_mlp_dense_fwd": (_i, [_i, _i, _i, _p, _l, _p, _p, _i, _p, _p, _l, _p]),
    "cf_mlp_dense_bwd_data": (_i, [_i, _i, _i, _p, _p, _p, _p, _p]),
    "cf_mlp_dense_bwd_weight": (_i, [_i, _i, _i, _p, _p, _l, _p, _p, _p]),
    "cf_mlp_mse": (_i, [_i, _p, _p, _p, _p, _p, _p]),
    "cf_mlp_adam": (_i, [_l, _p, _p, _p, _p, _f, _f, _f, _f, _p, _p, _p]),
    "cf_to_bf16": (_i, [_l, _p, _p, _p]),
    "cf_mcmc_propose": (_i, [_i, _i, _p, _p, _p, _i, _p, _p, _p, _p, _p, _p, _p, _p]),
    "cf_mcmc_stage1": (_i, [_i, _i, _p, _p, _d, _d, _p, _p, _p, _p, _p, _p, _p, _i, _p, _p]),
    "cf_mcmc_stage2": (_i, [_i, _i, _p, _p, _p, _p, _p, _p, _p, _p, _p, _p, _i, _p, _p, _p]),
    "cf_qform_reduce_f64": (_i, [_i, _i, _l, _p, _l, _p, _l, _l, _i, _d, _p, _l, _i, _p]),
    "cf_qform_reduce_f32": (_i, [_i, _i, _l, _p, _l, _p, _l, _l, _i, _d, _p, _l, _i, _p]),
    "cf_mcmc_mh_accept": (_i, [_i, _i, _p, _p, _p, _p, _p, _p, _p, _p, _i, _p, _p, _p]),
    "cf_mcmc_sub_accept": (_i, [_i, _i, _p, _p, _d, _d, _p, _p, _p, _p, _p, _p]),
    "cf_mcmc_sub_final": (_i, [_i, _i, _p, _p, _p, _p, _p, _p, _p, _p, _p, _i, _p, _p, _p]),
    "cf_mcmc_subchain": (_i, [_i, _i, _i, _i, _p, _p, _i, _p, _p, _p, _p, _p, _p, _p, _d, _d, _p, _p, _p, _p,
                              _p]),
}

_lib = None


class DeviceError(RuntimeError):
    pass


def lib():
    """Load the library (once); raise if it or a CUDA device is missing."""
    global _lib
    if _lib is None:
        if not LIB_PATH.exists():
            raise DeviceError(
                f"{LIB_PATH.name} is not built; run `python -m cosmoforge_b200._build` "
                "(the device path has no CPU fallback)")
        if not torch.cuda.is_available():
            raise DeviceError("no CUDA device: cosmoforge_b200 runs on the GPU only")
        handle = C.CDLL(str(LIB_PATH))
        for name, (res, args) in SIGNATURES.items():
            fn = getattr(handle, name)
            fn.restype = res
            fn.argtypes = args
        _lib = handle
    return _lib


def load_without_device():
    """Load the library for symbol inspection only (no compute calls)."""
    return C.CDLL(str(LIB_PATH))


def check(rc: int, what: str = "") -> None:
    if rc == CF_OK:
        return
    names = {CF_ERR_ARG: "invalid argument", CF_ERR_CUDA: "CUDA launch error",
             CF_ERR_TIMEOUT: "timeout", CF_ERR_UNSUPPORTED: "unsupported",
             CF_ERR_TOO_LARGE: "size exceeds the static scratch capacity"}
    raise DeviceError(f"{what}: {names.get(rc, rc)}")


def ptr(t) -> int | None:
    if t is None:
        return None
    return t.data_ptr()


def stream(s=None) -> int:
    s = torch.cuda.current_stream() if s is None else s
    return s.cuda_stream
