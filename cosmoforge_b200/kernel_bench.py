"""Single-kernel timing cases for the tensor-core and FP64 kernels.

    python -m cosmoforge_b200.kernel_bench umma_gemm M,N,K [--planes 3] [--reps 5] [--kc 16]
    python -m cosmoforge_b200.kernel_bench umma_trace P1,P2,K1,K2 [--planes 3]
    python -m cosmoforge_b200.kernel_bench dgemm M,N,K
    python -m cosmoforge_b200.kernel_bench spd_inverse N
    python -m cosmoforge_b200.kernel_bench harmonic 1        (config-1 harmonic-basis solve)
    python -m cosmoforge_b200.kernel_bench map_solves NMAPS [--precision fp64|mixed]

Each case fills seeded random operands on cuda:0, runs two untimed launches,
then times `reps` launches with CUDA events on the launching stream and prints
one line: case, shape, ms per launch, throughput.  The autotuner
(cosmoforge_b200.autotune) times the same closures.
"""

from __future__ import annotations

import argparse
import ctypes

import torch

from . import _lib

X3 = ([0, 0, 1], [0, 1, 0])
X6 = ([0, 0, 1, 0, 1, 2], [0, 1, 0, 2, 1, 0])


def _terms(planes):
    t = X6 if planes == 3 else X3
    ta = (ctypes.c_int * len(t[0]))(*t[0])
    tb = (ctypes.c_int * len(t[1]))(*t[1])
    return len(t[0]), ctypes.cast(ta, ctypes.c_void_p), ctypes.cast(tb, ctypes.c_void_p), (ta, tb)


def time_launches(fn, reps):
    """Mean ms per call of fn over `reps` calls (two untimed calls first)."""
    fn()
    fn()
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    for _ in range(reps):
        fn()
    e1.record()
    torch.cuda.synchronize()
    return e0.elapsed_time(e1) / reps


def umma_gemm_case(M, N, K, planes=3, with_outputs=True):
    """Closure launching one split-product GEMM C = sum_t A_t B_t^T; returns (fn, flops, err)."""
    lib = _lib.lib()
    nt, ta, tb, keep = _terms(planes)
    g = torch.Generator(device="cuda").manual_seed(0)
    A = torch.randn((planes, M, K), device="cuda", generator=g).to(torch.bfloat16)
    B = torch.randn((planes, N, K), device="cuda", generator=g).to(torch.bfloat16)
    ldn, ldm = (N + 7) // 8 * 8, (M + 7) // 8 * 8
    X = torch.empty((planes, M, ldn), device="cuda", dtype=torch.bfloat16) if with_outputs else None
    XT = torch.empty((planes, N, ldm), device="cuda", dtype=torch.bfloat16) if with_outputs else None
    Cf = None if with_outputs else torch.empty((M, N), device="cuda", dtype=torch.float32)
    err = torch.zeros(1, dtype=torch.int32, device="cuda")
    st = torch.cuda.current_stream().cuda_stream

    def fn():
        rc = lib.cf_umma_gemm_bf16(
            M, N, K, nt, ta, tb, A.data_ptr(), K, M * K, planes, B.data_ptr(), K, N * K, planes,
            X.data_ptr() if X is not None else None, ldn, M * ldn, planes,
            XT.data_ptr() if XT is not None else None, ldm, N * ldm,
            Cf.data_ptr() if Cf is not None else None, N, err.data_ptr(), st)
        if rc != 0:
            raise RuntimeError(f"cf_umma_gemm_bf16 returned {rc}")

    fn._keep = (keep, A, B, X, XT, Cf)
    return fn, 2.0 * M * N * K * nt, err


def umma_trace_case(P1, P2, K1, K2, planes=3, splits=0):
    """Closure launching one split-product trace contraction into an FP64 F."""
    lib = _lib.lib()
    nt, ta, tb, keep = _terms(planes)
    g = torch.Generator(device="cuda").manual_seed(1)
    K2p = (K2 + 7) // 8 * 8
    Xp = torch.randn((planes, P1, K1, K2p), device="cuda", generator=g).to(torch.bfloat16)
    Yp = torch.randn((planes, P2, K1, K2p), device="cuda", generator=g).to(torch.bfloat16)
    F = torch.zeros((P1, P2), dtype=torch.float64, device="cuda")
    err = torch.zeros(1, dtype=torch.int32, device="cuda")
    st = torch.cuda.current_stream().cuda_stream

    def fn():
        rc = lib.cf_umma_trace_bf16(P1, P2, K1, K2, nt, ta, tb, Xp.data_ptr(), K1 * K2p, K2p, P1 * K1 * K2p, planes,
                                    Yp.data_ptr(), K1 * K2p, K2p, P2 * K1 * K2p, planes, 1.0, F.data_ptr(), P2, 0, 0,
                                    0, splits, err.data_ptr(), st)
        if rc != 0:
            raise RuntimeError(f"cf_umma_trace_bf16 returned {rc}")

    fn._keep = (keep, Xp, Yp, F)
    return fn, 2.0 * P1 * P2 * K1 * K2 * nt, err


def dgemm_case(M, N, K):
    lib = _lib.lib()
    g = torch.Generator(device="cuda").manual_seed(2)
    A = torch.randn((M, K), dtype=torch.float64, device="cuda", generator=g)
    B = torch.randn((K, N), dtype=torch.float64, device="cuda", generator=g)
    C = torch.empty((M, N), dtype=torch.float64, device="cuda")
    st = torch.cuda.current_stream().cuda_stream

    def fn():
        rc = lib.cf_dgemm(0, 0, M, N, K, 1.0, A.data_ptr(), K, 0, B.data_ptr(), N, 0, 0.0, C.data_ptr(), N, 0,
                          None, 0, 0, 1, 0, st)
        if rc != 0:
            raise RuntimeError(f"cf_dgemm returned {rc}")

    fn._keep = (A, B, C)
    return fn, 2.0 * M * N * K, None


def spd_inverse_case(n):
    """Inverse of one n x n SPD matrix (potrf + trtri + Y^T Y = n^3 flop)."""
    lib = _lib.lib()
    g = torch.Generator(device="cuda").manual_seed(3)
    R = torch.randn((n, n), dtype=torch.float64, device="cuda", generator=g)
    C0 = R @ R.T / n + torch.eye(n, dtype=torch.float64, device="cuda")
    A = C0.clone()
    work = torch.empty(lib.cf_spd_inverse_workspace(n, 1) // 8 + 1, dtype=torch.float64, device="cuda")
    info = torch.zeros(1, dtype=torch.int32, device="cuda")
    st = torch.cuda.current_stream().cuda_stream

    def fn():
        A.copy_(C0)
        rc = lib.cf_spd_inverse(n, A.data_ptr(), n, n * n, 1, work.data_ptr(), info.data_ptr(), st)
        if rc != 0:
            raise RuntimeError(f"cf_spd_inverse returned {rc}")

    fn._keep = (C0, A, work, info)
    return fn, float(n) ** 3, None


def harmonic_case(which):
    """One harmonic-basis QML solve of the TQU nside-16 problem (which = 1:
    n = 5952, l = 2..47; S, C^-1, F, bias, q, F^-1, C_hat), seeded map."""
    from . import harmonic, qube, workloads
    from .engine import Engine
    from .layout import build_layout

    if which != 1:
        raise SystemExit("harmonic: only the config-1 problem (shape 1) is defined")
    pb = workloads.config1()
    L = build_layout(pb.params, pb.mask, pb.beam)
    E = Engine(L)
    N = torch.from_numpy(pb.noise).cuda()
    x = qube.draw_maps(L, pb.cls, N, 1, seed=0)
    plan = harmonic.HarmonicPlan(E)

    def fn():
        harmonic.qml_solve(E, pb.cls, N, x, plan=plan)

    n, nm = L.n, plan.nm
    flop = 2.0 * n * n * nm * 3 + 2.0 * nm * nm * n + n ** 3  # V^T LV, Z, Z N; G; inverse
    fn._keep = (E, N, x, plan)
    return fn, flop, None


def map_solves_case(nmaps, precision="mixed"):
    """Raw q of nmaps seeded maps given C^-1 on the TQU nside-16 problem
    (config 2 part 1): signal build, C^-1 and the maps are set up once; each
    call is batch.map_solves (GEMMs against the derivative blocks and the
    k_qform reductions)."""
    from . import batch, qube, workloads
    from .engine import Engine
    from .layout import build_layout

    pb = workloads.config1()
    L = build_layout(pb.params, pb.mask, pb.beam)
    E = Engine(L)
    N = torch.from_numpy(pb.noise).cuda()
    Cinv = E.spd_inverse(E.signal(L.smoothed_cl_table(pb.cls)) + N)
    X = qube.draw_maps(L, pb.cls, N, nmaps, seed=0)

    def fn():
        batch.map_solves(E, Cinv, X, precision=precision)

    fn._keep = (E, N, Cinv, X)
    return fn, 0.0, None


def main(argv=None):
    ap = argparse.ArgumentParser(description=__doc__, formatter_class=argparse.RawDescriptionHelpFormatter)
    ap.add_argument("case", choices=["umma_gemm", "umma_trace", "dgemm", "spd_inverse", "harmonic",
                                           "map_solves"])
    ap.add_argument("shape", help="comma-separated sizes")
    ap.add_argument("--planes", type=int, default=3)
    ap.add_argument("--reps", type=int, default=5)
    ap.add_argument("--kc", type=int, default=16, help="promotion interval of the tensor-core kernels")
    ap.add_argument("--splits", type=int, default=0)
    ap.add_argument("--precision", choices=["fp64", "mixed"], default="mixed", help="map_solves only")
    a = ap.parse_args(argv)
    dims = [int(x) for x in a.shape.split(",")]
    lib = _lib.lib()
    lib.cf_umma_set_promotion(a.kc)
    if a.case == "umma_gemm":
        fn, fl, err = umma_gemm_case(*dims, planes=a.planes)
    elif a.case == "umma_trace":
        fn, fl, err = umma_trace_case(*dims, planes=a.planes, splits=a.splits)
    elif a.case == "dgemm":
        fn, fl, err = dgemm_case(*dims)
    elif a.case == "harmonic":
        fn, fl, err = harmonic_case(*dims)
    elif a.case == "map_solves":
        fn, fl, err = map_solves_case(*dims, precision=a.precision)
    else:
        fn, fl, err = spd_inverse_case(*dims)
    ms = time_launches(fn, a.reps)
    bad = int(err.item()) if err is not None else 0
    print(f"{a.case} {a.shape} planes={a.planes} kc={a.kc}: {ms:.3f} ms  {fl / ms / 1e9:.1f} TFLOP/s  err={bad}"
          if fl else f"{a.case} {a.shape} {a.precision}: {ms:.3f} ms per call")
    if bad:
        raise SystemExit("a bounded device wait ran out")


if __name__ == "__main__":
    main()
