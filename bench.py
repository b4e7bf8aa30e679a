#!/usr/bin/env python
"""QML solves/s on the TQU nside-16 problem (n = 5952 pixels, 276 Fisher parameters).

One step = one complete QML solve for one map: signal matrix S, C = S + N,
C^-1, the 276 x 276 Fisher matrix, raw bandpowers q, noise bias, F^-1 and
C_hat.  ``value`` is whole-job solves/s with every input already resident in
HBM, for the mixed-precision path by default (BF16x6 split products on the
tensor cores); the same step in plain FP64 is timed in the same run
(``fp64``) together with the mixed path's error against it.  ``e2e`` is the
metric through the drop-in ``Fisher`` / ``Spectra`` API with host inputs
(pinned) copied in and results copied out each step.

Secondary sections of the same line (skipped with ``--no-extra``): the
batched pixel likelihood (1024 parameter points, FP64 and FP32+refinement),
the emulator and delayed-acceptance sampler against exact Metropolis, the
bandpower window function, the same QML solve in the harmonic basis, the
2048-map solves and the 48-patch batch.

``--impl reference`` times the CPU restatement of the reference algorithm
(the oracle: C build with OpenMP, LAPACK/OpenBLAS linear algebra) on a
bounded sample of the same problem and extrapolates it to a full solve.

Multi-GPU (``torchrun``): the path does not shard (one GPU per
problem), so N GPUs run N independent replicas; time is the max over ranks.
"""

from __future__ import annotations

import argparse
import json
import math
import os
import statistics
import subprocess
import sys
import tempfile
import time
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))
WORKLOAD = "config1_tqu_nside16_qml"
METRIC = "QML solves/s (TQU nside16, n=5952, 276 bandpowers)"
UNIT = "solves/s"


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=3)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--precision", choices=["fp64", "mixed"], default="mixed")
    ap.add_argument("--fp64-steps", type=int, default=2,
                    help="timed FP64 steps beside a mixed headline (0: skip)")
    ap.add_argument("--no-extra", action="store_true", help="headline only (no secondary sections)")
    ap.add_argument("--scheme", choices=["bf16x3", "bf16x6"], default="bf16x6",
                    help="split-product scheme of the mixed path")
    ap.add_argument("--e2e-steps", type=int, default=2)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--sub-steps", type=int, default=128,
                    help="emulator Metropolis steps per exact evaluation in the two-level sampler")
    ap.add_argument("--lmax", type=int, default=None,
                    help="override the inference lmax (smaller profiling case; not a bench line)")
    return ap.parse_args()


# --------------------------------------------------------------------------
# CPU baseline: oracle on a bounded sample of the workload, extrapolated
# --------------------------------------------------------------------------
def cpu_sample(pb, L, k_params: int = 2):
    """Time S, C^-1, k parameters (dC, A = C^-1 dC, bias, q) and their traces.

    Extrapolates t_fixed + 276 t_param + 276*277/2 t_trace to one full solve.
    """
    from oracle import oracle as orc

    t0 = time.perf_counter()
    S = orc.signal_matrix(L, L.smoothed_cl_table(pb.cls))
    t_s = time.perf_counter() - t0
    N = pb.noise
    t0 = time.perf_counter()
    Cinv = orc.matrix_inverse_symm(S + N)
    Y = Cinv @ pb.extra["maps"]
    M = Cinv @ (N @ Cinv)
    t_inv = time.perf_counter() - t0
    W = L.param_weights()
    picks = np.linspace(0, L.n_params - 1, k_params).astype(int)
    A, AT = [], []
    t0 = time.perf_counter()
    for p in picks:
        dC = orc.binned_derivative(L, int(p), W)
        a = Cinv @ dC
        A.append(a)
        AT.append(np.ascontiguousarray(a.T))
        _ = 0.5 * orc.trace_product(M, dC)
        _ = 0.5 * np.sum(Y * (dC @ Y))
    t_param = (time.perf_counter() - t0) / k_params
    t0 = time.perf_counter()
    ntr = 0
    for i in range(k_params):
        for j in range(i, k_params):
            orc.trace_product(A[i], A[j], AT[j])
            ntr += 1
    t_trace = (time.perf_counter() - t0) / ntr
    P = L.n_params
    total = t_s + t_inv + P * t_param + P * (P + 1) / 2 * t_trace
    sample = (f"S + C^-1 + {k_params} of {P} parameters (dC, A=C^-1 dC, bias, q) + {ntr} traces, "
              f"extrapolated: t_S {t_s:.2f}s + t_inv {t_inv:.2f}s + {P} x {t_param:.2f}s + "
              f"{P * (P + 1) // 2} x {t_trace:.3f}s = {total:.0f}s per solve")
    return 1.0 / total, sample, total


def cpu_threads() -> int:
    try:
        return len(os.sched_getaffinity(0))
    except AttributeError:
        return os.cpu_count() or 1


def max_over_ranks(value: float, world: int, device) -> float:
    """The largest of a per-rank scalar over all ranks (a multi-GPU time is the
    slowest replica's); the identity for one rank."""
    import torch

    t = torch.tensor([value], dtype=torch.float64, device=device)
    if world > 1:
        import torch.distributed as dist

        dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def job_throughput(units_per_rank: float, seconds_max: float, world: int) -> float:
    """Whole-job throughput of `world` replicas that each processed
    units_per_rank units, timed as the slowest rank."""
    return world * units_per_rank / seconds_max


def bench_config(L) -> dict:
    """The ``config`` object of both arms' lines (identical by construction)."""
    return {"workload": WORKLOAD, "n_pixels": L.n, "n_params": L.n_params, "nsims": 1,
            "lmax_signal": L.lmax_signal, "parallelism": "replicas",
            "l2": "inputs larger than L2 (C^-1 283 MB, A_b slabs 56 GB)"}


def cpu_config0(reps: int = 3):
    """Full config-0 QML solves (TT nside 8, n = 480, 23 bandpowers) by the
    oracle port on the host: median seconds over `reps` after one warm-up."""
    from cosmoforge_b200 import workloads
    from cosmoforge_b200.layout import build_layout
    from oracle import oracle as orc

    pb = workloads.config0()
    L = build_layout(pb.params, pb.mask, pb.beam)
    x = np.random.default_rng(0).standard_normal((L.n, 1)) * 30.0
    orc.qml_solve(L, pb.cls, pb.noise, x)
    ts = []
    for _ in range(reps):
        t0 = time.perf_counter()
        orc.qml_solve(L, pb.cls, pb.noise, x)
        ts.append(time.perf_counter() - t0)
    t = statistics.median(ts)
    return {"workload": "config0_tt_nside8_qml", "n_pixels": L.n, "n_params": L.n_params,
            "solves_per_s": 1.0 / t, "ms_per_solve": t * 1e3, "runs": reps,
            "what": "whole solves (S, C^-1, F, q, bias, F^-1, C_hat), measured, not extrapolated"}


def run_reference(args):
    """Reference arm: the oracle restatement on host cores (rank 0 only).

    One step = one bounded sample of the config-1 solve (S, C^-1, one of the
    276 parameters with its derivative, A = C^-1 dC, bias, q and trace);
    ``ms_per_step`` is that sample's measured time and ``value`` the solves/s
    it implies (the sample's parts scaled to the whole solve).  The config-0
    section times whole solves, with no extrapolation."""
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    from cosmoforge_b200 import workloads
    from cosmoforge_b200.layout import build_layout

    pb = workloads.config1()
    L = build_layout(pb.params, pb.mask, pb.beam)
    pb.extra["maps"] = np.random.default_rng(0).standard_normal((L.n, 1))
    vals, times = [], []
    sample = ""
    for i in range(args.warmup + args.steps):
        t0 = time.perf_counter()
        v, sample, _ = cpu_sample(pb, L, k_params=1)
        dt = time.perf_counter() - t0
        if i >= args.warmup:
            vals.append(v)
            times.append(dt)
    v = statistics.median(vals)
    cores = cpu_threads()
    line = {
        "impl": "reference", "metric": METRIC, "value": v, "unit": UNIT, "n_gpus": args.gpus,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": statistics.median(times) * 1e3,
        "step": "one bounded sample of the solve; value = solves/s the sample implies",
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
        "data": "synthetic (seeded)", "config": bench_config(L),
        "cpu_baseline": {"value": v, "unit": UNIT, "cores": cores, "kind": "port", "sample": sample},
        "e2e": {"value": v, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
        "sections": {"config0": cpu_config0()},
    }
    print(json.dumps(line), flush=True)


# --------------------------------------------------------------------------
# GPU arm
# --------------------------------------------------------------------------
class ClockSampler:
    def __init__(self, index: int):
        self.f = tempfile.NamedTemporaryFile("w+", suffix=".csv", delete=False)
        self.p = None
        self.index = index

    def __enter__(self):
        try:
            self.p = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.index), "--query-gpu=clocks.sm,clocks.max.sm,"
                 "clocks_event_reasons.active,clocks_event_reasons.hw_slowdown,"
                 "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
                 "clocks_event_reasons.sw_power_cap", "--format=csv,noheader,nounits", "-lms", "200"],
                stdout=self.f, stderr=subprocess.DEVNULL)
        except OSError:
            self.p = None
        return self

    def __exit__(self, *exc):
        if self.p is not None:
            self.p.terminate()
            self.p.wait()

    def summary(self):
        self.f.flush()
        rows = []
        for line in open(self.f.name):
            parts = [x.strip() for x in line.split(",")]
            if len(parts) >= 7 and parts[0].isdigit():
                rows.append(parts)
        os.unlink(self.f.name)
        if not rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}
        sm = [int(r[0]) for r in rows]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[k] for r in rows for k in range(4) if r[3 + k].lower() == "active"})
        return {"sm_mhz": statistics.median(sm), "sm_max_mhz": int(rows[0][1]), "reasons": reasons,
                "samples": len(rows)}


def fp64_peak_tflops(torch):
    """Measured FP64 tensor peak: cuBLAS DGEMM 8192^3, best of 3 (for the FP64 roofline)."""
    a = torch.randn(8192, 8192, dtype=torch.float64, device="cuda")
    b = torch.randn(8192, 8192, dtype=torch.float64, device="cuda")
    torch.matmul(a, b)
    best = 1e9
    for _ in range(3):
        s, e = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        s.record()
        torch.matmul(a, b)
        e.record()
        torch.cuda.synchronize()
        best = min(best, s.elapsed_time(e) / 1e3)
    del a, b
    return 2 * 8192**3 / best / 1e12


def _cuda_ms(torch, fn, reps):
    """Mean ms of fn() over reps calls, CUDA events on the current stream (one untimed call first)."""
    fn()
    torch.cuda.synchronize()
    a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    a.record()
    for _ in range(reps):
        out = fn()
    b.record()
    torch.cuda.synchronize()
    return a.elapsed_time(b) / reps, out


def gpu_config0(dev, reps: int = 10):
    """Config-0 QML solves (TT nside 8, n = 480, 23 bandpowers) in plain FP64:
    on the device with resident inputs (CUDA events), and through the drop-in
    Fisher / Spectra API with host inputs (wall clock)."""
    import torch

    from cosmoforge_b200 import engine, qube, workloads
    from cosmoforge_b200.layout import build_layout

    pb = workloads.config0()
    L = build_layout(pb.params, pb.mask, pb.beam)
    E = engine.Engine(L, dev)
    N = torch.from_numpy(pb.noise).to(dev)
    x = qube.draw_maps(L, pb.cls, N, 1, seed=0, device=dev)
    ms, _ = _cuda_ms(torch, lambda: engine.qml_solve(E, pb.cls, N, x), reps)
    xh = x.cpu().numpy()
    ts = []
    for i in range(reps + 1):
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        f = qube.Fisher(pb.params, basis=False, mask=pb.mask, noise_cov1=pb.noise, cls_data=pb.cls,
                        beam=pb.beam, device=dev)
        f.run()
        s = qube.Spectra(pb.params, fisher=f, maps1=xh)
        s.run()
        s.get_power_spectra()
        torch.cuda.synchronize()
        if i > 0:
            ts.append(time.perf_counter() - t0)
    t_api = statistics.median(ts)
    return {"workload": "config0_tt_nside8_qml", "n_pixels": L.n, "n_params": L.n_params, "precision": "fp64",
            "solves_per_s": 1e3 / ms, "ms_per_solve": ms,
            "e2e_solves_per_s": 1.0 / t_api, "e2e_ms_per_solve": t_api * 1e3,
            "what": "whole solves (S, C^-1, F, q, bias, F^-1, C_hat); e2e = Fisher + Spectra API, host inputs"}


def secondary(args, dev):
    """Config 3 (batched lnL), config 4 (emulator + delayed acceptance) and config 2 (batched QML)."""
    import torch

    from cosmoforge_b200 import batch, engine, qube, sampler, workloads
    from cosmoforge_b200.emulator import MLPEmulator
    from cosmoforge_b200.layout import build_layout

    out = {}
    # ---- config 3: pixel likelihood over 1024 Sobol points ----
    pb = workloads.config3()
    L = build_layout(pb.params, pb.mask, pb.beam)
    E = engine.Engine(L, dev)
    N = torch.from_numpy(pb.noise).to(dev)
    X = qube.draw_maps(L, pb.cls, N, 1, seed=0, device=dev)
    T = sampler.ModelTables(L, dev)
    th = torch.as_tensor(workloads.sobol_points(1024), device=dev)
    cl = T(th)
    s = th[:, 4].contiguous()
    res = {}
    graph_ms = {}
    for prec in ("fp64", "mixed"):
        ms, r = _cuda_ms(torch, lambda: E.lnl(cl, N, X, noise_scale=s, precision=prec), 3)
        res[prec] = (ms, r)
        G = engine.LnlGraph(E, N, X, 1024, precision=prec)
        graph_ms[prec], _ = _cuda_ms(torch, lambda: G(cl, s), 3)
        del G
    # the opt-in tensor-core build of C (FP32 C, refinement against it)
    ms_tc, r_tc = _cuda_ms(torch, lambda: E.lnl(cl, N, X, noise_scale=s, precision="mixed", build="basis_tc"), 3)
    d = (res["mixed"][1][2] - res["fp64"][1][2]).abs()
    d_tc = (r_tc[2] - res["fp64"][1][2]).abs()
    # the autotuner's verified choice for this problem (product kernel and C build,
    # |dlnL| <= 0.05 against FP64 on its probe points with these maps)
    from cosmoforge_b200 import autotune

    choice, _ = autotune.tune_lnl(E, N, X, "mixed", batches=(1024,), use_cache=False)
    prev_t = E.lib.cf_potrf_f32_set_tensor(choice["tensor"])
    ms_tu, r_tu = _cuda_ms(torch, lambda: E.lnl(cl, N, X, noise_scale=s, precision="mixed", build=choice["build"]), 3)
    E.lib.cf_potrf_f32_set_tensor(prev_t)
    d_tu = (r_tu[2] - res["fp64"][1][2]).abs()
    lnl = {"workload": "config3_tqu_nside8_lnl", "n_pixels": L.n, "points_per_batch": 1024,
           "fp64_evals_per_s": 1024 / res["fp64"][0] * 1e3, "mixed_evals_per_s": 1024 / res["mixed"][0] * 1e3,
           "fp64_graph_evals_per_s": 1024 / graph_ms["fp64"] * 1e3,
           "mixed_graph_evals_per_s": 1024 / graph_ms["mixed"] * 1e3,
           "mixed_over_fp64": res["fp64"][0] / res["mixed"][0],
           "mixed_max_abs_dlnL": float(d.max()),
           "mixed_tc_build_evals_per_s": 1024 / ms_tc * 1e3,
           "mixed_tc_build_over_fp64": res["fp64"][0] / ms_tc,
           "mixed_tc_build_max_abs_dlnL": float(d_tc.max()),
           "mixed_tuned": {"choice": choice, "evals_per_s": 1024 / ms_tu * 1e3, "over_fp64": res["fp64"][0] / ms_tu,
                           "max_abs_dlnL": float(d_tu.max())},
           "build": "lower triangle of C(theta) from the per-multipole basis (one FP64 GEMM per block region; "
                    "mixed: the FP32 copy from the same epilogue); tc build: C in FP32 from BF16x6 tensor-core "
                    "products",
           "mixed_form": "FP32 Cholesky (diagonal blocks per CTA; panel solves, in-pass and trailing updates as "
                         "BF16x6 products on the one-tile tcgen05 kernel, the work panel as split planes), "
                         "FP64-refined chi2 against the FP64 C"}
    if int(os.environ.get("WORLD_SIZE", "1")) == 1 and not args.no_cpu_baseline:
        from oracle import oracle as orc

        thc = workloads.sobol_points(8, seed=5)
        xh = X.cpu().numpy()
        t0 = time.perf_counter()
        for t in thc:
            orc.lnl_point(L, workloads.model_cls(t, L.lmax_signal), pb.noise, xh, noise_scale=t[4])
        dt = time.perf_counter() - t0
        lnl["cpu_baseline"] = {"value": len(thc) / dt, "unit": "evals/s", "cores": cpu_threads(), "kind": "port",
                               "sample": f"{len(thc)} points, oracle S build + Jacobi inverse + logdet"}
    out["lnl"] = lnl

    # ---- config 4: emulator trained on exact evaluations, delayed acceptance ----
    t0 = time.perf_counter()
    th_tr, m2 = sampler.training_set(E, T, N, X, 32768, seed=0)
    torch.cuda.synchronize()
    t_set = time.perf_counter() - t0
    emu = MLPEmulator(workloads.THETA_LO, workloads.THETA_HI, seed=0, device=dev)
    t0 = time.perf_counter()
    hist = emu.fit(th_tr, m2, steps=3000, batch=1024, lr=1e-3)
    torch.cuda.synchronize()
    t_fit = time.perf_counter() - t0
    F = sampler.fisher_theta(E, T, N, workloads.THETA_CENTRE)
    prop = sampler.proposal_cov(F)
    rng = np.random.default_rng(7)
    pts = np.clip(rng.multivariate_normal(workloads.THETA_CENTRE, prop, 2048), workloads.THETA_LO,
                  workloads.THETA_HI)
    ex, _ = sampler.exact_m2lnl(E, T, N, X, pts)
    em = emu.predict_m2lnl(pts)
    dd = em - ex
    rms = float(0.5 * (dd - dd.mean()).pow(2).mean().sqrt())
    Xq = emu.normalise(pts[:64])
    emu_ms, _ = _cuda_ms(torch, lambda: emu.predict_std(Xq), 20)
    ex_ms, _ = _cuda_ms(torch, lambda: sampler.exact_m2lnl(E, T, N, X, pts[:64]), 3)
    s_da = sampler.Sampler(E, N, X, emulator=emu, prop_cov=prop, seed=1)
    ch_da, st_da = s_da.run_da(64, 400)
    s_sub = sampler.Sampler(E, N, X, emulator=emu, prop_cov=prop, seed=3)
    ch_sub, st_sub = s_sub.run_da_subchain(64, 200, sub_steps=args.sub_steps)
    s_mh = sampler.Sampler(E, N, X, prop_cov=prop, seed=2)
    ch_mh, st_mh = s_mh.run_exact_mh(64, 300)
    ess_da = sampler.effective_sample_size(ch_da.samples.cpu().numpy(), burn=80)
    ess_sub = sampler.effective_sample_size(ch_sub.samples.cpu().numpy(), burn=20)
    ess_mh = sampler.effective_sample_size(ch_mh.samples.cpu().numpy(), burn=50)
    out["emulator"] = {
        "workload": "config4_mlp_delayed_acceptance", "chains": 64,
        "training_points": 32768, "training_set_s": t_set, "fit_steps": 3000, "fit_s": t_fit,
        "final_loss": hist[-1][1], "rms_dlnL_near_posterior": rms,
        "emulated_evals_per_s": 64 / emu_ms * 1e3, "exact_evals_per_s_batch64": 64 / ex_ms * 1e3,
        "da": {"steps": st_da["steps"], "seconds": st_da["seconds"], "steps_per_s": st_da["steps"] / st_da["seconds"],
               "exact_evals_per_step": st_da["exact_evals"] / st_da["steps"],
               "stage2_acceptance": st_da["accepted"] / max(st_da["exact_evals"], 1),
               "min_ess_per_s": float(ess_da.min()) / st_da["seconds"]},
        "da_two_level": {"sub_steps": st_sub["sub_steps"], "steps": st_sub["steps"], "seconds": st_sub["seconds"],
                         "steps_per_s": st_sub["steps"] / st_sub["seconds"],
                         "emulator_steps_per_s": st_sub["steps"] * st_sub["sub_steps"] / st_sub["seconds"],
                         "exact_evals_per_step": st_sub["exact_evals"] / st_sub["steps"],
                         "sub_chain_acceptance": st_sub["sub_accepted"] / (st_sub["steps"] * st_sub["sub_steps"]),
                         "stage2_acceptance": st_sub["accepted"] / max(st_sub["exact_evals"], 1),
                         "min_ess": float(ess_sub.min()),
                         "min_ess_per_s": float(ess_sub.min()) / st_sub["seconds"],
                         "exact_evals_per_ess": st_sub["exact_evals"] / float(ess_sub.min())},
        "exact_mh": {"steps": st_mh["steps"], "seconds": st_mh["seconds"],
                     "steps_per_s": st_mh["steps"] / st_mh["seconds"],
                     "exact_evals_per_step": st_mh["exact_evals"] / st_mh["steps"],
                     "acceptance": st_mh["accepted"] / st_mh["steps"],
                     "min_ess": float(ess_mh.min()),
                     "min_ess_per_s": float(ess_mh.min()) / st_mh["seconds"],
                     "exact_evals_per_ess": st_mh["exact_evals"] / float(ess_mh.min())},
    }
    em_ = out["emulator"]
    em_["da_over_exact_steps_per_s"] = em_["da"]["steps_per_s"] / em_["exact_mh"]["steps_per_s"]
    em_["da_over_exact_ess_per_s"] = em_["da"]["min_ess_per_s"] / em_["exact_mh"]["min_ess_per_s"]
    em_["two_level_over_exact_ess_per_s"] = em_["da_two_level"]["min_ess_per_s"] / em_["exact_mh"]["min_ess_per_s"]
    em_["two_level_exact_evals_saved"] = (em_["exact_mh"]["exact_evals_per_ess"]
                                          / em_["da_two_level"]["exact_evals_per_ess"])
    del E, ch_da, ch_mh, ch_sub

    # ---- bandpower window function on config 1 binned by 5 multipoles ----
    pbw = workloads.config1()
    bw = {"workload": "config1_bandpower_window_dl5", "precision": "mixed"}
    fw = qube.Fisher(pbw.params | {"delta_ell": 5}, basis=False, mask=pbw.mask, noise_cov1=pbw.noise,
                     cls_data=pbw.cls, beam=pbw.beam, precision="mixed", device=dev)
    fw.run()
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    Wbp = fw.get_bandpower_window_function()
    torch.cuda.synchronize()
    Lw = fw.layout
    lmin_w, n_ell_w = int(fw.params.lmin), int(fw.params.lmax) - int(fw.params.lmin) + 1
    Qw = np.zeros((Lw.nbins, n_ell_w))
    for b, (lo, hi) in enumerate(zip(Lw.bin_lmins, Lw.bin_lmaxs)):
        Qw[b, lo - lmin_w: hi - lmin_w + 1] = 1.0
    Qw = np.kron(np.eye(Lw.nspectra), Qw)
    bw.update(seconds=time.perf_counter() - t0, shape=list(Wbp.shape),
              max_abs_WQt_minus_I=float(np.max(np.abs(Wbp @ Qw.T - np.eye(Qw.shape[0])))))
    out["bandpower"] = bw
    del fw, Wbp

    # ---- config 2: 2048 map-solves given C, and 48 sky patches ----
    pb1 = workloads.config1()
    L1 = build_layout(pb1.params, pb1.mask, pb1.beam)
    E1 = engine.Engine(L1, dev)
    N1 = torch.from_numpy(pb1.noise).to(dev)

    # ---- config 1 in the harmonic basis (the reference's default basis here) ----
    from cosmoforge_b200 import harmonic

    x1 = qube.draw_maps(L1, pb1.cls, N1, 1, seed=0, device=dev)
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    hplan = harmonic.HarmonicPlan(E1)
    torch.cuda.synchronize()
    t_plan = time.perf_counter() - t0
    ms_h, rh = _cuda_ms(torch, lambda: harmonic.qml_solve(E1, pb1.cls, N1, x1, plan=hplan), 3)
    Fp, _, _ = E1.fisher_qml(rh["Cinv"])
    dg = torch.diagonal(Fp)
    out["harmonic"] = {
        "workload": "config1_tqu_nside16_harmonic_basis", "modes": hplan.nm, "precision": "fp64",
        "basis_chosen_by_reference_cost_model": harmonic.auto_method(L1),
        "solves_per_s": 1e3 / ms_h, "ms_per_solve": ms_h, "plan_seconds": t_plan,
        "fisher_vs_pixel_fp64_corr_normalised": float(((rh["fisher"] - Fp).abs()
                                                        / torch.sqrt(torch.outer(dg, dg))).max()),
        "step": "S = S_fixed + V^T Lambda V, C^-1, Z = V C^-1, G = Z V^T, F, bias, q, F^-1, C_hat",
    }
    # the eigen-truncated pixel basis (epsilon 1e-3, noise-weighted) on the same problem
    tab1 = L1.smoothed_cl_table(pb1.cls)
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    cplan = harmonic.CompressedPlan(hplan, N1, tab1, epsilon=1e-3)
    torch.cuda.synchronize()
    t_cplan = time.perf_counter() - t0

    def csolve():
        Cci = E1.spd_inverse(cplan.project(hplan.signal(tab1) + N1))
        Fc, bc, _ = cplan.fisher_qml(Cci)
        _, _, qc = cplan.fisher_qml(Cci, with_bias=False, maps=x1, want_fisher=False)
        qc = qc - bc[None, :]
        return Fc, E1.gemm(qc, E1.spd_inverse(Fc.clone()))

    ms_c, (Fc, _) = _cuda_ms(torch, csolve, 3)
    out["harmonic"]["compressed"] = {
        "basis": {"method": "pixel", "epsilon": 1e-3, "compression_target": "noise_weighted"},
        "dim": cplan.dim, "of_n": L1.n, "setup_seconds": t_cplan, "solves_per_s": 1e3 / ms_c, "ms_per_solve": ms_c,
        "fisher_diag_rel_change_vs_uncompressed": float((torch.diagonal(Fc) / torch.diagonal(rh["fisher"]) - 1)
                                                        .abs().max()),
    }
    del rh, Fp, hplan, x1, cplan, Fc
    X1 = qube.draw_maps(L1, pb1.cls, N1, 2048, seed=0, device=dev)
    Cinv = E1.spd_inverse(E1.signal(L1.smoothed_cl_table(pb1.cls)) + N1)
    part1 = {}
    for prec in ("mixed", "fp64"):
        ms, q = _cuda_ms(torch, lambda: batch.map_solves(E1, Cinv, X1, precision=prec), 1)
        part1[prec] = (ms, q)
    del Cinv, X1, E1
    probs = []
    for j, p in enumerate(workloads.config2_patches()):
        Lp = build_layout(p.params, p.mask, p.beam)
        Np = torch.from_numpy(p.noise).to(dev)
        xp = qube.draw_maps(Lp, p.cls, Np, 1, seed=100 + j, device=dev)
        probs.append(dict(params=p.params, mask=p.mask, beam=p.beam, cls=p.cls, noise=p.noise, maps=xp.cpu().numpy()))
    pbat = batch.PatchBatch(probs, dev)
    pbat.run()
    ms2, _ = _cuda_ms(torch, pbat.run, 10)
    qm, qd = part1["mixed"][1], part1["fp64"][1]
    out["batched"] = {
        "map_solves": {"workload": "config2_part1_2048_maps", "maps": 2048,
                       "mixed_per_s": 2048 / part1["mixed"][0] * 1e3, "fp64_per_s": 2048 / part1["fp64"][0] * 1e3,
                       "mixed_max_rel_dq": float((qm - qd).abs().max() / qd.abs().max())},
        "patches": {"workload": "config2_part2_48_caps", "problems": 48, "pixels": [min(pbat.ns), max(pbat.ns)],
                    "bins": pbat.nb, "solves_per_s": 48 / ms2 * 1e3, "ms_per_batch": ms2,
                    "fisher_not_invertible": int((pbat.info_f != 0).sum()), "precision": "fp64",
                    "launch": "one CUDA graph replay per batch"},
    }
    return out


def main():
    args = parse()
    if args.impl == "reference":
        return run_reference(args)

    import torch
    import torch.distributed as dist

    from cosmoforge_b200 import _lib, engine, qube, workloads
    from cosmoforge_b200.layout import build_layout

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    if world > 1:
        import datetime

        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))

    def barrier():
        if world > 1:
            dist.barrier()

    pb = workloads.config1()
    if args.lmax is not None:
        pb.params["lmax"] = args.lmax
    L = build_layout(pb.params, pb.mask, pb.beam)
    dev = torch.device("cuda", local)
    E = engine.Engine(L, dev)
    N = torch.from_numpy(pb.noise).to(dev)
    X = qube.draw_maps(L, pb.cls, N, nsims=1, seed=0, device=dev)
    cl_tab = torch.from_numpy(L.smoothed_cl_table(pb.cls)).to(dev)
    lib = _lib.lib()

    def step(precision=args.precision, full=False):
        S = E.signal(cl_tab)
        C = S.add_(N)
        E.spd_inverse(C)
        if precision == "mixed":
            from cosmoforge_b200 import engine_mixed

            F, bias, q = engine_mixed.fisher_qml(E, C, N, X, scheme=args.scheme)
        else:
            F, bias, q = E.fisher_qml(C, N, X)
        Finv = E.spd_inverse(F.clone())
        if L.remove_nb:
            q = q - bias[None, :]
        clhat = E.gemm(q, Finv)
        return (clhat, F, Finv) if full else clhat

    tune_report = None
    if args.precision == "mixed":
        # one-time tuning of the A_b GEMM forms on this problem (cached per shape)
        from cosmoforge_b200 import autotune

        S0 = E.signal(cl_tab)
        C0 = S0.add_(N)
        E.spd_inverse(C0)
        t0 = time.perf_counter()
        forms, rep = autotune.tune_fisher(E, C0, args.scheme, use_cache=False)
        torch.cuda.synchronize()
        tune_report = {"seconds": time.perf_counter() - t0,
                       "forms": {L.spectra[k].label: {"all_planes": v[0], "kc": v[1],
                                                      "group_m": v[2] if len(v) > 2 else 16}
                                 for k, v in forms.items()}}
        del S0, C0
    for _ in range(args.warmup):
        step()
    torch.cuda.synchronize()
    E.probe = {}
    barrier()
    torch.cuda.synchronize()
    n0 = lib.cf_launch_count()
    with ClockSampler(local) as clk:
        t_start = torch.cuda.Event(enable_timing=True)
        t_end = torch.cuda.Event(enable_timing=True)
        t_start.record()
        for _ in range(args.steps):
            out = step()
        t_end.record()
        torch.cuda.synchronize()
    barrier()
    launches = (lib.cf_launch_count() - n0) // max(args.steps, 1)
    elapsed = max_over_ranks(t_start.elapsed_time(t_end) / 1e3, world, dev)
    value = job_throughput(args.steps, elapsed, world)
    clocks = clk.summary()
    tags = E.probe
    E.probe = None
    dom = "a_gemm" if args.precision == "fp64" else "a_gemm_mixed"
    recs = tags.get(dom, [])
    stage_ms = {k: round(sum(a.elapsed_time(b) for a, b, _ in v) / max(args.steps, 1), 2)
                for k, v in tags.items()}
    k_time = sum(a.elapsed_time(b) for a, b, _ in recs) / 1e3
    k_work = sum(w for _, _, w in recs)
    n_launch = max(len(recs), 1)
    assert bool(torch.isfinite(out).all())

    # ---- the same step in plain FP64, and the mixed path's error against it ----
    fp64_leg = None
    if args.precision == "mixed" and args.fp64_steps > 0:
        ch_m, F_m, _ = step("mixed", full=True)
        ch_d, F_d, Finv_d = step("fp64", full=True)
        torch.cuda.synchronize()
        barrier()
        s0, s1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        s0.record()
        for _ in range(args.fp64_steps):
            step("fp64")
        s1.record()
        torch.cuda.synchronize()
        t64 = s0.elapsed_time(s1) / 1e3
        t64 = max_over_ranks(t64, world, dev)
        dF = (F_m - F_d).abs()
        dg = torch.diagonal(F_d)
        sig = torch.diagonal(Finv_d).sqrt()
        fp64_leg = {
            "value": job_throughput(args.fp64_steps, t64, world), "unit": UNIT,
            "ms_per_step": t64 / args.fp64_steps * 1e3, "steps": args.fp64_steps,
            "mixed_over_fp64": job_throughput(args.steps, elapsed, world) / job_throughput(args.fp64_steps, t64, world),
            "mixed_error": {
                "fisher_max_rel_diag": float((torch.diagonal(dF) / dg).max()),
                "fisher_max_corr_normalised": float((dF / torch.sqrt(torch.outer(dg, dg))).max()),
                "clhat_max_shift_in_sigma": float(((ch_m - ch_d).abs() / sig[None, :]).max()),
                "targets": "|dF|/F <= 1e-5, |dC_hat| <= 1e-3 sigma",
            },
        }

    # ---- end-to-end through the public API, host inputs and outputs ----
    Nh = torch.from_numpy(pb.noise).pin_memory()
    Xh = X.cpu().pin_memory()
    h2d = Nh.numel() * 8 + Xh.numel() * 8
    e2e_times = []
    d2h = 0
    for i in range(args.e2e_steps + 1 if args.e2e_steps > 0 else 0):
        torch.cuda.synchronize()
        barrier()
        t0 = time.perf_counter()
        f = qube.Fisher(pb.params, basis=False, mask=pb.mask, noise_cov1=Nh, cls_data=pb.cls,
                        beam=pb.beam, precision=args.precision, device=dev)
        f.run()
        s = qube.Spectra(pb.params, fisher=f, maps1=Xh)
        s.run()
        clhat = s.get_power_spectra()
        torch.cuda.synchronize()
        dt = time.perf_counter() - t0
        d2h = (f.fisher.nbytes + s.qml_results.nbytes + s.qml_noise_bias.nbytes + s.invfisher.nbytes
               + clhat.nbytes)
        if i > 0:
            e2e_times.append(dt)
    t_e2e = max_over_ranks(max(e2e_times) if e2e_times else float("nan"), world, dev)
    e2e_value = job_throughput(1, t_e2e, world) if e2e_times else None

    line = None
    if rank == 0:
        import json as _json

        peaks = {}
        pk = ROOT / "MEASURED_PEAKS.json"
        if pk.exists():
            peaks = _json.loads(pk.read_text())
        if args.precision == "fp64":
            peak = fp64_peak_tflops(torch)
            peak_src = "measured cuBLAS DGEMM 8192^3 in this run (FP64 tensor)"
        else:
            # the GEMM runs inside a long step under the power cap: sustained figure
            peak = peaks.get("bf16_tflops_sustained", 1400.0)
            peak_src = ("MEASURED_PEAKS.json bf16_tflops_sustained (kernel timed inside a long step)"
                        if peaks else "fallback 1.4 PFLOP/s sustained")
        achieved = k_work / k_time / 1e12 if k_time > 0 else 0.0
        traffic = None
        tf = ROOT / "profiles" / "traffic.json"
        if tf.exists():
            traffic = _json.loads(tf.read_text()).get(f"{dom}_{args.precision}")
        cpu = None
        if not args.no_cpu_baseline and world == 1:  # the host baseline is an N = 1 figure
            pbc = workloads.config1()
            pbc.extra["maps"] = X.cpu().numpy()
            v, sample, _ = cpu_sample(pbc, L, k_params=2)
            cpu = {"value": v, "unit": UNIT, "cores": cpu_threads(), "kind": "port", "sample": sample}
        line = {
            "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": elapsed / args.steps * 1e3,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": "f64" if args.precision == "fp64" else f"{args.scheme} split products, f32 tensor accumulation, f64 promotion/reductions",
            "data": "synthetic (seeded): config-1 TQU problem, x ~ N(0, C) drawn on device",
            "config": bench_config(L), "precision": args.precision, "replicas": world,
            "e2e": {"value": e2e_value, "unit": UNIT, "h2d_bytes_per_step": int(h2d),
                    "d2h_bytes_per_step": int(d2h)},
            "stage_ms_per_step": stage_ms,
            "roofline": {"bound": "tensor", "kernel": dom, "achieved": achieved, "peak": peak,
                         "peak_source": peak_src, "unit": "TFLOP/s", "frac": achieved / peak,
                         "traffic": traffic, "launches_timed": n_launch,
                         "work_per_launch": k_work / n_launch},
            "cpu_baseline": cpu,
            "clocks": clocks,
            "gpu_launches": int(launches),
            "fp64": fp64_leg,
            "autotune": tune_report,
        }
    c0 = gpu_config0(dev)
    extra = {} if args.no_extra else secondary(args, dev)
    if line is not None:
        line["sections"] = {"config0": c0, **extra}
    if rank == 0:
        print(json.dumps(line), flush=True)
    if world > 1:
        dist.barrier()
        dist.destroy_process_group()


# --------------------------------------------------------------------------
# single-kernel timing cases (profiling commands in profiles/ use these)
# --------------------------------------------------------------------------
KERNEL_DOC = """Single-kernel timing cases (``python bench.py kernel CASE SHAPE``).

    python bench.py kernel umma_gemm M,N,K [--planes 3] [--reps 5] [--kc 16] [--form 1|2|0]
    python bench.py kernel umma_trace P1,P2,K1,K2 [--planes 3|2] [--layout flat|rows]
    python bench.py kernel dgemm M,N,K
    python bench.py kernel spd_inverse N
    python bench.py kernel harmonic 1        (config-1 harmonic-basis solve)
    python bench.py kernel map_solves NMAPS [--precision fp64|mixed]
    python bench.py kernel lnl POINTS [--precision fp64|mixed]      (config-3 likelihood batch)

Each case fills seeded random operands on cuda:0, runs two untimed launches,
then times `reps` launches with CUDA events on the launching stream and prints
one line: case, shape, ms per launch, throughput.
"""

import ctypes  # noqa: E402

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


def umma_trace_case(P1, P2, K1, K2, planes=3, splits=0, layout="flat"):
    """Closure launching one split-product trace contraction into an FP64 F.

    Three planes: the six BF16x6 products; two planes: the four products of the
    mixed Fisher's stored slabs.  layout "flat": each parameter's (k, l) block
    contiguous; "rows": the Fisher's segment buffers, X with the parameters'
    column slabs side by side along each row k (X[k][p K2 + l]), Y = their
    transposes, parameter-major (Y[q K1 + k][l])."""
    lib = _lib.lib()
    if planes == 2:
        t4 = ([0, 0, 1, 1], [0, 1, 0, 1])
        ta_ = (ctypes.c_int * 4)(*t4[0])
        tb_ = (ctypes.c_int * 4)(*t4[1])
        nt, ta, tb, keep = 4, ctypes.cast(ta_, ctypes.c_void_p), ctypes.cast(tb_, ctypes.c_void_p), (ta_, tb_)
    else:
        nt, ta, tb, keep = _terms(planes)
    g = torch.Generator(device="cuda").manual_seed(1)
    K2p = (K2 + 7) // 8 * 8
    Xp = torch.empty((planes, P1 * K1 * K2p), dtype=torch.bfloat16, device="cuda")
    Yp = torch.empty((planes, P2 * K1 * K2p), dtype=torch.bfloat16, device="cuda")
    for p in range(planes):
        Xp[p].normal_(generator=g)
        Yp[p].normal_(generator=g)
    if layout == "rows":
        sX, ldX = K2p, P1 * K2p
    else:
        sX, ldX = K1 * K2p, K2p
    F = torch.zeros((P1, P2), dtype=torch.float64, device="cuda")
    err = torch.zeros(1, dtype=torch.int32, device="cuda")
    st = torch.cuda.current_stream().cuda_stream

    def fn():
        rc = lib.cf_umma_trace_bf16(P1, P2, K1, K2, nt, ta, tb, Xp.data_ptr(), sX, ldX, P1 * K1 * K2p, planes,
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
    from cosmoforge_b200 import harmonic, qube, workloads
    from cosmoforge_b200.engine import Engine
    from cosmoforge_b200.layout import build_layout

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
    from cosmoforge_b200 import batch, qube, workloads
    from cosmoforge_b200.engine import Engine
    from cosmoforge_b200.layout import build_layout

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


def lnl_case(points, precision="mixed", build="auto"):
    """Batched likelihood of `points` Sobol points of the config-3 problem (TQU
    nside 8, n = 1312): C(theta), Cholesky factor, chi2 and ln|C| per call."""
    from cosmoforge_b200 import engine, qube, sampler, workloads
    from cosmoforge_b200.layout import build_layout

    pb = workloads.config3()
    L = build_layout(pb.params, pb.mask, pb.beam)
    E = engine.Engine(L)
    N = torch.from_numpy(pb.noise).cuda()
    x = qube.draw_maps(L, pb.cls, N, 1, seed=0)
    th = torch.as_tensor(workloads.sobol_points(points), device="cuda")
    cl = sampler.ModelTables(L, "cuda")(th)
    s = th[:, 4].contiguous()

    def fn():
        E.lnl(cl, N, x, noise_scale=s, precision=precision, build=build)

    fn._keep = (E, N, x, cl, s)
    return fn, float(points) * L.n ** 3 / 3.0, None


def kernel_main(argv=None):
    global torch, _lib
    import torch
    from cosmoforge_b200 import _lib

    ap = argparse.ArgumentParser(prog="bench.py kernel", description=KERNEL_DOC,
                                 formatter_class=argparse.RawDescriptionHelpFormatter)
    ap.add_argument("case", choices=["umma_gemm", "umma_trace", "dgemm", "spd_inverse", "harmonic",
                                           "map_solves", "lnl"])
    ap.add_argument("shape", help="comma-separated sizes")
    ap.add_argument("--planes", type=int, default=3)
    ap.add_argument("--reps", type=int, default=5)
    ap.add_argument("--kc", type=int, default=16, help="promotion interval of the tensor-core kernels")
    ap.add_argument("--splits", type=int, default=0)
    ap.add_argument("--layout", choices=["flat", "rows"], default="flat",
                    help="umma_trace: parameter-major X, or the Fisher's segment buffers")
    ap.add_argument("--precision", choices=["fp64", "mixed"], default="mixed", help="map_solves and lnl")
    ap.add_argument("--form", type=int, choices=[0, 1, 2], default=1,
                    help="tensor-core GEMM form: 1 = all planes per 32-wide k-slice, 2 = the same on CTA pairs, "
                         "0 = term by term")
    a = ap.parse_args(argv)
    dims = [int(x) for x in a.shape.split(",")]
    lib = _lib.lib()
    lib.cf_umma_set_promotion(a.kc)
    lib.cf_umma_set_all_planes(a.form)
    if a.case == "umma_gemm":
        fn, fl, err = umma_gemm_case(*dims, planes=a.planes)
    elif a.case == "umma_trace":
        fn, fl, err = umma_trace_case(*dims, planes=a.planes, splits=a.splits, layout=a.layout)
    elif a.case == "dgemm":
        fn, fl, err = dgemm_case(*dims)
    elif a.case == "harmonic":
        fn, fl, err = harmonic_case(*dims)
    elif a.case == "map_solves":
        fn, fl, err = map_solves_case(*dims, precision=a.precision)
    elif a.case == "lnl":
        fn, fl, err = lnl_case(*dims, precision=a.precision)
    else:
        fn, fl, err = spd_inverse_case(*dims)
    ms = time_launches(fn, a.reps)
    bad = int(err.item()) if err is not None else 0
    print(f"{a.case} {a.shape} planes={a.planes} kc={a.kc}: {ms:.3f} ms  {fl / ms / 1e9:.1f} TFLOP/s  err={bad}"
          if fl else f"{a.case} {a.shape} {a.precision}: {ms:.3f} ms per call")
    if bad:
        raise SystemExit("a bounded device wait ran out")



if __name__ == "__main__":
    if len(sys.argv) > 1 and sys.argv[1] == "kernel":
        kernel_main(sys.argv[2:])
    else:
        main()
