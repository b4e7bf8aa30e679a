"""Delayed-acceptance Metropolis on the pixel likelihood, emulator as stage 1.

Chains run in lock step on the device.  One *round* is
  1. `inner` emulator passes: every chain with no pending proposal draws a
     Gaussian proposal, the MLP emulator scores it and stage 1 accepts
     (the proposal becomes pending) or rejects it (a completed step);
  2. one batched exact FP64 likelihood evaluation (`Engine.lnl`) of all
     pending proposals;
  3. stage 2 accepts or rejects every pending proposal with the exact
     likelihood ratio corrected by the emulator ratio.
The chain's stationary distribution is the exact posterior (flat prior on
the box); the emulator only decides how many exact evaluations are spent.
Plain exact-likelihood Metropolis (`run_exact_mh`) is the baseline.

Two-level form (`run_da_subchain`): a round runs J Metropolis steps of every
chain on the emulator posterior (a sub-chain reversible with respect to it),
then one batched exact evaluation decides on each sub-chain's end point as the
exact chain's proposal with the same corrected ratio (the surrogate-transition
method of J. S. Liu, Monte Carlo Strategies in Scientific Computing, 2001,
9.4.3; multilevel delayed acceptance, Lykkegaard et al., SIAM/ASA JUQ 11,
2023).  One exact evaluation per chain and round buys J emulator moves, so
successive exact-chain points are nearly independent once J exceeds the
emulator chain's autocorrelation time; the gain is measured as effective
samples per second (`effective_sample_size`).

C_l(theta) of the five-parameter model (amplitude A, tilt n, reionisation
bump h, BB/EE ratio r, noise scale s) is built on the device from theta, so
a round needs no host round trip.  No counterpart in the reference (which
has no sampler).
"""

from __future__ import annotations

import time

import numpy as np
import torch

from . import workloads
from ._lib import check, lib, stream

F64 = torch.float64


class ModelTables:
    """Beam-smoothed C_l tables of :func:`workloads.model_cls` for a batch of theta, on the device."""

    def __init__(self, layout, device=None):
        self.dev = torch.device(device or "cuda")
        L = layout.lmax_signal
        sh = workloads.tqu_shapes(L)
        ell = np.arange(L + 1, dtype=np.float64)
        self.logl = torch.as_tensor(np.log(np.maximum(ell, 1.0) / workloads.PIVOT_ELL), device=self.dev)
        self.lmask = torch.as_tensor((ell >= 2).astype(np.float64), device=self.dev)
        self.bump = torch.as_tensor(workloads.reion_bump(L), device=self.dev)
        self.labels = [s.label for s in layout.spectra]
        self.base = {k: torch.as_tensor(v, device=self.dev) for k, v in sh.items()}
        self.smooth = torch.as_tensor(np.stack([layout.smoothing(s) for s in layout.spectra]), device=self.dev)

    def __call__(self, theta):
        th = torch.as_tensor(theta, dtype=F64, device=self.dev)
        A, n, h, r = th[:, 0:1], th[:, 1:2], th[:, 2:3], th[:, 3:4]
        t = A * torch.exp(n * self.logl) * self.lmask
        ee = (t * self.base["EE"] + h * self.bump) * self.lmask
        cls = {"TT": t * self.base["TT"], "EE": ee, "BB": r * ee, "TE": t * self.base["TE"]}
        zero = torch.zeros_like(t)
        tab = torch.stack([cls.get(lab, zero) for lab in self.labels], dim=1)
        return tab * self.smooth[None]


def exact_m2lnl(E, tables, N, X, theta):
    """-2 lnL (FP64) of a batch of points: C = S(theta) + s N, one map column."""
    th = torch.as_tensor(theta, dtype=F64, device=E.dev)
    chi2, logdet, lnl, info = E.lnl(tables(th), N, X, noise_scale=th[:, 4].contiguous())
    return -2.0 * lnl[:, 0], info


def training_set(E, tables, N, X, n_points: int, seed: int = 0, batch: int = 1024):
    """(theta, -2 lnL) at n_points scrambled-Sobol points of the box, exact FP64."""
    th = workloads.sobol_points(n_points, seed=seed)
    out = []
    for b0 in range(0, n_points, batch):
        m2, info = exact_m2lnl(E, tables, N, X, th[b0:b0 + batch])
        if int(info.abs().max()) != 0:
            raise ValueError("non positive-definite covariance in the training set")
        out.append(m2)
    return th, torch.cat(out)


def fisher_theta(E, tables, N, theta0, rel_step: float = 1e-3):
    """Fisher matrix in theta at theta0 from finite differences of C(theta).

    F_ab = 1/2 Tr(C^-1 dC_a C^-1 dC_b), dC_a = [C(theta + h_a e_a) - C(theta - h_a e_a)] / 2 h_a,
    with the noise scale entering as C = S + s N.
    """
    th0 = np.asarray(theta0, np.float64)
    D = th0.size
    span = workloads.THETA_HI - workloads.THETA_LO
    pts = [th0]
    for a in range(D):
        for sgn in (1.0, -1.0):
            p = th0.copy()
            p[a] += sgn * rel_step * span[a]
            pts.append(p)
    pts = torch.as_tensor(np.stack(pts), device=E.dev)
    C = E.signal(tables(pts))
    C += pts[:, 4, None, None] * N[None]
    Cinv = E.spd_inverse(C[0].clone())
    A = []
    for a in range(D):
        dC = (C[1 + 2 * a] - C[2 + 2 * a]) / (2.0 * rel_step * span[a])
        A.append(E.gemm(Cinv, dC))
    F = np.zeros((D, D))
    for a in range(D):
        for b in range(a, D):
            F[a, b] = F[b, a] = 0.5 * float(torch.sum(A[a] * A[b].T))
    return F


def proposal_cov(F, scale: float | None = None, box_frac: float = 0.25):
    """Gaussian proposal covariance from the Fisher matrix F in theta.

    The Fisher covariance F^-1 keeps its correlations, each standard deviation
    is capped at box_frac of the parameter's prior span (a parameter the data
    barely constrain would otherwise propose far outside the box), and the
    result is scaled by `scale` (default 2.38^2 / D).
    """
    cov = np.linalg.inv(np.asarray(F, np.float64))
    D = cov.shape[0]
    sig = np.sqrt(np.diag(cov))
    corr = cov / np.outer(sig, sig)
    sig = np.minimum(sig, box_frac * (workloads.THETA_HI - workloads.THETA_LO))
    scale = 2.38 ** 2 / D if scale is None else scale
    return scale * corr * np.outer(sig, sig)


def effective_sample_size(samples, burn: int = 0):
    """Per-parameter ESS of C chains (C x steps x D) from the integrated autocorrelation
    time of the chain-averaged autocovariance (Geyer's initial positive sequence)."""
    x = np.asarray(samples, np.float64)[:, burn:]
    C, T, D = x.shape
    x = x - x.mean(axis=1, keepdims=True)
    out = np.zeros(D)
    for d in range(D):
        f = np.fft.rfft(x[:, :, d], n=2 * T, axis=1)
        ac = np.fft.irfft(f * np.conj(f), axis=1)[:, :T].mean(axis=0)
        if ac[0] <= 0:
            out[d] = C * T
            continue
        rho = ac / ac[0]
        tau = 1.0
        for k in range(1, T - 1, 2):
            pair = rho[k] + rho[k + 1]
            if pair <= 0:
                break
            tau += 2.0 * pair
        out[d] = C * T / tau
    return out


class Chains:
    """State of C chains in D dimensions (all on the device)."""

    def __init__(self, C, D, max_steps, theta0, dev):
        def z():
            return torch.zeros(C, dtype=F64, device=dev)

        self.C, self.D, self.max_steps = C, D, max_steps
        self.theta = torch.as_tensor(theta0, dtype=F64, device=dev).clone()
        self.theta_p = self.theta.clone()
        self.xin = torch.zeros((C, D), dtype=torch.float32, device=dev)
        self.active = torch.zeros(C, dtype=torch.int32, device=dev)
        self.pending = torch.zeros(C, dtype=torch.int32, device=dev)
        self.steps = torch.zeros(C, dtype=torch.int32, device=dev)
        self.n_stage1 = torch.zeros(C, dtype=torch.int32, device=dev)
        self.n_exact = torch.zeros(C, dtype=torch.int32, device=dev)
        self.n_accept = torch.zeros(C, dtype=torch.int32, device=dev)
        self.n_sub = torch.zeros(C, dtype=torch.int32, device=dev)
        self.lexact = z()
        self.lexact_p = z()
        self.ltil = z()
        self.ltil_p = z()
        self.samples = torch.zeros((C, max_steps, D), dtype=F64, device=dev)

    def stats(self):
        steps = int(self.steps.sum())
        return dict(steps=steps, exact_evals=int(self.n_exact.sum()), stage1_accepted=int(self.n_stage1.sum()),
                    accepted=int(self.n_accept.sum()), sub_accepted=int(self.n_sub.sum()))


class Sampler:
    def __init__(self, E, N, X, emulator=None, prop_cov=None, seed: int = 0):
        self.E, self.N, self.X = E, N, X
        self.dev = E.dev
        self.lib = lib()
        self.tables = ModelTables(E.L, self.dev)
        self.emu = emulator
        self.lo = torch.as_tensor(workloads.THETA_LO, device=self.dev)
        self.hi = torch.as_tensor(workloads.THETA_HI, device=self.dev)
        self.Lp = torch.as_tensor(np.linalg.cholesky(np.asarray(prop_cov, np.float64)), device=self.dev).contiguous()
        self.gen = torch.Generator(device=self.dev)
        self.gen.manual_seed(seed)

    def _start(self, C, max_steps, theta0):
        D = self.Lp.shape[0]
        if theta0 is None:
            c = torch.as_tensor(workloads.THETA_CENTRE, device=self.dev)
            theta0 = c[None] + 0.1 * torch.randn((C, D), dtype=F64, device=self.dev, generator=self.gen) @ self.Lp.T
            theta0 = torch.minimum(torch.maximum(theta0, self.lo), self.hi)
        ch = Chains(C, D, max_steps, theta0, self.dev)
        m2, _ = exact_m2lnl(self.E, self.tables, self.N, self.X, ch.theta)
        ch.lexact.copy_(-0.5 * m2)
        if self.emu is not None:
            ch.ltil.copy_(-0.5 * self.emu.predict_m2lnl(ch.theta))
        return ch

    def _propose(self, ch, xi):
        check(self.lib.cf_mcmc_propose(ch.C, ch.D, ch.theta.data_ptr(), ch.pending.data_ptr(), ch.steps.data_ptr(),
                                       ch.max_steps, self.Lp.data_ptr(), xi.data_ptr(), self.lo.data_ptr(),
                                       self.hi.data_ptr(), ch.theta_p.data_ptr(), ch.xin.data_ptr(),
                                       ch.active.data_ptr(), stream()), "cf_mcmc_propose")

    def _exact_at(self, ch, which):
        """Exact lnL at theta_p where `which` is set, at the current point elsewhere."""
        th = torch.where(which[:, None] != 0, ch.theta_p, ch.theta)
        m2, _ = exact_m2lnl(self.E, self.tables, self.N, self.X, th)
        ch.lexact_p.copy_(-0.5 * m2)

    def _da_round(self, ch, xi, u1, u2, inner):
        C, D, emu = ch.C, ch.D, self.emu
        for i in range(inner):
            self._propose(ch, xi[i])
            y = emu.predict_std(ch.xin)
            check(self.lib.cf_mcmc_stage1(C, D, ch.active.data_ptr(), y.data_ptr(), emu.mu, emu.sigma,
                                          u1[i].data_ptr(), ch.theta.data_ptr(), ch.ltil.data_ptr(),
                                          ch.ltil_p.data_ptr(), ch.pending.data_ptr(), ch.steps.data_ptr(),
                                          ch.samples.data_ptr(), ch.max_steps, ch.n_stage1.data_ptr(),
                                          stream()), "cf_mcmc_stage1")
        self._exact_at(ch, ch.pending)
        check(self.lib.cf_mcmc_stage2(C, D, ch.lexact_p.data_ptr(), ch.lexact.data_ptr(), ch.ltil.data_ptr(),
                                      ch.ltil_p.data_ptr(), u2.data_ptr(), ch.theta.data_ptr(),
                                      ch.theta_p.data_ptr(), ch.pending.data_ptr(), ch.steps.data_ptr(),
                                      ch.samples.data_ptr(), ch.max_steps, ch.n_exact.data_ptr(),
                                      ch.n_accept.data_ptr(), stream()), "cf_mcmc_stage2")

    def _emulator_shape(self):
        """Hidden-layer count of the emulator for the fused sub-chain kernel (widths 256)."""
        emu = self.emu
        sz = emu.sizes
        if sz[0] != self.Lp.shape[0] or sz[-1] != 1 or any(w != 256 for w in sz[1:-1]) or len(sz) < 3:
            raise ValueError(f"fused sub-chain kernel needs sizes (D, 256, ..., 256, 1), got {sz}")
        if not (torch.equal(emu.lo, self.lo) and torch.equal(emu.hi, self.hi)):
            raise ValueError("emulator and sampler must share the prior box")
        return len(sz) - 2

    def _sub_round(self, ch, theta_s, ltil_s, zeros, xi, u1, u2, J, n_hidden=None):
        C, D, emu = ch.C, ch.D, self.emu
        if n_hidden is not None:
            check(self.lib.cf_mcmc_subchain(C, D, J, n_hidden, ch.theta.data_ptr(), ch.steps.data_ptr(),
                                            ch.max_steps, self.Lp.data_ptr(), xi.data_ptr(), u1.data_ptr(),
                                            self.lo.data_ptr(), self.hi.data_ptr(), emu.p16.data_ptr(),
                                            emu.p.data_ptr(), emu.mu, emu.sigma, theta_s.data_ptr(),
                                            ch.ltil.data_ptr(), ltil_s.data_ptr(), ch.n_sub.data_ptr(), stream()),
                  "cf_mcmc_subchain")
        for j in range(J if n_hidden is None else 0):
            check(self.lib.cf_mcmc_propose(C, D, theta_s.data_ptr(), zeros.data_ptr(), ch.steps.data_ptr(),
                                           ch.max_steps, self.Lp.data_ptr(), xi[j].data_ptr(), self.lo.data_ptr(),
                                           self.hi.data_ptr(), ch.theta_p.data_ptr(), ch.xin.data_ptr(),
                                           ch.active.data_ptr(), stream()), "cf_mcmc_propose")
            y = emu.predict_std(ch.xin)
            check(self.lib.cf_mcmc_sub_accept(C, D, ch.active.data_ptr(), y.data_ptr(), emu.mu, emu.sigma,
                                              u1[j].data_ptr(), ch.theta_p.data_ptr(), theta_s.data_ptr(),
                                              ltil_s.data_ptr(), ch.n_sub.data_ptr(), stream()),
                  "cf_mcmc_sub_accept")
        m2, _ = exact_m2lnl(self.E, self.tables, self.N, self.X, theta_s)
        ch.lexact_p.copy_(-0.5 * m2)
        check(self.lib.cf_mcmc_sub_final(C, D, ch.lexact_p.data_ptr(), ch.lexact.data_ptr(), ch.ltil.data_ptr(),
                                         ltil_s.data_ptr(), u2.data_ptr(), ch.theta.data_ptr(), theta_s.data_ptr(),
                                         ch.steps.data_ptr(), ch.samples.data_ptr(), ch.max_steps,
                                         ch.n_exact.data_ptr(), ch.n_accept.data_ptr(), stream()),
              "cf_mcmc_sub_final")

    def run_da_subchain(self, n_chains: int, n_steps: int, sub_steps: int = 128, theta0=None, graph: bool = True,
                        fused: bool = True):
        """Two-level delayed acceptance: `sub_steps` emulator Metropolis steps per
        exact evaluation; one recorded step per exact evaluation of each chain.
        fused: the whole sub-chain of every chain in one launch
        (`cf_mcmc_subchain`), else one proposal / emulator / acceptance
        launch sequence per sub-step."""
        if self.emu is None:
            raise ValueError("delayed acceptance needs an emulator")
        if sub_steps < 1:
            raise ValueError("sub_steps must be >= 1")
        nh = self._emulator_shape() if fused else None
        ch = self._start(n_chains, n_steps, theta0)
        C, D, J = ch.C, ch.D, sub_steps
        theta_s = ch.theta.clone()
        ltil_s = ch.ltil.clone()
        zeros = torch.zeros(C, dtype=torch.int32, device=self.dev)
        xi = torch.empty((J, C, D), dtype=F64, device=self.dev)
        u1 = torch.empty((J, C), dtype=F64, device=self.dev)
        u2 = torch.empty(C, dtype=F64, device=self.dev)

        def rand():
            xi.normal_(generator=self.gen)
            u1.uniform_(generator=self.gen)
            u2.uniform_(generator=self.gen)

        torch.cuda.synchronize()
        t0 = time.perf_counter()
        rounds = self._loop(lambda: self._sub_round(ch, theta_s, ltil_s, zeros, xi, u1, u2, J, nh), rand, graph,
                            lambda r: r >= n_steps)
        torch.cuda.synchronize()
        st = ch.stats()
        st.update(seconds=time.perf_counter() - t0, rounds=rounds, sub_steps=J)
        return ch, st

    def _mh_step(self, ch, xi, u):
        self._propose(ch, xi)
        self._exact_at(ch, (ch.active == 1).to(torch.int32))
        check(self.lib.cf_mcmc_mh_accept(ch.C, ch.D, ch.active.data_ptr(), ch.lexact_p.data_ptr(),
                                         ch.lexact.data_ptr(), u.data_ptr(), ch.theta.data_ptr(),
                                         ch.theta_p.data_ptr(), ch.steps.data_ptr(), ch.samples.data_ptr(),
                                         ch.max_steps, ch.n_exact.data_ptr(), ch.n_accept.data_ptr(),
                                         stream()), "cf_mcmc_mh_accept")

    def _loop(self, body, rand, graph, done):
        """Run body() until done(); random buffers are refilled by rand() before
        every call.  With graph, the first call runs eagerly and one captured
        call is replayed after it."""
        g = None
        rounds = 0
        while True:
            rand()
            if g is not None:
                g.replay()
            else:
                body()
                if graph:
                    g = torch.cuda.CUDAGraph()
                    with torch.cuda.graph(g):
                        body()
            rounds += 1
            if done(rounds):
                break
        return rounds

    def run_da(self, n_chains: int, n_steps: int, inner: int = 8, theta0=None, max_rounds: int | None = None,
               graph: bool = True):
        """Delayed-acceptance chains; returns (Chains, stats dict with timing)."""
        if self.emu is None:
            raise ValueError("delayed acceptance needs an emulator")
        ch = self._start(n_chains, n_steps, theta0)
        C, D = ch.C, ch.D
        xi = torch.empty((inner, C, D), dtype=F64, device=self.dev)
        u1 = torch.empty((inner, C), dtype=F64, device=self.dev)
        u2 = torch.empty(C, dtype=F64, device=self.dev)

        def rand():
            xi.normal_(generator=self.gen)
            u1.uniform_(generator=self.gen)
            u2.uniform_(generator=self.gen)

        def done(r):
            if max_rounds is not None and r >= max_rounds:
                return True
            return r % 4 == 0 and int(ch.steps.min()) >= n_steps

        torch.cuda.synchronize()
        t0 = time.perf_counter()
        rounds = self._loop(lambda: self._da_round(ch, xi, u1, u2, inner), rand, graph, done)
        torch.cuda.synchronize()
        st = ch.stats()
        st.update(seconds=time.perf_counter() - t0, rounds=rounds)
        return ch, st

    def run_exact_mh(self, n_chains: int, n_steps: int, theta0=None, graph: bool = True):
        """Plain Metropolis with the exact likelihood at every step (the baseline)."""
        ch = self._start(n_chains, n_steps, theta0)
        C, D = ch.C, ch.D
        xi = torch.empty((C, D), dtype=F64, device=self.dev)
        u = torch.empty(C, dtype=F64, device=self.dev)

        def rand():
            xi.normal_(generator=self.gen)
            u.uniform_(generator=self.gen)

        torch.cuda.synchronize()
        t0 = time.perf_counter()
        rounds = self._loop(lambda: self._mh_step(ch, xi, u), rand, graph, lambda r: r >= n_steps)
        torch.cuda.synchronize()
        st = ch.stats()
        st.update(seconds=time.perf_counter() - t0, rounds=rounds)
        return ch, st
