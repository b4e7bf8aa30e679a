"""Emulator training kernels and the delayed-acceptance sampler on the GPU.

* Device gradients (FP32 accumulation, BF16 weight matrices) against the FP64
  CPU oracle on the same BF16 weights: relative 2e-4 of the largest entry.
* Adam against its closed form; a graph-captured training run equals the
  eager one bit for bit.
* On the config-3 likelihood: the trained network's stage 1 lets the sampler
  spend fewer exact evaluations per step than plain exact Metropolis, with a
  high stage-2 acceptance that an untrained network does not reach, and both
  samplers agree on the posterior mean.
* Two-level form: the sub-chain kernels against a NumPy restatement of the
  round, the fused sub-chain kernel against the FP64 network and against one
  launch per step; on config 3 the sampler matches exact Metropolis' posterior mean and
  width and buys more effective samples per exact evaluation.
"""

import numpy as np
import pytest
import torch

from cosmoforge_b200 import workloads
from cosmoforge_b200.layout import build_layout
from oracle import mlp_oracle

pytestmark = pytest.mark.gpu

GRAD_REL = 2e-4


def _emu(seed=0):
    from cosmoforge_b200.emulator import MLPEmulator

    return MLPEmulator(workloads.THETA_LO, workloads.THETA_HI, seed=seed)


@pytest.mark.parametrize("M", [300, 1024])
def test_mlp_gradient_matches_oracle(M):
    emu = _emu(3)
    rng = np.random.default_rng(M)
    X = rng.uniform(-1, 1, (M, 5)).astype(np.float32)
    t = rng.normal(0, 1, M).astype(np.float32)
    loss, g = emu.loss_and_grad(torch.from_numpy(X).cuda(), torch.from_numpy(t).cuda())
    p16 = emu.p16.float().cpu().numpy().astype(np.float64)
    p32 = emu.p.cpu().numpy().astype(np.float64)
    ref_loss, ref_g = mlp_oracle.loss_and_grad(p16, p32, emu.sizes, X, t)
    g = g.cpu().numpy()
    err = np.max(np.abs(g - ref_g)) / np.max(np.abs(ref_g))
    print(f"M={M}: loss {loss:.6e} vs {ref_loss:.6e}, grad rel {err:.2e}")
    assert abs(loss - ref_loss) <= 1e-5 * ref_loss
    assert err <= GRAD_REL


def test_adam_matches_closed_form():
    from cosmoforge_b200 import _lib

    lib = _lib.lib()
    n = 1000
    rng = np.random.default_rng(1)
    p0 = rng.normal(0, 1, n).astype(np.float32)
    grads = [rng.normal(0, 1, n).astype(np.float32) for _ in range(3)]
    p = torch.from_numpy(p0.copy()).cuda()
    m = torch.zeros_like(p)
    v = torch.zeros_like(p)
    step = torch.zeros(1, dtype=torch.int32, device="cuda")
    p16 = torch.empty(n, dtype=torch.bfloat16, device="cuda")
    lr, b1, b2, eps = 1e-3, 0.9, 0.999, 1e-8
    rp, rm, rv = p0.astype(np.float64), np.zeros(n), np.zeros(n)
    for k, gk in enumerate(grads, start=1):
        g = torch.from_numpy(gk).cuda()
        assert lib.cf_mlp_adam(n, p.data_ptr(), g.data_ptr(), m.data_ptr(), v.data_ptr(), lr, b1, b2, eps,
                               step.data_ptr(), p16.data_ptr(), torch.cuda.current_stream().cuda_stream) == 0
        rm = b1 * rm + (1 - b1) * gk
        rv = b2 * rv + (1 - b2) * gk.astype(np.float64) ** 2
        rp = rp - lr * (rm / (1 - b1 ** k)) / (np.sqrt(rv / (1 - b2 ** k)) + eps)
    assert int(step.item()) == 3
    assert np.max(np.abs(p.cpu().numpy() - rp)) <= 1e-6
    assert torch.equal(p16, p.to(torch.bfloat16))


def test_graph_training_equals_eager():
    rng = np.random.default_rng(2)
    th = workloads.THETA_LO + rng.uniform(0, 1, (4096, 5)) * (workloads.THETA_HI - workloads.THETA_LO)
    u = (th - workloads.THETA_CENTRE) / (workloads.THETA_HI - workloads.THETA_LO)
    y = 50.0 * np.sum(u ** 2, axis=1) + 10.0 * u[:, 0] * u[:, 1]
    a, b = _emu(5), _emu(5)
    ha = a.fit(th, y, steps=120, batch=512, graph=True)
    hb = b.fit(th, y, steps=120, batch=512, graph=False)
    assert torch.equal(a.p, b.p)
    assert ha[-1][1] < 0.5 * ha[0][1]
    assert hb == ha


@pytest.fixture(scope="module")
def config3():
    from cosmoforge_b200 import engine, qube, sampler

    pb = workloads.config3()
    L = build_layout(pb.params, pb.mask, pb.beam)
    E = engine.Engine(L)
    N = torch.from_numpy(pb.noise).cuda()
    X = qube.draw_maps(L, pb.cls, N, 1, seed=0)
    tables = sampler.ModelTables(L)
    return E, N, X, tables


def test_device_tables_match_model(config3):
    E, N, X, tables = config3
    th = workloads.sobol_points(16, seed=3)
    dev = tables(th).cpu().numpy()
    ref = np.stack([E.L.smoothed_cl_table(workloads.model_cls(t, E.L.lmax_signal)) for t in th])
    assert np.max(np.abs(dev - ref)) <= 1e-13 * np.max(np.abs(ref))


@pytest.fixture(scope="module")
def trained(config3):
    from cosmoforge_b200 import sampler

    E, N, X, tables = config3
    th, m2 = sampler.training_set(E, tables, N, X, 8192, seed=0)
    emu = _emu(0)
    emu.fit(th, m2, steps=1500, batch=1024)
    F = sampler.fisher_theta(E, tables, N, workloads.THETA_CENTRE)
    return emu, F


def _sub_round_restated(theta, ltil, lexact, Lp, xi, u1, y_of, u2, lexact_of, lo, hi, mu, sigma):
    """One two-level round in NumPy: J emulator Metropolis steps from theta,
    then the exact decision on the end point (the kernels' specification)."""
    C, D = theta.shape
    ts, ls = theta.copy(), ltil.copy()
    for j in range(xi.shape[0]):
        tp = ts + xi[j] @ Lp.T
        inside = np.all((tp >= lo) & (tp <= hi), axis=1)
        lp = -0.5 * (mu + sigma * y_of(j, tp).astype(np.float64))
        acc = inside & (np.log(u1[j]) < lp - ls)
        ts[acc], ls[acc] = tp[acc], lp[acc]
    le_p = lexact_of(ts)
    acc = np.log(u2) < (le_p - lexact) - (ls - ltil)
    th, lt, le = theta.copy(), ltil.copy(), lexact.copy()
    th[acc], lt[acc], le[acc] = ts[acc], ls[acc], le_p[acc]
    return th, lt, le, acc


def test_subchain_kernels_match_restatement():
    """cf_mcmc_propose / cf_mcmc_sub_accept / cf_mcmc_sub_final against the
    NumPy restatement, with a closed-form stand-in for both likelihoods."""
    from cosmoforge_b200 import _lib

    lib = _lib.lib()
    st = torch.cuda.current_stream().cuda_stream
    rng = np.random.default_rng(11)
    C, D, J, T = 64, 5, 6, 4
    lo, hi = workloads.THETA_LO, workloads.THETA_HI
    span = hi - lo
    A = rng.normal(0, 1, (D, D))
    Lp = np.linalg.cholesky(0.02 * np.diag(span ** 2) + 1e-4 * A @ A.T * np.outer(span, span))
    mu, sigma = 3.0, 2.0

    def quad(t):
        return np.sum(((t - workloads.THETA_CENTRE) / (0.2 * span)) ** 2, axis=1)

    def y_of(j, t):  # standardised emulator output -2 lnL~, FP32
        return ((quad(t) - mu) / sigma).astype(np.float32)

    def lexact_of(t):  # "exact" lnL differs from the emulator by a smooth term
        return -0.5 * quad(t) + 0.05 * np.sin(t @ np.arange(1, D + 1))

    theta = workloads.THETA_CENTRE + 0.05 * rng.normal(0, 1, (C, D)) * span
    ltil = -0.5 * (mu + sigma * y_of(0, theta).astype(np.float64))
    lexact = lexact_of(theta)
    dev = lambda a, dt=torch.float64: torch.as_tensor(np.ascontiguousarray(a), dtype=dt, device="cuda")
    d_theta, d_ltil, d_lexact = dev(theta), dev(ltil), dev(lexact)
    d_ts, d_ls = d_theta.clone(), d_ltil.clone()
    d_Lp, d_lo, d_hi = dev(Lp), dev(lo), dev(hi)
    zeros = torch.zeros(C, dtype=torch.int32, device="cuda")
    steps = torch.zeros(C, dtype=torch.int32, device="cuda")
    tp = torch.empty((C, D), dtype=torch.float64, device="cuda")
    xin = torch.empty((C, D), dtype=torch.float32, device="cuda")
    active = torch.empty(C, dtype=torch.int32, device="cuda")
    n_sub, n_exact, n_acc = (torch.zeros(C, dtype=torch.int32, device="cuda") for _ in range(3))
    samples = torch.zeros((C, T, D), dtype=torch.float64, device="cuda")
    lexact_p = torch.empty(C, dtype=torch.float64, device="cuda")
    h_theta, h_ltil, h_lexact = theta.copy(), ltil.copy(), lexact.copy()
    n_acc_ref = np.zeros(C, int)
    for r in range(T):
        xi = rng.normal(0, 1, (J, C, D))
        xi[:, :4] *= 30.0  # some proposals leave the box
        u1, u2 = rng.uniform(size=(J, C)), rng.uniform(size=C)
        for j in range(J):
            assert lib.cf_mcmc_propose(C, D, d_ts.data_ptr(), zeros.data_ptr(), steps.data_ptr(), T,
                                       d_Lp.data_ptr(), dev(xi[j]).data_ptr(), d_lo.data_ptr(), d_hi.data_ptr(),
                                       tp.data_ptr(), xin.data_ptr(), active.data_ptr(), st) == 0
            y = dev(y_of(j, tp.cpu().numpy()), torch.float32)
            assert lib.cf_mcmc_sub_accept(C, D, active.data_ptr(), y.data_ptr(), mu, sigma, dev(u1[j]).data_ptr(),
                                          tp.data_ptr(), d_ts.data_ptr(), d_ls.data_ptr(), n_sub.data_ptr(),
                                          st) == 0
        lexact_p.copy_(dev(lexact_of(d_ts.cpu().numpy())))
        assert lib.cf_mcmc_sub_final(C, D, lexact_p.data_ptr(), d_lexact.data_ptr(), d_ltil.data_ptr(),
                                     d_ls.data_ptr(), dev(u2).data_ptr(), d_theta.data_ptr(), d_ts.data_ptr(),
                                     steps.data_ptr(), samples.data_ptr(), T, n_exact.data_ptr(),
                                     n_acc.data_ptr(), st) == 0
        h_theta, h_ltil, h_lexact, acc = _sub_round_restated(h_theta, h_ltil, h_lexact, Lp, xi, u1, y_of, u2,
                                                             lexact_of, lo, hi, mu, sigma)
        n_acc_ref += acc
        got = d_theta.cpu().numpy()
        assert np.max(np.abs(got - h_theta) / span) <= 1e-14, r
        np.testing.assert_allclose(d_ltil.cpu().numpy(), h_ltil, rtol=0, atol=1e-9)
        assert torch.equal(d_ts, d_theta) and torch.equal(d_ls, d_ltil)
        assert np.max(np.abs(samples[:, r].cpu().numpy() - h_theta) / span) <= 1e-14
    assert torch.equal(n_acc.cpu(), torch.as_tensor(n_acc_ref, dtype=torch.int32))
    assert int(n_exact.sum()) == C * T and int(steps.min()) == T
    assert 0 < int(n_sub.sum()) < C * J * T


def test_fused_subchain_kernel(trained):
    """cf_mcmc_subchain: its emulator value against the training kernels' forward
    and the FP64 oracle; J fused steps equal J one-step launches bit for bit;
    every step's decision equals the restated one (FP64 oracle network) where
    the acceptance margin exceeds the FP32 forward's error."""
    from cosmoforge_b200 import _lib, sampler

    emu, F = trained
    lib = _lib.lib()
    st = torch.cuda.current_stream().cuda_stream
    C, D, J = 64, 5, 8
    rng = np.random.default_rng(21)
    prop = sampler.proposal_cov(F)
    Lp = np.linalg.cholesky(prop)
    lo, hi = workloads.THETA_LO, workloads.THETA_HI
    theta = np.clip(rng.multivariate_normal(workloads.THETA_CENTRE, 0.5 * prop, C), lo, hi)
    xi = rng.normal(0, 1, (J, C, D))
    u = rng.uniform(size=(J, C))
    dev = lambda a: torch.as_tensor(np.ascontiguousarray(a), dtype=torch.float64, device="cuda")
    d_Lp, d_lo, d_hi, d_xi, d_u = dev(Lp), dev(lo), dev(hi), dev(xi), dev(u)
    steps = torch.zeros(C, dtype=torch.int32, device="cuda")

    def run(th, J_, xi_, u_):
        ts = torch.empty((C, D), dtype=torch.float64, device="cuda")
        lt, ls = (torch.empty(C, dtype=torch.float64, device="cuda") for _ in range(2))
        ns = torch.zeros(C, dtype=torch.int32, device="cuda")
        assert lib.cf_mcmc_subchain(C, D, J_, 3, th.data_ptr(), steps.data_ptr(), 10, d_Lp.data_ptr(),
                                    xi_.data_ptr(), u_.data_ptr(), d_lo.data_ptr(), d_hi.data_ptr(),
                                    emu.p16.data_ptr(), emu.p.data_ptr(), emu.mu, emu.sigma, ts.data_ptr(),
                                    lt.data_ptr(), ls.data_ptr(), ns.data_ptr(), st) == 0
        return ts, lt, ls, ns

    layers = mlp_oracle.unpack(np.concatenate([
        np.concatenate([emu.p16.float().cpu().numpy()[w:b], emu.p.cpu().numpy()[b:b + n_out]])
        for (w, b, n_in, n_out) in emu.layout]).astype(np.float64), emu.sizes)

    def y64(t):
        x = 2.0 * (t - lo) / (hi - lo) - 1.0
        return mlp_oracle.forward(layers, x.astype(np.float32).astype(np.float64))[1][-1][:, 0]

    d_th = dev(theta)
    _, lt0, _, _ = run(d_th, 0, d_xi, d_u)
    ref_train = -0.5 * emu.predict_m2lnl(d_th)
    ref64 = -0.5 * (emu.mu + emu.sigma * y64(theta))
    tol = 2e-5 * emu.sigma
    print(f"sigma {emu.sigma:.3e}: |d ltil| vs training forward {float((lt0 - ref_train).abs().max()):.2e}, "
          f"vs FP64 {np.max(np.abs(lt0.cpu().numpy() - ref64)):.2e}")
    assert float((lt0 - ref_train).abs().max()) <= tol
    assert np.max(np.abs(lt0.cpu().numpy() - ref64)) <= tol

    ts_f, lt_f, ls_f, ns_f = run(d_th, J, d_xi, d_u)
    assert torch.equal(lt_f, lt0)
    th = d_th
    compared = n_inside = 0
    ns_total = torch.zeros_like(ns_f)
    for j in range(J):
        ts, lt, ls, ns = run(th, 1, d_xi[j:j + 1].contiguous(), d_u[j:j + 1].contiguous())
        ns_total += ns
        t_np, ts_np = th.cpu().numpy(), ts.cpu().numpy()
        tp = t_np + xi[j] @ Lp.T
        inside = np.all((tp >= lo) & (tp <= hi), axis=1)
        lr = -0.5 * emu.sigma * (y64(tp) - y64(t_np))
        moved = np.any(ts_np != t_np, axis=1)
        clear = inside & (np.abs(np.log(u[j]) - lr) > 2 * tol)
        assert not np.any(moved & ~inside)
        np.testing.assert_array_equal(moved[clear], (np.log(u[j]) < lr)[clear])
        np.testing.assert_allclose(ts_np[moved], tp[moved], rtol=1e-14, atol=0)
        compared += int(clear.sum())
        n_inside += int(inside.sum())
        th = ts
    print(f"{compared} of {n_inside} in-box decisions compared, {int(ns_f.sum())} accepted")
    assert compared >= 0.9 * n_inside and n_inside >= J * C // 4
    assert torch.equal(th, ts_f) and torch.equal(ls, ls_f) and torch.equal(ns_total, ns_f)
    assert 0 < int(ns_f.sum()) < J * C


def test_delayed_acceptance_saves_exact_evaluations(config3, trained):
    from cosmoforge_b200 import sampler

    E, N, X, tables = config3
    emu, F = trained
    # held-out accuracy near the posterior
    cov = np.linalg.inv(F)
    rng = np.random.default_rng(7)
    pts = rng.multivariate_normal(workloads.THETA_CENTRE, cov, 512)
    pts = np.clip(pts, workloads.THETA_LO, workloads.THETA_HI)
    ex, _ = sampler.exact_m2lnl(E, tables, N, X, pts)
    em = emu.predict_m2lnl(pts)
    d = (em - ex) - (em - ex).mean()
    rms = float(0.5 * d.pow(2).mean().sqrt())
    print(f"emulator RMS Delta lnL near the posterior: {rms:.3f}")

    prop = sampler.proposal_cov(F)
    n_chains, n_steps = 64, 120
    s_da = sampler.Sampler(E, N, X, emulator=emu, prop_cov=prop, seed=1)
    ch_da, st_da = s_da.run_da(n_chains, n_steps)
    s_mh = sampler.Sampler(E, N, X, prop_cov=prop, seed=2)
    ch_mh, st_mh = s_mh.run_exact_mh(n_chains, n_steps)
    untrained = _emu(9)
    untrained.mu, untrained.sigma = emu.mu, emu.sigma
    s_un = sampler.Sampler(E, N, X, emulator=untrained, prop_cov=prop, seed=3)
    _, st_un = s_un.run_da(n_chains, n_steps)
    print("DA", st_da, "\nMH", st_mh, "\nuntrained", st_un)
    per_step_da = st_da["exact_evals"] / st_da["steps"]
    per_step_mh = st_mh["exact_evals"] / st_mh["steps"]
    acc2 = st_da["accepted"] / st_da["exact_evals"]
    acc2_un = st_un["accepted"] / max(st_un["exact_evals"], 1)
    assert per_step_da < 0.6 * per_step_mh
    assert acc2 > 0.6
    assert acc2 > acc2_un + 0.1
    burn = 40
    x_da = ch_da.samples[:, burn:].cpu().numpy()
    x_mh = ch_mh.samples[:, burn:].cpu().numpy()
    sig = x_mh.reshape(-1, 5).std(0)
    m_da, m_mh = x_da.reshape(-1, 5).mean(0), x_mh.reshape(-1, 5).mean(0)
    print("posterior mean DA", m_da, "MH", m_mh, "std", sig)
    assert np.all(np.abs(m_da - m_mh) <= 0.5 * sig)
    assert rms <= 0.1


def test_two_level_da_effective_samples(config3, trained):
    """The emulator sub-chain sampler targets the same posterior as exact
    Metropolis and buys more effective samples per exact evaluation."""
    from cosmoforge_b200 import sampler

    E, N, X, tables = config3
    emu, F = trained
    prop = sampler.proposal_cov(F)
    s_sub = sampler.Sampler(E, N, X, emulator=emu, prop_cov=prop, seed=4)
    ch_sub, st_sub = s_sub.run_da_subchain(64, 120, sub_steps=24)
    s_mh = sampler.Sampler(E, N, X, prop_cov=prop, seed=5)
    ch_mh, st_mh = s_mh.run_exact_mh(64, 240)
    ess_sub = sampler.effective_sample_size(ch_sub.samples.cpu().numpy(), burn=20)
    ess_mh = sampler.effective_sample_size(ch_mh.samples.cpu().numpy(), burn=40)
    per_eval_sub = ess_sub.min() / st_sub["exact_evals"]
    per_eval_mh = ess_mh.min() / st_mh["exact_evals"]
    acc2 = st_sub["accepted"] / st_sub["exact_evals"]
    print("two-level", st_sub, "min ESS", ess_sub.min(), "\nMH", st_mh, "min ESS", ess_mh.min())
    assert st_sub["steps"] == 64 * 120 and st_sub["exact_evals"] == 64 * 120
    assert acc2 > 0.8
    assert per_eval_sub > 3.0 * per_eval_mh
    x_sub = ch_sub.samples[:, 20:].cpu().numpy().reshape(-1, 5)
    x_mh = ch_mh.samples[:, 40:].cpu().numpy().reshape(-1, 5)
    sig = x_mh.std(0)
    print("posterior mean two-level", x_sub.mean(0), "MH", x_mh.mean(0), "std", sig, x_sub.std(0))
    assert np.all(np.abs(x_sub.mean(0) - x_mh.mean(0)) <= 0.3 * sig)
    assert np.all(np.abs(x_sub.std(0) / sig - 1.0) <= 0.25)
