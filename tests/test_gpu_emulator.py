"""Emulator training kernels and the delayed-acceptance sampler on the GPU.

* Device gradients (FP32 accumulation, BF16 weight matrices) against the FP64
  CPU oracle on the same BF16 weights: relative 2e-4 of the largest entry.
* Adam against its closed form; a graph-captured training run equals the
  eager one bit for bit.
* On the config-3 likelihood: the trained network's stage 1 lets the sampler
  spend fewer exact evaluations per step than plain exact Metropolis, with a
  high stage-2 acceptance that an untrained network does not reach, and both
  samplers agree on the posterior mean.
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


def test_delayed_acceptance_saves_exact_evaluations(config3):
    from cosmoforge_b200 import sampler

    E, N, X, tables = config3
    th, m2 = sampler.training_set(E, tables, N, X, 8192, seed=0)
    emu = _emu(0)
    emu.fit(th, m2, steps=1500, batch=1024)
    # held-out accuracy near the posterior
    F = sampler.fisher_theta(E, tables, N, workloads.THETA_CENTRE)
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
