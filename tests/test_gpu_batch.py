"""Batched QML: many maps against one C (map_solves) and many patches at once (PatchBatch).

map_solves FP64 must equal the per-spectrum QML reductions to 1e-12 relative
(same products, different summation order); the split-product form is held
to 1e-5 relative of max |q| (BF16x6, FP32 GEMM output).  PatchBatch must
reproduce the single-problem device path to 1e-10 relative and, on a small
patch, the CPU oracle to 1e-10.
"""

import numpy as np
import pytest
import torch

from cosmoforge_b200 import workloads
from cosmoforge_b200.layout import build_layout
from golden_cases import cls_of, load, noise_of, params_of

pytestmark = pytest.mark.gpu


def _rel(a, b):
    a, b = np.asarray(a), np.asarray(b)
    return float(np.max(np.abs(a - b)) / np.max(np.abs(b)))


@pytest.mark.parametrize("name", ["tqu_cut_nside4", "nside4_TEB", "config0_tt_nside8"])
def test_map_solves_match_qml_reductions(name):
    from cosmoforge_b200 import batch, engine

    d = load(name)
    L = build_layout(params_of(d), d["mask"], d["beam"])
    E = engine.Engine(L)
    N = torch.from_numpy(noise_of(d)).cuda()
    S = E.signal(L.smoothed_cl_table(cls_of(d)))
    Cinv = E.spd_inverse(S + N)
    g = torch.Generator(device="cuda").manual_seed(5)
    X = torch.randn((L.n, 300), dtype=torch.float64, device="cuda", generator=g) * 30.0
    q64 = batch.map_solves(E, Cinv, X).cpu().numpy()
    _, _, qref = E.fisher_qml(Cinv, None, X[:, :4], want_fisher=False)
    assert _rel(q64[:4], qref.cpu().numpy()) <= 1e-12
    qm = batch.map_solves(E, Cinv, X, precision="mixed").cpu().numpy()
    print(f"{name}: mixed vs fp64 {_rel(qm, q64):.2e}")
    assert _rel(qm, q64) <= 1e-5


def _patch_dicts(k_max=6, seed=0):
    from cosmoforge_b200 import engine, qube

    probs = workloads.config2_patches(seed=seed)[:k_max]
    out = []
    for j, p in enumerate(probs):
        L = build_layout(p.params, p.mask, p.beam)
        N = torch.from_numpy(p.noise).cuda()
        x = qube.draw_maps(L, p.cls, N, 1, seed=100 + j)
        out.append(dict(params=p.params, mask=p.mask, beam=p.beam, cls=p.cls, noise=p.noise,
                        maps=x.cpu().numpy()))
    return out


def test_patch_batch_matches_single_problem_path():
    from cosmoforge_b200 import batch, engine

    probs = _patch_dicts(8)
    pb = batch.PatchBatch(probs)
    res = pb.run(graph=False).results()
    for p, r in zip(probs, res):
        L = build_layout(p["params"], p["mask"], p["beam"])
        E = engine.Engine(L)
        N = torch.from_numpy(p["noise"]).cuda()
        Cinv = E.spd_inverse(E.signal(L.smoothed_cl_table(p["cls"])) + N)
        F, b, q = E.fisher_qml(Cinv, N, torch.from_numpy(p["maps"]).cuda())
        assert r["info_cov"] == 0
        assert _rel(r["fisher"], F.cpu().numpy()) <= 1e-10
        assert _rel(r["bias"], b.cpu().numpy()) <= 1e-10
        assert _rel(r["q"], q.cpu().numpy()) <= 1e-10


def test_patch_batch_graph_replay_matches_eager():
    from cosmoforge_b200 import batch

    probs = _patch_dicts(5, seed=1)
    a = batch.PatchBatch(probs).run(graph=False)
    ra = [dict(r) for r in a.results()]
    b = batch.PatchBatch(probs)
    b.run(graph=True)   # eager first call, then captured
    b.run(graph=True)   # replay
    rb = b.results()
    # the split-K Fisher contraction adds partial sums with atomics, so runs
    # agree to rounding, not bit for bit
    for x, y in zip(ra, rb):
        for k in ("fisher", "q", "bias"):
            assert _rel(y[k], x[k]) <= 1e-13


def test_patch_batch_small_patch_matches_oracle():
    from cosmoforge_b200 import batch
    from oracle import oracle

    probs = _patch_dicts(48)
    small = [p for p in probs if int(p["mask"].sum()) <= 60][:2]
    assert small, "expected caps below 60 pixels"
    res = batch.PatchBatch(small).run(graph=False).results()
    for p, r in zip(small, res):
        L = build_layout(p["params"], p["mask"], p["beam"])
        ref = oracle.qml_solve(L, p["cls"], p["noise"], p["maps"])
        assert _rel(r["fisher"], ref["fisher"]) <= 1e-10
        assert _rel(r["bias"], ref["bias"]) <= 1e-10
        assert _rel(r["q"] - r["bias"][None], ref["q"]) <= 1e-10
