"""Autotuner: the mixed Fisher GEMM forms it picks keep F within its tolerance
of the FP64 path and round-trip through the cache; the patch-batch bucket
count it picks gives the single-bucket results; the likelihood launch shape
it picks keeps the mixed lnL within tolerance of FP64."""

import numpy as np
import pytest
import torch

from cosmoforge_b200.layout import build_layout
from golden_cases import cls_of, load, noise_of, params_of

pytestmark = pytest.mark.gpu


# bounds as for BF16x6 in test_gpu_mixed: the full-sky noiseless nside-4 case is
# ill-conditioned and carries a larger split-product error whatever the form
BOUND = {"tqu_cut_nside4": 1e-5, "nside4_TEB": 5e-5}


@pytest.mark.parametrize("name", sorted(BOUND))
def test_tuned_forms_meet_fisher_tolerance(name, tmp_path, monkeypatch):
    from cosmoforge_b200 import autotune, engine, engine_mixed

    monkeypatch.setenv("CFB200_TUNE_CACHE", str(tmp_path / "tuning.json"))
    autotune._MEM.clear()
    d = load(name)
    L = build_layout(params_of(d), d["mask"], d["beam"])
    E = engine.Engine(L)
    N = torch.from_numpy(noise_of(d)).cuda()
    Cinv = E.spd_inverse(E.signal(L.smoothed_cl_table(cls_of(d))) + N)
    forms, report = autotune.tune_fisher(E, Cinv, use_cache=False)
    assert set(forms) == set(range(L.nspectra))
    assert all(ap in (0, 1, 2) and kc in (8, 16, 32) and gm in autotune.GROUPS for ap, kc, gm in forms.values())
    assert set(report) == {s.label for s in L.spectra}
    F64 = E.fisher_qml(Cinv)[0].cpu().numpy()
    Fm = engine_mixed.fisher(E, Cinv, forms=forms).cpu().numpy()
    err = np.max(np.abs(np.diag(Fm) / np.diag(F64) - 1))
    print(f"{name}: forms {forms} diag err {err:.2e}")
    assert err <= BOUND[name]
    # cached: a second call returns the same forms without tuning
    autotune._MEM.clear()
    again, rep2 = autotune.tune_fisher(E, Cinv)
    assert rep2 is None and again == forms


def test_tuned_patch_buckets_keep_results(tmp_path, monkeypatch):
    from cosmoforge_b200 import autotune, batch
    from test_gpu_batch import _patch_dicts

    monkeypatch.setenv("CFB200_TUNE_CACHE", str(tmp_path / "tuning.json"))
    autotune._MEM.clear()
    probs = _patch_dicts(12, seed=3)
    k, rep = autotune.tune_patches(probs, candidates=(1, 2, 3), reps=2)
    assert k in (1, 2, 3) and set(rep["ms_per_batch"]) == {"1", "2", "3"}
    tuned = batch.PatchBatch(probs)  # buckets from the cache
    assert tuned.buckets == k or (k > 1 and tuned.buckets < k)
    ra = batch.PatchBatch(probs, buckets=1).run(graph=False).results()
    rb = tuned.run(graph=True).results()
    for x, y in zip(ra, rb):
        for key in ("fisher", "q", "bias"):
            assert np.max(np.abs(y[key] - x[key])) <= 1e-12 * np.max(np.abs(x[key]))


def test_tuned_likelihood_shape(tmp_path, monkeypatch):
    from cosmoforge_b200 import autotune, engine, workloads

    monkeypatch.setenv("CFB200_TUNE_CACHE", str(tmp_path / "tuning.json"))
    autotune._MEM.clear()
    pb = workloads.config3()
    L = build_layout(pb.params, pb.mask, pb.beam)
    E = engine.Engine(L)
    N = torch.from_numpy(pb.noise).cuda()
    X = torch.randn((L.n, 1), dtype=torch.float64, device="cuda") * 10.0
    choice, rep = autotune.tune_lnl(E, N, X, precision="mixed", batches=(128, 256), probe_points=256)
    assert choice["batch"] in (128, 256) and choice["tensor"] in (0, 1) and choice["build"] in ("auto", "basis_tc")
    picked = [r for r in rep["candidates"]
              if (r["batch"], r["tensor"], r["build"]) == (choice["batch"], choice["tensor"], choice["build"])]
    assert len(picked) == 1 and picked[0]["max_abs_dlnL"] <= 0.05
    # the FP64-built C keeps every batch size within the tolerance
    assert all(r["max_abs_dlnL"] <= 0.05 for r in rep["candidates"] if r["build"] == "auto" and r["tensor"] == 1)
    again, rep2 = autotune.tune_lnl(E, N, X, precision="mixed")
    assert rep2 is None and again == choice
