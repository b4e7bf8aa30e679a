"""Autotuner of the mixed Fisher GEMM forms: the forms it picks keep F within
its tolerance of the FP64 path, and the choice round-trips through the cache."""

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
    assert all(ap in (0, 1) and kc in (8, 16, 32) for ap, kc in forms.values())
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
