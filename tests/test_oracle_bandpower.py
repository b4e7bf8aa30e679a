"""Bandpower window function of the CPU oracle against the reference's outputs.

W = F_b^-1 Q F_perell (qube/fisher.py:1050-1190) from the oracle's Fisher
matrices with bins of 3 multipoles and of one multipole; effective
multipoles as window centroids (qube/fisher.py:1192-1234).
"""

import numpy as np
import pytest

from cosmoforge_b200.layout import build_layout
from golden_cases import cls_of, load, noise_of, params_of
from oracle import oracle


def oracle_window(d):
    p = params_of(d)
    L = build_layout(p, d["mask"], d["beam"])
    S = oracle.signal_matrix(L, L.smoothed_cl_table(cls_of(d)))
    Cinv = oracle.matrix_inverse_symm(S + noise_of(d))
    Fb = oracle.fisher(L, Cinv)
    L1 = build_layout(p | {"delta_ell": 1}, d["mask"], d["beam"])
    F1 = oracle.fisher(L1, Cinv)
    lmin, lmax = p["lmin"], p["lmax"]
    n_ell = lmax - lmin + 1
    Qb = np.zeros((L.nbins, n_ell))
    for b, (lo, hi) in enumerate(zip(L.bin_lmins, L.bin_lmaxs)):
        Qb[b, lo - lmin: hi - lmin + 1] = 1.0
    Q = np.kron(np.eye(L.nspectra), Qb)
    W = np.linalg.solve(Fb, Q @ F1)
    ells = np.arange(lmin, lmax + 1, dtype=np.float64)
    nb = L.nbins
    eff = np.concatenate([(W[s * nb:(s + 1) * nb, s * n_ell:(s + 1) * n_ell] @ ells)
                          / W[s * nb:(s + 1) * nb, s * n_ell:(s + 1) * n_ell].sum(axis=1)
                          for s in range(L.nspectra)])
    return Fb, W, eff


@pytest.mark.parametrize("name", ["bandpower_tt_nside8", "bandpower_tqu_cut_nside4"])
def test_oracle_bandpower_window_matches_reference(name):
    d = load(name)
    Fb, W, eff = oracle_window(d)
    assert np.max(np.abs(Fb - d["ref_fisher"])) <= 1e-12 * np.max(np.abs(d["ref_fisher"]))
    assert np.max(np.abs(W - d["ref_window"])) <= 1e-10 * np.max(np.abs(d["ref_window"]))
    assert np.max(np.abs(eff - d["ref_eff_ells"])) <= 1e-10 * np.max(d["ref_eff_ells"])
