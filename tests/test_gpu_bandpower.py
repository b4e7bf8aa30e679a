"""Bandpower window function and effective multipoles of the drop-in Fisher
against the reference's own outputs (qube/fisher.py:1050-1234): F, W and
l_eff within 1e-10 relative on the FP64 path; the mixed path's W within 1e-4
of the largest window entry."""

import numpy as np
import pytest

from golden_cases import cls_of, load, noise_of, params_of

pytestmark = pytest.mark.gpu


def _rel(a, b):
    return float(np.max(np.abs(np.asarray(a) - np.asarray(b))) / np.max(np.abs(np.asarray(b))))


@pytest.mark.parametrize("name", ["bandpower_tt_nside8", "bandpower_tqu_cut_nside4"])
@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_bandpower_window_matches_reference(name, precision):
    from cosmoforge_b200 import qube

    d = load(name)
    f = qube.Fisher(params_of(d), basis=False, mask=d["mask"], noise_cov1=noise_of(d), cls_data=cls_of(d),
                    beam=d["beam"], precision=precision)
    f.run()
    W = f.get_bandpower_window_function()
    eff = f.get_effective_ells()
    assert W.shape == d["ref_window"].shape
    e_f, e_w, e_l = _rel(f.get_fisher_matrix(), d["ref_fisher"]), _rel(W, d["ref_window"]), _rel(eff, d["ref_eff_ells"])
    print(f"{name} {precision}: F {e_f:.1e}  W {e_w:.1e}  l_eff {e_l:.1e}")
    if precision == "fp64":
        assert e_f <= 1e-10 and e_w <= 1e-10 and e_l <= 1e-10
    else:
        assert e_w <= 1e-4 and e_l <= 1e-5
    # rows of W sum to one over each bin's own multipoles (W Q^T = I)
    assert W is f.get_bandpower_window_function()


@pytest.mark.parametrize("basis", ["harmonic"])
def test_bandpower_window_other_bases(basis):
    """Per-multipole Fisher through the harmonic contractions: on the spin-0 TT
    case (where the harmonic and pixel-space estimators agree to rounding) the
    window and effective multipoles equal the pixel-space reference's."""
    from cosmoforge_b200 import qube

    d = load("bandpower_tt_nside8")
    f = qube.Fisher(params_of(d), basis=basis, mask=d["mask"], noise_cov1=noise_of(d), cls_data=cls_of(d),
                    beam=d["beam"])
    f.run()
    W = f.get_bandpower_window_function()
    e_w, e_l = _rel(W, d["ref_window"]), _rel(f.get_effective_ells(), d["ref_eff_ells"])
    print(f"{basis}: W {e_w:.1e}  l_eff {e_l:.1e}")
    assert e_w <= 1e-9 and e_l <= 1e-9
