"""Host logic of the basis= argument (no GPU): the request mapping of
cosmocore/core.py:135-160, the reference's auto rule
(cosmocore/basis/__init__.py:87-115) and the eigenvector selection of the
compressed basis (cosmocore/basis/pixel.py:265-311) against the oracle's."""

import numpy as np
import pytest

from cosmoforge_b200 import harmonic, workloads
from cosmoforge_b200.layout import build_layout
from cosmoforge_b200.qube import _check_basis, _compression_of
from oracle import harmonic_oracle as ho


@pytest.mark.parametrize("basis,method", [
    (False, "pixel"), (None, "auto"), ("auto", "auto"), ("pixel", "pixel"), ("harmonic", "harmonic"),
    ({"method": "harmonic"}, "harmonic"), ({}, "auto"), ({"method": "pixel", "epsilon": 1e-4}, "compressed"),
    ({"method": "pixel", "mode_fraction": 0.5}, "compressed"),
    ({"method": "pixel", "epsilon": None, "compression_target": "harmonic"}, "pixel")])
def test_basis_request(basis, method):
    assert _check_basis(basis) == method


@pytest.mark.parametrize("basis,exc", [("smw", ValueError), (3, TypeError), ({"method": "svd"}, ValueError),
                                       ({"method": "pixel", "pixel_filter": 1}, NotImplementedError),
                                       ({"epsilon": 1e-3}, NotImplementedError),
                                       ({"method": "harmonic", "mode_fraction": 0.5}, NotImplementedError)])
def test_basis_rejects(basis, exc):
    with pytest.raises(exc):
        _check_basis(basis)


def test_compression_options():
    c = _compression_of({"method": "pixel", "epsilon": 1e-3})
    assert c == {"epsilon": 1e-3, "mode_fraction": None, "target": "noise_weighted", "C_ell": None}
    c = _compression_of({"method": "pixel", "epsilon": [1e-3, (1e-3, 1e-2)], "compression_target": "snr",
                         "C_ell": [0.0, 1.0]})
    assert c["target"] == "snr" and c["epsilon"] == [1e-3, (1e-3, 1e-2)] and c["C_ell"] == [0.0, 1.0]
    assert _compression_of("harmonic") == {}


def test_auto_rule_matches_cost_model():
    for pb, want in ((workloads.config0(), "harmonic"), (workloads.config1(), "harmonic")):
        L = build_layout(pb.params, pb.mask, pb.beam)
        n_modes = harmonic.n_modes_reference(L)
        cost_h, cost_p = float(n_modes) ** 3, float(L.nbins + 1) * float(L.n) ** 3
        assert harmonic.auto_method(L) == ("harmonic" if cost_h <= cost_p else "pixel") == want
    # many pixels, few multipoles and one bin: the pixel basis is cheaper
    pb = workloads.config0()
    L = build_layout(pb.params | {"lmax": 24, "delta_ell": 23}, pb.mask, pb.beam)
    assert L.nbins == 1 and harmonic.auto_method(L) == "pixel"


@pytest.mark.parametrize("kw", [dict(epsilon=1e-3), dict(epsilon=0.5), dict(mode_fraction=0.3),
                                dict(mode_fraction=1.0), dict()])
def test_keep_modes_matches_oracle(kw):
    rng = np.random.default_rng(5)
    ev = np.concatenate([rng.uniform(1e-14, 1e-12, 20), 10 ** rng.uniform(-6, 2, 80)])
    rng.shuffle(ev)
    got = harmonic.keep_modes(ev, kw.get("epsilon"), kw.get("mode_fraction"))
    ref = ho.keep_modes(ev, kw.get("epsilon"), kw.get("mode_fraction"))
    assert np.array_equal(got, ref)
    assert np.all(np.diff(ev[got]) <= 0)


def test_per_field_thresholds():
    assert harmonic._per_field(1e-3, 2, "epsilon") == [1e-3, 1e-3]
    assert harmonic._per_field([0.7, 0.6], 2, "mode_fraction") == [0.7, 0.6]
    with pytest.raises(ValueError):
        harmonic._per_field([0.7], 2, "mode_fraction")
    # an (E, B) pair per spin-2 field (cosmocore/basis/pixel.py:447-557)
    assert harmonic._per_field([0.6, (0.7, 0.5)], 2, "mode_fraction") == [0.6, (0.7, 0.5)]
    assert harmonic._per_field([1e-3, [1e-3, 1e-2]], 2, "epsilon") == [1e-3, (1e-3, 1e-2)]


def test_auto_falls_back_to_pixel_for_unsupported_layouts():
    from cosmoforge_b200.qube import _resolve_method

    class _L:  # four components: two spin-0 fields and a spin-2 field
        lmin, lmax, n, nbins = 2, 10, 10 ** 6, 1
        fields = [type("F", (), {"spin": s})() for s in (0, 0, 2)]

    assert _resolve_method("auto", _L) == "pixel"
    assert _resolve_method("harmonic", _L) == "harmonic"  # an explicit request is passed on (and raises later)
