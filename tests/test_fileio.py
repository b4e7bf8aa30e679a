"""File adapters (cosmoforge_b200.fileio) against the arrays the golden fixtures hold.

The nside-4 fixtures were produced by the reference from its own test data
(mask.fits, NCVM1.bin, dls.txt, the beam table, all_sims_TQU.fits); reading the
same files here must give the same arrays.  That test reads the reference's
data files from the checkout named by ``COSMOFORGE_REFERENCE`` and is skipped
when the variable is unset.  Round trips of the plain formats run everywhere.
"""

import os
from pathlib import Path

import numpy as np
import pytest

from cosmoforge_b200 import fileio, params as prm
from cosmoforge_b200.layout import build_layout
from golden_cases import cls_of, load, params_of

_REF_ROOT = os.environ.get("COSMOFORGE_REFERENCE")
QDATA = (Path(_REF_ROOT) / "src" / "cosmoforge.qube" / "tests" / "data") if _REF_ROOT else None


def test_covmat_and_cls_round_trip(tmp_path):
    d = load("tqu_cut_nside4")
    p = params_of(d)
    L = build_layout(p, d["mask"], d["beam"])
    npix, ncomp = 12 * L.nside ** 2, 3
    full = np.zeros((npix * ncomp, npix * ncomp))
    act = fileio.active_indices(L)
    full[np.ix_(act, act)] = d["noise"]
    (tmp_path / "N.bin").write_bytes(full.tobytes())
    assert np.array_equal(fileio.read_covmat(str(tmp_path / "N.bin"), npix, ncomp, act), d["noise"])
    (tmp_path / "Nr.bin").write_bytes(np.ascontiguousarray(d["noise"]).tobytes())
    assert np.array_equal(fileio.read_covmat_reduced(str(tmp_path / "Nr.bin"), L.n), d["noise"])
    ell = np.arange(2, 17)
    tt = 1000.0 / (ell * (ell + 1.0))
    path = tmp_path / "cls.txt"
    np.savetxt(path, np.column_stack([ell, tt, 0.1 * tt]), header="ell TT EE")
    cls = fileio.read_cls(str(path), 16, "Cl")
    assert np.array_equal(cls["TT"][2:], tt) and cls["TT"][:2].sum() == 0.0
    dl = fileio.read_cls(str(path), 16, "Dl")
    assert np.allclose(dl["TT"][2:], tt * 2 * np.pi / (ell * (ell + 1.0)), rtol=1e-15)


def test_gaussian_beam_polarisation_factor():
    b = fileio.gaussian_beam_pol(60.0, 30)
    s2 = (np.radians(1.0) / np.sqrt(8 * np.log(2))) ** 2
    ell = np.arange(31)
    assert np.allclose(b[0], np.exp(-0.5 * ell * (ell + 1) * s2), rtol=1e-14)
    assert np.allclose(b[1], b[0] * np.exp(2 * s2), rtol=1e-14) and np.array_equal(b[1], b[2])


@pytest.mark.skipif(QDATA is None or not QDATA.exists(), reason="COSMOFORGE_REFERENCE not set")
@pytest.mark.parametrize("fields", ["T", "TQU"])
def test_reference_files_give_the_fixture_arrays(fields):
    import yaml

    d = load(f"nside4_{fields}")
    D = QDATA / "nside4" / fields
    cfg = yaml.safe_load(open(D / "config.yaml"))
    p = params_of(d)
    ncomp = sum(1 if s == 0 else 2 for s in p["spins"])
    mask = fileio.read_mask(str(D / "mask.fits"), ncomp)
    assert np.array_equal(mask, d["mask"])
    L = build_layout(p, mask, d["beam"])
    N = fileio.read_covmat(str(D / "NCVM1.bin"), 12 * L.nside ** 2, ncomp, fileio.active_indices(L))
    assert np.array_equal(np.diag(N), d["noise_diag"])
    cls = fileio.read_cls(str(D / "dls.txt"), int(p["lmax_signal"]), "Dl")
    ref = cls_of(d)
    for lab, v in ref.items():
        if lab in cls:
            n = min(len(v), len(cls[lab]))
            assert np.allclose(cls[lab][:n], v[:n], rtol=1e-13, atol=0)
    sims = QDATA / "nside4" / "maps" / "all_sims_TQU.fits"
    phys = prm.resolve(cfg)["physical_labels"] or (["T", "Q", "U"] if ncomp == 3 else ["T"])
    pixact = [f.pixels for f in L.fields for _ in range(1 if f.spin == 0 else 2)]
    maps = fileio.read_maps(str(sims), pixact, list(phys), d["maps"].shape[1])
    assert np.array_equal(maps, d["maps"])
