"""The drop-in Fisher / Spectra driven by the reference's file parameters
(covmatfile1 + load_reduced, inputclfile, inputmapfile1) give the same
results as with the arrays injected."""

import numpy as np
import pytest

from golden_cases import cls_of, load, noise_of, params_of

pytestmark = pytest.mark.gpu


def test_file_inputs_match_injected(tmp_path):
    from cosmoforge_b200 import qube
    from cosmoforge_b200.layout import build_layout

    d = load("tqu_cut_nside4")
    p = params_of(d)
    N = noise_of(d)
    cls = cls_of(d)
    (tmp_path / "N.bin").write_bytes(np.ascontiguousarray(N).tobytes())
    L = build_layout(p, d["mask"], d["beam"])
    lmax_sig = int(p["lmax_signal"])
    labels = sorted(cls)
    ell = np.arange(lmax_sig + 1)
    np.savetxt(tmp_path / "cls.txt", np.column_stack([ell] + [cls[k][:lmax_sig + 1] for k in labels]),
               header="ell " + " ".join(labels))
    npix = 12 * L.nside ** 2
    comps = [f for f in L.fields for _ in range(1 if f.spin == 0 else 2)]
    full = np.zeros((len(comps), npix, d["maps"].shape[1]))
    r = 0
    for c, f in enumerate(comps):
        full[c, f.pixels] = d["maps"][r:r + f.npix]
        r += f.npix
    np.save(tmp_path / "maps.npy", full)
    pf = dict(p, covmatfile1=str(tmp_path / "N.bin"), load_reduced=True, inputclfile=str(tmp_path / "cls.txt"),
              input_convention="Cl", inputmapfile1=str(tmp_path / "maps.npy"), physical_labels=["T", "Q", "U"])

    f1 = qube.Fisher(pf, basis=False, mask=d["mask"], beam=d["beam"])
    f1.run()
    s1 = qube.Spectra(pf, fisher=f1)
    s1.run()
    f0 = qube.Fisher(p, basis=False, mask=d["mask"], noise_cov1=N, cls_data=cls, beam=d["beam"])
    f0.run()
    s0 = qube.Spectra(p, fisher=f0, maps1=d["maps"])
    s0.run()
    F0, F1 = f0.get_fisher_matrix(), f1.get_fisher_matrix()
    assert np.max(np.abs(F1 - F0)) <= 1e-13 * np.max(np.abs(F0))
    c0, c1 = s0.get_power_spectra(), s1.get_power_spectra()
    assert np.max(np.abs(c1 - c0)) <= 1e-12 * np.max(np.abs(c0))
