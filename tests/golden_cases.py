"""Load the golden fixtures into (params, mask, noise, cls, beam, maps) tuples."""

from __future__ import annotations

from pathlib import Path

import numpy as np

GOLDEN = Path(__file__).resolve().parent / "golden"


def load(name: str) -> dict:
    d = dict(np.load(GOLDEN / f"{name}.npz", allow_pickle=False))
    return d


def params_of(d: dict) -> dict:
    return dict(
        nside=int(d["p_nside"]), spins=[int(s) for s in d["p_spins"]],
        labels=[str(s) for s in d["p_labels"]], lmin=int(d["p_lmin"]), lmax=int(d["p_lmax"]),
        lmax_signal=int(d["p_lmax_signal"]),
        delta_ell=int(d["p_delta_ell"]) if "p_delta_ell" in d else 1, ordering="RING",
        nsims=int(d["maps"].shape[1]) if "maps" in d else 1,
        remove_nb=bool(int(d["p_remove_nb"])),
        output_convention=str(d["p_output_convention"]), feedback=0,
    )


def cls_of(d: dict) -> dict:
    return {k[3:]: v for k, v in d.items() if k.startswith("cl_")}


def noise_of(d: dict) -> np.ndarray:
    if "noise" in d:
        return d["noise"]
    return np.diag(d["noise_diag"])


QML_CASES = ["fortran_qube_nside8_B", "nside4_T", "nside4_QU", "nside4_TQU", "nside4_TEB",
             "config0_tt_nside8", "tqu_cut_nside4"]


def smoothed_cls(d: dict) -> dict:
    """{label: C_l b_l^2} with the fixture's beam rows (T, E, B): the
    beam-smoothed spectra passed as a compressed basis's ``C_ell``
    (tests/golden/make_golden.py builds the same arrays)."""
    beam = d["beam"]
    row = {"T": 0, "E": 1, "B": 2}
    out = {}
    for lab, c in cls_of(d).items():
        c = np.asarray(c, dtype=np.float64)
        n = min(c.size, beam.shape[1])
        out[lab] = c[:n] * beam[row[lab[0]], :n] * beam[row[lab[1]], :n]
    return out
