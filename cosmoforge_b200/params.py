"""Analysis parameters in the reference's format (dict, YAML path or object).

Mirrors the subset of ``cosmocore/settings.py`` (``InputParams`` defaults at
178-253, label expansion at 451-507) that the pixel-space QML / Fisher /
likelihood path reads.  File-path parameters (``maskfile``, ``covmatfile1``,
``load_reduced``, ``inputclfile``, ``beam_file``, ``inputmapfile1``) are read by
``fileio`` when the matching array is not injected; output-file parameters are
ignored.
"""

from __future__ import annotations

from types import SimpleNamespace

DEFAULTS = dict(
    nside=16, spins=[0, 2], labels=["T", "E", "B"], physical_labels=None, feedback=1,
    do_cross=False, ordering="RING", lmax=64, lmin=2, lmax_signal=None, delta_ell=1,
    bin_lmins=None, bin_lmaxs=None, nsims=None, remove_nb=True, input_convention="Cl",
    output_convention="Cl", smoothing_type="cosine_legacy", apply_pixwin=True, fwhmarcmin=440.0,
    parameters={}, lmin_signal=2,
)


def resolve(params=None, params_file=None) -> dict:
    """Return a plain dict of parameters with the reference defaults filled in."""
    if params is not None and params_file is not None:
        raise TypeError("pass params or params_file, not both")
    src = params if params is not None else params_file
    out = dict(DEFAULTS)
    if src is None:
        return out
    if isinstance(src, str):
        import yaml

        with open(src) as fh:
            src = yaml.safe_load(fh) or {}
    elif not isinstance(src, dict):
        src = {k: v for k, v in vars(src).items() if not k.startswith("_")}
    for k, v in src.items():
        if k == "physical_labels" and isinstance(v, list):
            v = [c for item in v for c in (list(item) if item == "QU" else [item])]
        out[k] = v
    return out


def as_namespace(d: dict) -> SimpleNamespace:
    return SimpleNamespace(**d)
