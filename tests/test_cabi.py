"""The C-ABI library loads (without a GPU) and exports every declared symbol."""

import re
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parent.parent


def _declared():
    names = set()
    for h in (ROOT / "include").glob("*.h"):
        text = re.sub(r"/\*.*?\*/", "", h.read_text(), flags=re.S)
        names |= set(re.findall(r"\b(cf_[a-z0-9_]+)\s*\(", text))
    return sorted(names)


def test_header_declares_entry_points():
    names = _declared()
    assert "cf_build_block" in names and "cf_dgemm" in names and len(names) >= 10


def test_library_exports_every_declared_symbol():
    from cosmoforge_b200 import _build, _lib

    _build.build()
    handle = _lib.load_without_device()
    missing = [n for n in _declared() if not hasattr(handle, n)]
    assert not missing, missing
    assert handle.cf_version() >= 1


def test_bindings_cover_declarations():
    from cosmoforge_b200 import _lib

    assert set(_declared()) <= set(_lib.SIGNATURES)


def test_device_path_refuses_cpu_fallback(monkeypatch):
    import torch

    from cosmoforge_b200 import _lib

    monkeypatch.setattr(_lib, "_lib", None)
    monkeypatch.setattr(torch.cuda, "is_available", lambda: False)
    with pytest.raises(_lib.DeviceError):
        _lib.lib()
