"""Minimal FITS binary-table reader for the reference's HEALPix fixtures.

Test infrastructure only. The fixtures are single-HDU ``BINTABLE`` files
whose columns are all ``TFORM='D'`` (big-endian float64) or ``'nD'`` vectors;
that is all this reader supports.
"""

from __future__ import annotations

import numpy as np

_BLOCK = 2880


def _parse_header(buf: bytes, off: int):
    cards = {}
    order = []
    while True:
        block = buf[off:off + _BLOCK].decode("ascii", "replace")
        off += _BLOCK
        done = False
        for i in range(0, _BLOCK, 80):
            card = block[i:i + 80]
            key = card[:8].strip()
            if key == "END":
                done = True
                break
            if card[8:10] == "= ":
                val = card[10:].split("/")[0].strip()
                if val.startswith("'"):
                    val = val.strip("'").strip()
                cards[key] = val
                order.append(key)
        if done:
            return cards, off


def read_bintable(path: str) -> dict[str, np.ndarray]:
    """Return ``{TTYPE: column}`` of the first BINTABLE extension in ``path``."""
    buf = open(path, "rb").read()
    off = 0
    hdr, off = _parse_header(buf, off)
    naxis = int(hdr.get("NAXIS", 0))
    if naxis:
        size = abs(int(hdr["BITPIX"])) // 8
        for k in range(1, naxis + 1):
            size *= int(hdr[f"NAXIS{k}"])
        off += (size + _BLOCK - 1) // _BLOCK * _BLOCK
    while off < len(buf):
        hdr, off = _parse_header(buf, off)
        if hdr.get("XTENSION") != "BINTABLE":
            raise ValueError(f"{path}: unsupported extension {hdr.get('XTENSION')}")
        rowlen = int(hdr["NAXIS1"])
        nrows = int(hdr["NAXIS2"])
        nfields = int(hdr["TFIELDS"])
        dtype_fields = []
        names = []
        for k in range(1, nfields + 1):
            form = hdr[f"TFORM{k}"].strip()
            rep = int(form[:-1]) if len(form) > 1 else 1
            if form[-1] != "D":
                raise ValueError(f"{path}: unsupported TFORM {form}")
            name = hdr.get(f"TTYPE{k}", f"COL{k}").strip()
            names.append(name)
            dtype_fields.append((name, ">f8", (rep,)) if rep > 1 else (name, ">f8"))
        dt = np.dtype(dtype_fields)
        if dt.itemsize != rowlen:
            raise ValueError(f"{path}: row length {rowlen} != {dt.itemsize}")
        table = np.frombuffer(buf, dtype=dt, count=nrows, offset=off)
        return {n: np.asarray(table[n], dtype=np.float64).reshape(-1) for n in names}
    raise ValueError(f"{path}: no BINTABLE found")


def read_image_hdus(path: str) -> dict[str, np.ndarray]:
    """Return ``{EXTNAME: array}`` for every IMAGE extension (BITPIX -64)."""
    buf = open(path, "rb").read()
    off = 0
    out = {}
    first = True
    while off < len(buf):
        hdr, off = _parse_header(buf, off)
        naxis = int(hdr.get("NAXIS", 0))
        shape = [int(hdr[f"NAXIS{k}"]) for k in range(1, naxis + 1)]
        size = abs(int(hdr.get("BITPIX", 8))) // 8
        for s in shape:
            size *= s
        if naxis and not first:
            if int(hdr["BITPIX"]) != -64:
                raise ValueError(f"{path}: unsupported BITPIX {hdr['BITPIX']}")
            arr = np.frombuffer(buf, dtype=">f8", count=size // 8, offset=off)
            out[hdr.get("EXTNAME", f"HDU{len(out)}").strip()] = (
                arr.reshape(shape[::-1]).astype(np.float64))
        if naxis:
            off += (size + _BLOCK - 1) // _BLOCK * _BLOCK
        first = False
    return out
