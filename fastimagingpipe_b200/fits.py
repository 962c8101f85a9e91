"""Minimal FITS image files for the drop-in command line's inputs and output.

The reference reads and writes 1-D/2-D float images with cfitsio
(pipe_interface.cpp:12-137) and its preprocessing writes them with astropy
(SVD_MFS.py:117-120); neither library is needed for this subset of the FITS
standard: 2880-byte records, 80-character header cards, big-endian data,
BITPIX -32/-64/8/16/32/64 read with BSCALE/BZERO, BITPIX -32 written.
NAXIS1 is the fastest axis, so a numpy array of shape (rows, cols) is stored
with NAXIS1 = cols, NAXIS2 = rows.
"""
from __future__ import annotations

import numpy as np

_BLOCK = 2880
_DT = {8: ">u1", 16: ">i2", 32: ">i4", 64: ">i8", -32: ">f4", -64: ">f8"}


def _card(key: str, value: str = "") -> bytes:
    s = f"{key:<8.8s}" + (f"= {value:>20s}" if value else "")
    return s.ljust(80)[:80].encode("ascii")


def write_image(path: str, data) -> None:
    """Writes a FLOAT_IMG primary HDU, replacing any existing file."""
    a = np.ascontiguousarray(data, dtype=">f4")
    axes = list(reversed(a.shape)) if a.ndim else [1]
    hdr = _card("SIMPLE", "T") + _card("BITPIX", "-32") + _card("NAXIS", str(len(axes)))
    for k, n in enumerate(axes):
        hdr += _card(f"NAXIS{k + 1}", str(n))
    hdr += _card("END")
    hdr += b" " * (-len(hdr) % _BLOCK)
    body = a.tobytes()
    body += b"\0" * (-len(body) % _BLOCK)
    with open(path, "wb") as f:
        f.write(hdr + body)


def read_all(path: str):
    """All HDUs as (extname or '', array or None)."""
    raw = open(path, "rb").read()
    pos, out = 0, []
    while pos + _BLOCK <= len(raw):
        cards = {}
        order = []
        end = False
        while not end:
            block = raw[pos:pos + _BLOCK]
            if len(block) < _BLOCK:
                raise ValueError(f"truncated FITS header in {path}")
            for c in range(0, _BLOCK, 80):
                card = block[c:c + 80].decode("ascii", "replace")
                key = card[:8].strip()
                if key == "END":
                    end = True
                    break
                if card[8:10] == "= ":
                    val = card[10:].split("/")[0].strip().strip("'").strip()
                    cards[key] = val
                    order.append(key)
            pos += _BLOCK
        bitpix = int(cards.get("BITPIX", "8"))
        naxis = int(cards.get("NAXIS", "0"))
        axes = [int(cards[f"NAXIS{k + 1}"]) for k in range(naxis)]
        count = int(np.prod(axes)) if naxis else 0
        nbytes = abs(bitpix) // 8 * int(cards.get("GCOUNT", "1")) * (
            int(cards.get("PCOUNT", "0")) + count)
        arr = None
        if count and cards.get("XTENSION", "IMAGE") == "IMAGE":
            arr = np.frombuffer(raw[pos:pos + count * abs(bitpix) // 8],
                                dtype=_DT[bitpix]).astype(np.float64)
            arr = arr * float(cards.get("BSCALE", "1")) + float(cards.get("BZERO", "0"))
            arr = arr.astype(np.float32).reshape(list(reversed(axes)))
        out.append((cards.get("EXTNAME", ""), arr))
        pos += -(-nbytes // _BLOCK) * _BLOCK
    return out


def read_image(path: str) -> np.ndarray:
    """First HDU with data (1-D or 2-D), like the reference's read_fits_image."""
    for _, arr in read_all(path):
        if arr is not None:
            return arr
    raise ValueError(f"no image data in {path}")
