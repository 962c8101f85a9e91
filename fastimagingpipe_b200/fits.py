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


def _hdu(cards, body: bytes) -> bytes:
    hdr = b"".join(cards) + _card("END")
    hdr += b" " * (-len(hdr) % _BLOCK)
    return hdr + body + b"\0" * (-len(body) % _BLOCK)


def _str(v: str) -> str:
    """A FITS string value, quoted and padded to at least 8 characters."""
    return "'" + v.ljust(8) + "'"


def _strcard(key: str, value: str) -> bytes:
    return (f"{key:<8.8s}= " + _str(value)).ljust(80)[:80].encode("ascii")


def write_table(path: str, columns, extname: str = "LOCATIONS") -> None:
    """An empty primary HDU and one BINTABLE extension.  columns: list of
    (name, array) with int32 ('J') or float32 ('E') arrays of equal length."""
    arrs = []
    for name, a in columns:
        a = np.asarray(a)
        if a.dtype.kind in "iu":
            arrs.append((name, "J", a.astype(">i4")))
        else:
            arrs.append((name, "E", a.astype(">f4")))
    nrows = len(arrs[0][2]) if arrs else 0
    prim = _hdu([_card("SIMPLE", "T"), _card("BITPIX", "8"), _card("NAXIS", "0"),
                 _card("EXTEND", "T")], b"")
    cards = [_strcard("XTENSION", "BINTABLE"), _card("BITPIX", "8"), _card("NAXIS", "2"),
             _card("NAXIS1", str(4 * len(arrs))), _card("NAXIS2", str(nrows)),
             _card("PCOUNT", "0"), _card("GCOUNT", "1"), _card("TFIELDS", str(len(arrs)))]
    for k, (name, form, _) in enumerate(arrs):
        cards += [_strcard(f"TTYPE{k + 1}", name), _strcard(f"TFORM{k + 1}", "1" + form)]
    cards.append(_strcard("EXTNAME", extname))
    rows = np.empty(nrows, dtype=[(name, a.dtype) for name, _, a in arrs])
    for name, _, a in arrs:
        rows[name] = a
    with open(path, "wb") as f:
        f.write(prim + _hdu(cards, rows.tobytes()))


def read_table(path: str, extname: str = "LOCATIONS") -> dict:
    """Columns of the named BINTABLE extension ('J' and 'E' columns) as a dict
    of numpy arrays."""
    raw = open(path, "rb").read()
    pos = 0
    while pos + _BLOCK <= len(raw):
        cards, end = {}, False
        while not end:
            block = raw[pos:pos + _BLOCK]
            for c in range(0, _BLOCK, 80):
                card = block[c:c + 80].decode("ascii", "replace")
                if card[:8].strip() == "END":
                    end = True
                    break
                if card[8:10] == "= ":
                    cards[card[:8].strip()] = card[10:].split("/")[0].strip().strip("'").strip()
            pos += _BLOCK
        naxis = int(cards.get("NAXIS", "0"))
        axes = [int(cards[f"NAXIS{k + 1}"]) for k in range(naxis)]
        nbytes = (abs(int(cards.get("BITPIX", "8"))) // 8 * int(cards.get("GCOUNT", "1")) *
                  (int(cards.get("PCOUNT", "0")) + (int(np.prod(axes)) if naxis else 0)))
        if cards.get("XTENSION") == "BINTABLE" and cards.get("EXTNAME") == extname:
            nf = int(cards["TFIELDS"])
            dt = [(cards[f"TTYPE{k + 1}"], {"J": ">i4", "E": ">f4"}[cards[f"TFORM{k + 1}"][-1]])
                  for k in range(nf)]
            rows = np.frombuffer(raw[pos:pos + axes[0] * axes[1]], dtype=dt)
            return {name: rows[name].astype(rows[name].dtype.newbyteorder("=")) for name, _ in dt}
        pos += -(-nbytes // _BLOCK) * _BLOCK
    raise ValueError(f"no BINTABLE {extname!r} in {path}")


def write_combined(path: str, vis_re, vis_im, B, V, num_snapshots: int) -> None:
    """The preprocessing tool's combined input file (write_combined_input_fits,
    SVDPreprocessMain.cpp:182-258): an empty BYTE_IMG primary HDU, then IMAGE
    extensions "TRANSFORMATION MATRICES" [S][3][3], "VISIBILITIES"
    [S][samples][2] (real, imaginary interleaved) and "R-COORDINATES"
    [S][samples][2], FLOAT_IMG."""
    s = int(num_snapshots)
    vr = np.asarray(vis_re, np.float32).reshape(s, -1)
    vis = np.stack([vr, np.asarray(vis_im, np.float32).reshape(s, -1)], axis=-1)
    rc = np.asarray(B, np.float32).reshape(s, -1, 2)
    tm = np.asarray(V, np.float32).reshape(s, 3, 3)
    out = _hdu([_card("SIMPLE", "T"), _card("BITPIX", "8"), _card("NAXIS", "0"),
                _card("EXTEND", "T")], b"")
    for name, a in (("TRANSFORMATION MATRICES", tm), ("VISIBILITIES", vis), ("R-COORDINATES", rc)):
        a = np.ascontiguousarray(a, ">f4")
        cards = [_strcard("XTENSION", "IMAGE"), _card("BITPIX", "-32"),
                 _card("NAXIS", str(a.ndim))]
        cards += [_card(f"NAXIS{k + 1}", str(n)) for k, n in enumerate(reversed(a.shape))]
        cards += [_card("PCOUNT", "0"), _card("GCOUNT", "1"), _strcard("EXTNAME", name)]
        out += _hdu(cards, a.tobytes())
    with open(path, "wb") as f:
        f.write(out)


def read_combined(path: str):
    """The combined input file -> (vis_re, vis_im, B, V, samples, snapshots) in
    FIpipe's snapshot-concatenated layout."""
    ext = {name: arr for name, arr in read_all(path)}
    tm, vis, rc = ext["TRANSFORMATION MATRICES"], ext["VISIBILITIES"], ext["R-COORDINATES"]
    s, samples = vis.shape[0], vis.shape[1]
    return (np.ascontiguousarray(vis[..., 0].reshape(-1)),
            np.ascontiguousarray(vis[..., 1].reshape(-1)), rc.reshape(-1), tm.reshape(-1),
            samples, s)
