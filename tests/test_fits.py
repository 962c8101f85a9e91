"""CPU tests of the FITS subset used by the drop-in command line."""
import numpy as np

from fastimagingpipe_b200 import fits


def test_roundtrip_2d(tmp_path):
    a = np.random.default_rng(0).standard_normal((7, 5)).astype(np.float32)
    p = tmp_path / "a.fits"
    fits.write_image(str(p), a)
    raw = p.read_bytes()
    assert len(raw) % 2880 == 0
    assert raw[:80].startswith(b"SIMPLE  =")
    assert b"NAXIS1  =                    5" in raw[:2880]
    assert b"NAXIS2  =                    7" in raw[:2880]
    b = fits.read_image(str(p))
    assert b.shape == (7, 5) and np.array_equal(a, b)


def test_roundtrip_1d_and_column_vector(tmp_path):
    a = np.arange(10, dtype=np.float32)
    fits.write_image(str(tmp_path / "v.fits"), a)
    assert np.array_equal(fits.read_image(str(tmp_path / "v.fits")), a)
    col = a[:, None]  # the shape SVD_MFS.py writes for Visreal (nb, 1)
    fits.write_image(str(tmp_path / "c.fits"), col)
    assert np.array_equal(fits.read_image(str(tmp_path / "c.fits")), col)


def test_reads_double_and_scaled_integers(tmp_path):
    def card(k, v=""):
        return (f"{k:<8}" + (f"= {v:>20}" if v else "")).ljust(80).encode()
    hdr = card("SIMPLE", "T") + card("BITPIX", "16") + card("NAXIS", "1") + card("NAXIS1", "3") + \
        card("BSCALE", "0.5") + card("BZERO", "10") + card("END")
    hdr += b" " * (-len(hdr) % 2880)
    body = np.array([1, -2, 3], ">i2").tobytes()
    body += b"\0" * (-len(body) % 2880)
    p = tmp_path / "i.fits"
    p.write_bytes(hdr + body)
    assert np.allclose(fits.read_image(str(p)), [10.5, 9.0, 11.5])


def test_binary_table_roundtrip(tmp_path):
    p = str(tmp_path / "t.fits")
    cols = [("TILE_ROW", np.array([3, 1], np.int32)), ("TLISI", np.array([0.5, 0.75], np.float32))]
    fits.write_table(p, cols)
    raw = open(p, "rb").read()
    assert len(raw) % 2880 == 0 and b"XTENSION= 'BINTABLE'" in raw
    t = fits.read_table(p)
    assert t["TILE_ROW"].tolist() == [3, 1] and t["TLISI"].tolist() == [0.5, 0.75]


def test_combined_input_roundtrip(tmp_path):
    """The preprocessing tool's layout: extensions found by EXTNAME, the
    visibilities interleaved (real, imaginary) per sample."""
    rng = np.random.default_rng(1)
    s, n = 3, 7
    vr, vi = rng.standard_normal(s * n), rng.standard_normal(s * n)
    B, V = rng.standard_normal(s * n * 2), rng.standard_normal(s * 9)
    p = str(tmp_path / "input.fits")
    fits.write_combined(p, vr, vi, B, V, s)
    names = [name for name, _ in fits.read_all(p)]
    assert names == ["", "TRANSFORMATION MATRICES", "VISIBILITIES", "R-COORDINATES"]
    got = fits.read_combined(p)
    assert got[4:] == (n, s)
    for a, b in zip(got[:4], (vr, vi, B, V)):
        assert np.array_equal(a, np.float32(b))
