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
