"""FITS output (ilc_fits_write_image; host only, runs on the CPU): the file is
a valid primary HDU that reads back to the same floats, with the mandatory
cards, the reference's header keys (COMMENT + key, HIERARCH for long keys) and
2880-byte records."""
import numpy as np


def _read(path):
    raw = open(path, "rb").read()
    assert len(raw) % 2880 == 0
    cards, off = [], 0
    while True:
        c = raw[off:off + 80].decode("ascii")
        off += 80
        cards.append(c)
        if c.startswith("END"):
            break
    hdr_end = ((off + 2879) // 2880) * 2880
    return cards, raw[hdr_end:]


def test_fits_image_and_cube_round_trip(tmp_path):
    import illcrawl_b200 as ilc
    rng = np.random.default_rng(3)
    img = rng.standard_normal((5, 7)).astype(np.float32)
    img[0, 0] = np.inf
    p = tmp_path / "img.fits"
    ilc.write_fits(p, img, [("integration.rel_tol", 1e-3, "Relative integration tolerance"),
                            ("type", "image", "Type of this file"), ("NBINS", 128),
                            ("flag", True)])
    cards, data = _read(p)
    assert cards[0].startswith("SIMPLE  =                    T")
    assert cards[1].startswith("BITPIX  =                  -32")
    assert cards[2].startswith("NAXIS   =                    2")
    assert cards[3].startswith("NAXIS1  =                    7")
    assert cards[4].startswith("NAXIS2  =                    5")
    text = "".join(cards)
    assert "COMMENT Relative integration tolerance" in text
    assert "HIERARCH integration.rel_tol = 0.001" in text
    assert "NBINS   =                  128" in text
    assert all(len(c) == 80 for c in cards)
    back = np.frombuffer(data[:img.size * 4], ">f4").reshape(img.shape)
    assert np.array_equal(back.astype(np.float32).view(np.uint32), img.view(np.uint32))
    cube = rng.random((3, 4, 6)).astype(np.float32)
    ilc.write_fits(tmp_path / "cube.fits", cube)
    cards, data = _read(tmp_path / "cube.fits")
    assert cards[2].startswith("NAXIS   =                    3")
    assert cards[5].startswith("NAXIS3  =                    3")
    back = np.frombuffer(data[:cube.size * 4], ">f4").reshape(cube.shape)
    assert np.array_equal(back.astype(np.float32), cube)
    assert len(data) % 2880 == 0
