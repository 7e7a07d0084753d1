"""Input formats (src/io/npz.rs, src/io/fits.rs, read_inputs src/main.rs:50-132)
on the CPU: NPZ members of every supported dtype and byte order, the
reference's FITS binary-table and TAN-projection known-answer tests, the
grouping of several inputs, and malformed files (negative or oversized units,
axis counts, shapes; integers, repeats and headers the reference's parses
refuse), which must raise ValueError promptly instead of looping or wrapping."""
import math
import struct

import numpy as np
import pytest

from fbls_b200 import io

BLOCK = io.BLOCK


def test_npz_dtypes_and_byte_orders(tmp_path):
    arrays = {
        "f8": np.array([1.5, -2.25, math.pi]), "f4": np.array([0.5, 3.25], dtype=np.float32),
        "i8": np.array([[1, -2], [3, 4]], dtype=np.int64), "i4": np.array([7, -9], dtype=np.int32),
        "i2": np.array([-3], dtype=np.int16), "u1": np.array([200, 1], dtype=np.uint8),
        "b1": np.array([True, False, True]), "be": np.array([1.25, -8.5], dtype=">f8"),
        "scalar": np.float64(17.0),
    }
    path = tmp_path / "a.npz"
    np.savez(path, **arrays)
    got = io.read_npz(str(path))
    for k, v in arrays.items():
        a = np.asarray(v)
        assert got[k].shape == a.shape
        assert np.array_equal(got[k].data, a.astype(np.float64).reshape(-1))
    bad = tmp_path / "b.npz"
    np.savez(bad, c=np.array([1 + 2j]))
    with pytest.raises(ValueError, match="unsupported NPY dtype"):
        io.read_npz(str(bad))


def _card(key, value):
    s = f"{key:<8}= {value:>20}"[:80]
    return s.ljust(80).encode()


def _pad(b, fill):
    return b + fill * ((-len(b)) % BLOCK)


def test_fits_binary_table_round_trip(tmp_path):
    # fits.rs:354-402
    primary = b"".join(_card(k, v) for k, v in [("SIMPLE", "T"), ("BITPIX", "8"), ("NAXIS", "0")])
    primary = _pad(primary + b"END".ljust(80), b" ")
    ext = b"".join(_card(k, v) for k, v in [
        ("XTENSION", "'BINTABLE'"), ("BITPIX", "8"), ("NAXIS", "2"), ("NAXIS1", "16"), ("NAXIS2", "3"),
        ("PCOUNT", "0"), ("GCOUNT", "1"), ("TFIELDS", "3"), ("TTYPE1", "'TIME'"), ("TFORM1", "'D'"),
        ("TTYPE2", "'FLUX'"), ("TFORM2", "'E'"), ("TTYPE3", "'QUALITY'"), ("TFORM3", "'J'"),
        ("EXTNAME", "'LIGHTCURVE'")])
    ext = _pad(ext + b"END".ljust(80), b" ")
    data = b"".join(struct.pack(">d", 1.5 + r) + struct.pack(">f", 2.0 * r) + struct.pack(">i", 7 * r)
                    for r in range(3))
    path = tmp_path / "t.fits"
    path.write_bytes(primary + ext + _pad(data, b"\0"))
    hdus = io.read_fits(str(path))
    assert len(hdus) == 2
    t = hdus[1]
    assert t.name == "LIGHTCURVE"
    assert t.column_f64("TIME").tolist() == [1.5, 2.5, 3.5]
    assert t.column_f64("FLUX").tolist() == [0.0, 2.0, 4.0]
    assert t.column_f64("QUALITY").tolist() == [0.0, 7.0, 14.0]


def test_tan_projection_inverse_at_reference_point():
    # fits.rs:404-423
    h = io.Header([("CRPIX1", "6.635"), ("CRPIX2", "6.366"), ("CRVAL1", "26.2247"), ("CRVAL2", "-67.9748"),
                   ("CDELT1", "-0.00584"), ("CDELT2", "0.00584"), ("PC1_1", "-0.2788"), ("PC1_2", "0.9622"),
                   ("PC2_1", "0.9573"), ("PC2_2", "0.2828")])
    x, y = io.tan_world_to_pixel(h, 26.2247, -67.9748)
    assert abs(x - 5.635) < 1e-9 and abs(y - 5.366) < 1e-9


def test_read_inputs_groups_files_and_sectors(tmp_path):
    a, b, c = tmp_path / "a.npz", tmp_path / "b.npz", tmp_path / "c.npz"
    np.savez(a, time_bjd=np.arange(4.0), flux=np.ones(4), flux_err=np.full(4, 0.1), sector=np.array([3, 3, 4, 4]))
    np.savez(b, time_bjd=np.arange(10.0, 13.0), flux=np.ones(3), flux_err=np.full(3, 0.2), sector=np.array(3))
    np.savez(c, time_bjd=np.arange(3.0), flux=np.ones(3))
    obs = io.read_inputs([str(a), str(b)])
    assert obs.time.tolist() == [0.0, 1.0, 2.0, 3.0, 10.0, 11.0, 12.0]
    assert obs.group.tolist() == [0, 0, 1, 1, 2, 2, 2]  # per (file, sector)
    assert obs.err.tolist() == [0.1] * 4 + [0.2] * 3
    with pytest.raises(ValueError, match="either provide flux_err or omit it"):
        io.read_inputs([str(a), str(c)])
    assert io.read_inputs([str(c)]).err is None


def _table(cards, data=b""):
    primary = _pad(b"".join(_card(k, v) for k, v in [("SIMPLE", "T"), ("BITPIX", "8"), ("NAXIS", "0")])
                   + b"END".ljust(80), b" ")
    ext = _pad(b"".join(_card(k, v) for k, v in cards) + b"END".ljust(80), b" ")
    return primary + ext + _pad(data, b"\0")


@pytest.mark.timeout(20)
@pytest.mark.parametrize("cards,message", [
    ([("XTENSION", "'BINTABLE'"), ("BITPIX", "8"), ("NAXIS", "2"), ("NAXIS1", "8"), ("NAXIS2", "1"),
      ("PCOUNT", "-5760")], "truncated data unit"),       # would move the next header backwards
    ([("XTENSION", "'BINTABLE'"), ("BITPIX", "8"), ("NAXIS", "2"), ("NAXIS1", "8"), ("NAXIS2", "-1")],
     "truncated data unit"),
    ([("XTENSION", "'BINTABLE'"), ("BITPIX", "8"), ("NAXIS", "2"), ("NAXIS1", "4294967296"),
      ("NAXIS2", "4294967296")], "truncated data unit"),   # 2^64 bytes: no integer wrap
    ([("XTENSION", "'IMAGE'"), ("BITPIX", "8"), ("NAXIS", "1000000000")], "invalid NAXIS"),
    ([("XTENSION", "'IMAGE'"), ("BITPIX", "8"), ("NAXIS", "-3")], "invalid NAXIS"),
])
def test_fits_malformed_sizes_fail_cleanly(tmp_path, cards, message):
    path = tmp_path / "bad.fits"
    path.write_bytes(_table(cards, b"\0" * 8))
    with pytest.raises(ValueError, match=message):
        io.read_fits(str(path))


def test_fits_integers_and_repeats_parse_as_the_reference():
    h = io.Header([("A", "1_0"), ("B", "+7"), ("C", "-7"), ("D", "9223372036854775808"), ("E", "1_0.5"),
                   ("F", "2.5E3"), ("G", "٣")])
    assert h.i64("A") is None and h.i64("B") == 7 and h.i64("C") == -7 and h.i64("D") is None
    assert h.i64("G") is None
    assert h.f64("E") is None and h.f64("F") == 2500.0


def test_fits_tform_repeat_falls_back_to_one(tmp_path):
    cards = [("XTENSION", "'BINTABLE'"), ("BITPIX", "8"), ("NAXIS", "2"), ("NAXIS1", "8"), ("NAXIS2", "1"),
             ("PCOUNT", "0"), ("TFIELDS", "2"), ("TTYPE1", "'A'"), ("TFORM1", "'1_0E'"), ("TTYPE2", "'B'"),
             ("TFORM2", "'-2E'")]
    path = tmp_path / "r.fits"
    path.write_bytes(_table(cards, struct.pack(">ff", 1.5, 2.5)))
    t = io.read_fits(str(path))[1]
    assert [c.repeat for c in t.columns] == [1, 1]
    assert t.column_f64("A").tolist() == [1.5] and t.column_f64("B").tolist() == [2.5]


def _npy(header: str, body: bytes, version: int = 1) -> bytes:
    h = header.encode()
    if version == 1:
        return b"\x93NUMPY\x01\x00" + struct.pack("<H", len(h)) + h + body
    return b"\x93NUMPY\x02\x00" + struct.pack("<I", len(h)) + h + body


def test_npy_malformed_shapes_and_headers_fail_cleanly():
    body = struct.pack("<3d", 1.0, 2.0, 3.0)
    with pytest.raises(ValueError, match="invalid digit found in string"):
        io.parse_npy(_npy("{'descr': '<f8', 'fortran_order': False, 'shape': (-1,), }", body))
    with pytest.raises(ValueError, match="truncated NPY body"):
        io.parse_npy(_npy("{'descr': '<f8', 'fortran_order': False, 'shape': (4294967296, 4294967296), }", body))
    with pytest.raises(ValueError, match="number too large"):
        io.parse_npy(_npy("{'descr': '<f8', 'fortran_order': False, 'shape': (18446744073709551616,), }", body))
    with pytest.raises(ValueError, match="truncated NPY header"):
        io.parse_npy(b"\x93NUMPY\x02\x00\x10\x00")
    a = io.parse_npy(_npy("{'descr': '<f8', 'fortran_order': False, 'shape': (3,), }", body, version=2))
    assert a.shape == (3,) and a.data.tolist() == [1.0, 2.0, 3.0]
    s = io.parse_npy(_npy("{'descr': '<f8', 'fortran_order': False, 'shape': (), }", body))
    assert s.shape == () and s.data.tolist() == [1.0]


def _spoc(path, sector, rows):
    """A SPOC-like light-curve product: rows of (time, flux, err, quality)."""
    primary = _pad(b"".join(_card(k, v) for k, v in [
        ("SIMPLE", "T"), ("BITPIX", "8"), ("NAXIS", "0"), ("TICID", "123456789"), ("SECTOR", str(sector)),
        ("TESSMAG", "9.5"), ("TEFF", "5700.0"), ("RADIUS", "1.02"), ("LOGG", "4.4")]) + b"END".ljust(80), b" ")
    cols = [("TIME", "D"), ("PDCSAP_FLUX", "E"), ("PDCSAP_FLUX_ERR", "E"), ("MOM_CENTR1", "D"), ("MOM_CENTR2", "D"),
            ("QUALITY", "J")]
    cards = [("XTENSION", "'BINTABLE'"), ("BITPIX", "8"), ("NAXIS", "2"), ("NAXIS1", "36"),
             ("NAXIS2", str(len(rows))), ("PCOUNT", "0"), ("GCOUNT", "1"), ("TFIELDS", str(len(cols)))]
    for i, (name, form) in enumerate(cols, 1):
        cards += [(f"TTYPE{i}", f"'{name}'"), (f"TFORM{i}", f"'{form}'")]
    cards += [("EXTNAME", "'LIGHTCURVE'"), ("BJDREFI", "2457000"), ("BJDREFF", "0.5"), ("CROWDSAP", "0.99")]
    ext = _pad(b"".join(_card(k, v) for k, v in cards) + b"END".ljust(80), b" ")
    data = b"".join(struct.pack(">dffddi", t, f, e, 10.0, 20.0, q) for t, f, e, q in rows)
    path.write_bytes(primary + ext + _pad(data, b"\0"))


def test_read_light_curve_applies_the_quality_mask_and_bjd_reference(tmp_path):
    # fits.rs:284-333 with the default bitmask 17087 (fits.rs:214-217)
    rows = [(1.0, 100.0, 1.0, 0), (2.0, 101.0, 1.0, 1), (3.0, 102.0, 1.0, 2048), (4.0, math.nan, 1.0, 0),
            (math.nan, 103.0, 1.0, 0), (6.0, 104.0, 1.0, 16384), (7.0, 105.0, 1.5, 4096), (8.0, 106.0, 1.0, 512)]
    path = tmp_path / "lc.fits"
    _spoc(path, 14, rows)
    lc = io.read_light_curve(str(path))
    assert lc.tic == 123456789 and lc.sector == 14 and lc.points_total == 8
    # kept: quality 0, 2048 (bit 11) and 4096 (bit 12); dropped: bits 0, 14 and 9, NaN flux, NaN time
    assert (lc.time_bjd - 2457000.5).tolist() == [1.0, 3.0, 7.0]
    assert lc.flux.tolist() == [100.0, 102.0, 105.0] and lc.flux_err.tolist() == [1.0, 1.0, 1.5]
    assert lc.star.tmag == 9.5 and lc.star.teff == 5700.0 and lc.crowdsap == 0.99
    assert lc.target_pixel is None  # no APERTURE extension
    obs = io.read_inputs([str(path)])
    assert obs.time.tolist() == lc.time_bjd.tolist() and obs.err is not None and obs.group.tolist() == [0, 0, 0]
