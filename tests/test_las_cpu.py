"""LAS header parsing, schema mapping and the oracle's record decoding (no GPU).

The decode oracle is pinned two ways: the reference's own LAS round-trip test
values (crates/spatialrust-io/src/las/reader.rs:311-330) and an independent
numpy reading of the ASPRS LAS 1.4 record layouts (structured dtypes)."""
import numpy as np
import pytest

import oracle
import spatialrust_b200 as sr
from spatialrust_b200 import las


@pytest.fixture(scope="module", autouse=True)
def _built():
    oracle.build()


def records_of(buf: bytes, h):
    return np.frombuffer(buf, np.uint8, h.point_count * h.record_length, h.offset_to_point_data)


# independent layouts: (name, numpy type) per field, format by format
BASE = [("X", "<i4"), ("Y", "<i4"), ("Z", "<i4"), ("intensity", "<u2")]
LEGACY = BASE + [("flags", "u1"), ("cls", "u1"), ("angle", "i1"), ("user", "u1"), ("psid", "<u2")]
EXT = BASE + [("ret", "u1"), ("flags", "u1"), ("cls", "u1"), ("user", "u1"), ("angle", "<i2"),
              ("psid", "<u2"), ("gps", "<f8")]
RGB = [("r", "<u2"), ("g", "<u2"), ("b", "<u2")]
WAVE = [("wave", "V29")]
LAYOUTS = {0: LEGACY, 1: LEGACY + [("gps", "<f8")], 2: LEGACY + RGB,
           3: LEGACY + [("gps", "<f8")] + RGB, 4: LEGACY + [("gps", "<f8")] + WAVE,
           5: LEGACY + [("gps", "<f8")] + RGB + WAVE, 6: EXT, 7: EXT + RGB,
           8: EXT + RGB + [("nir", "<u2")], 9: EXT + WAVE, 10: EXT + RGB + [("nir", "<u2")] + WAVE}


def test_reference_roundtrip_values():
    # reader.rs:311-330: (1, 2, 3, 100), (4, 5, 6, 200) back within 1e-5 / 1e-3
    buf = las.encode_las([1.0, 4.0], [2.0, 5.0], [3.0, 6.0], point_format=0, intensity=[100, 200])
    h = las.parse_header(buf)
    d = oracle.las_decode(records_of(buf, h), h.point_format, h.record_length, h.scale, h.offset)
    assert len(d["x"]) == 2
    assert abs(d["x"][0] - 1.0) < 1e-5 and abs(d["y"][1] - 5.0) < 1e-5 and abs(d["z"][1] - 6.0) < 1e-5
    assert abs(d["intensity"][0] - 100.0) < 1e-3


@pytest.mark.parametrize("fmt", range(11))
def test_oracle_decode_matches_spec_layouts(fmt):
    std = las.LAS_LAYOUTS[fmt][0]
    assert np.dtype(LAYOUTS[fmt]).itemsize == std
    rng = np.random.default_rng(fmt)
    rl = std + 5  # extra bytes after the standard fields
    raw = rng.integers(0, 256, (3000, rl), dtype=np.uint8)
    view = raw[:, :std].copy().view(np.dtype(LAYOUTS[fmt])).reshape(-1)
    scale, offset = (0.01, 0.02, 0.005), (450000.0, 3900000.0, 50.0)
    d = oracle.las_decode(raw, fmt, rl, scale, offset)
    for a, k in enumerate("XYZ"):
        want = (scale[a] * view[k].astype(np.float64) + offset[a]).astype(np.float32)
        assert np.array_equal(d["xyz"[a]], want)
    assert np.array_equal(d["intensity"], view["intensity"].astype(np.float32))
    assert np.array_equal(d["classification"], view["cls"] if fmt >= 6 else view["cls"] & 0x1F)
    names = dict(LAYOUTS[fmt])
    if "gps" in names:
        assert np.array_equal(d["gps_time"].view(np.uint64), view["gps"].view(np.uint64))
    if "r" in names:
        for c, k in zip(("red", "green", "blue"), "rgb"):
            assert np.array_equal(d[c], view[k])


def test_origin_is_subtracted_in_fp64():
    x = np.array([450123.456, 450999.999])
    buf = las.encode_las(x, [3900000.5, 3900001.25], [10.0, 11.0], point_format=1,
                         offset=(450000.0, 3900000.0, 0.0))
    h = las.parse_header(buf)
    o = (450000.0, 3900000.0, 0.0)
    d = oracle.las_decode(records_of(buf, h), 1, h.record_length, h.scale, h.offset, origin=o)
    assert d["x"].tolist() == [np.float32(123.456), np.float32(999.999)]
    plain = oracle.las_decode(records_of(buf, h), 1, h.record_length, h.scale, h.offset)
    assert plain["x"].tolist() == [np.float32(450123.456), np.float32(450999.999)]


def test_header_fields_and_errors():
    buf = las.encode_las([0.0], [0.0], [0.0], point_format=3, version=(1, 2))
    h = las.parse_header(buf)
    assert h.version == (1, 2) and h.point_count == 1 and h.record_length == 34
    assert h.has_gps_time and h.has_color and not h.compressed
    compressed = bytearray(buf)
    compressed[104] |= 0x80  # LAZ sets the high bits of the format byte
    assert las.parse_header(bytes(compressed)).compressed
    with pytest.raises(las.LasError):
        las.parse_header(b"XXXX" + buf[4:])
    bad = bytearray(buf)
    bad[104] = 11
    with pytest.raises(las.LasError):
        las.parse_header(bytes(bad))
    with pytest.raises(sr.UnsupportedDType):
        las.decode_records(np.zeros(34, np.uint8), las.parse_header(bytes(compressed)))


def test_schema_for_las_header():
    # schema.rs:27-52
    names = {f: las.schema_for_las_header(las.parse_header(las.encode_las([0.0], [0.0], [0.0],
                                                                          point_format=f))).names()
             for f in (0, 1, 2, 3, 6, 7)}
    base = ["x", "y", "z", "intensity", "classification"]
    assert names[0] == base
    assert names[1] == base + ["gps_time"] and names[6] == base + ["gps_time"]
    assert names[2] == base + ["red", "green", "blue"]
    assert names[3] == base + ["gps_time", "red", "green", "blue"] == names[7]
