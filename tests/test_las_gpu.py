"""LAS record decoding on the device (srcu_las_decode) vs the oracle.

Bar: bit-exact.  Every column is integer/byte work or the f32 of the same
step-rounded FP64 arithmetic (scale * X + offset [- origin])."""
import numpy as np
import pytest

import oracle
from spatialrust_b200 import las, synthetic
from spatialrust_b200.streaming import SpoolOptions, StreamingVoxelConfig, StreamingVoxelSource

pytestmark = pytest.mark.gpu
F = np.float32


def header_for(fmt, rl, scale=(0.01, 0.02, 0.005), offset=(450000.0, 3900000.0, 50.0)):
    return las.LasHeader((1, 4), 375, 375, fmt, rl, 0, scale, offset, (0,) * 3, (0,) * 3, False)


def assert_same(got: dict, ref: dict, h):
    for k in ("x", "y", "z", "intensity", "classification"):
        g = got[k].cpu().numpy() if hasattr(got[k], "cpu") else got[k]
        assert np.array_equal(g.view(np.uint32) if g.dtype == np.float32 else g,
                              ref[k].view(np.uint32) if ref[k].dtype == np.float32 else ref[k]), k
    if h.has_gps_time:
        g = got["gps_time"].cpu().numpy() if hasattr(got["gps_time"], "cpu") else got["gps_time"]
        assert np.array_equal(g.view(np.uint64), ref["gps_time"].view(np.uint64))
    if h.has_color:
        for c in ("red", "green", "blue"):
            g = got[c].cpu().numpy() if hasattr(got[c], "cpu") else got[c]
            assert np.array_equal(g.view(np.uint16), ref[c])


@pytest.mark.parametrize("fmt", range(11))
def test_every_format_bit_exact(cuda_ctx, fmt):
    std = las.LAS_LAYOUTS[fmt][0]
    rng = np.random.default_rng(100 + fmt)
    for rl in (std, std + 3):  # odd extra bytes: records straddle the 16-byte staging lines
        raw = rng.integers(0, 256, (50_001, rl), dtype=np.uint8)
        h = header_for(fmt, rl)
        got = las.decode_records(raw, h)
        ref = oracle.las_decode(raw, fmt, rl, h.scale, h.offset)
        assert_same(got, ref, h)


def test_device_records_at_every_alignment(cuda_ctx):
    import torch
    rng = np.random.default_rng(3)
    rl = 34
    raw = rng.integers(0, 256, 20_000 * rl + 16, dtype=np.uint8)
    h = header_for(3, rl)
    dev = torch.from_numpy(raw).cuda()
    for shift in range(16):
        rec = raw[shift:shift + 20_000 * rl]
        got = las.decode_records(dev[shift:shift + 20_000 * rl], h)
        assert got["x"].is_cuda
        assert_same(got, oracle.las_decode(rec, 3, rl, h.scale, h.offset), h)


def test_fp64_origin_keeps_georeferenced_precision(cuda_ctx):
    c = synthetic.georef_scan(300_000, seed=21)
    world = [c.x.astype(np.float64) + c.origin[0], c.y.astype(np.float64) + c.origin[1],
             c.z.astype(np.float64) + c.origin[2]]
    buf = las.encode_las(*world, point_format=1, scale=(0.001,) * 3,
                         offset=tuple(np.floor(c.origin)), intensity=(c.intensity * 1000).astype(int))
    h = las.parse_header(buf)
    rec = np.frombuffer(buf, np.uint8, h.point_count * h.record_length, h.offset_to_point_data)
    for origin in (None, tuple(c.origin)):
        got = las.decode_records(rec, h, origin)
        assert_same(got, oracle.las_decode(rec, 1, h.record_length, h.scale, h.offset, origin), h)
    local = las.decode_records(rec, h, tuple(c.origin))
    # millimetre records: the local f32 columns are within 0.5 mm (+ f32 rounding) of the scan
    assert np.max(np.abs(local["x"] - c.x)) < 6e-4
    plain = las.decode_records(rec, h)  # reference semantics: f32 of the world coordinate
    assert np.max(np.abs(plain["x"].astype(np.float64) - world[0])) > 1e-3


def test_read_las_and_chunks_into_the_streaming_voxel(cuda_ctx, tmp_path):
    c = synthetic.georef_scan(250_000, seed=22)
    buf = las.encode_las(c.x, c.y, c.z, point_format=3, scale=(1e-4,) * 3,
                         intensity=(c.intensity * 65535).astype(int),
                         classification=np.arange(250_000) % 32,
                         gps_time=np.linspace(1e9, 1e9 + 60, 250_000),
                         rgb=[np.arange(250_000) % 65536] * 3)
    path = tmp_path / "scan.las"
    path.write_bytes(buf)
    cloud = las.read_las(str(path))
    assert cloud.schema.names() == ["x", "y", "z", "intensity", "classification", "gps_time",
                                    "red", "green", "blue"]
    assert cloud.metadata["frame_id"] == "las" and len(cloud) == 250_000
    h = las.parse_header(buf)
    rec = np.frombuffer(buf, np.uint8, h.point_count * h.record_length, h.offset_to_point_data)
    ref = oracle.las_decode(rec, 3, h.record_length, h.scale, h.offset)
    assert np.array_equal(cloud.field("x"), ref["x"])
    assert np.array_equal(cloud.field("red"), ref["red"])
    reader = las.LasReader.open(str(path))
    assert reader.header().point_count == 250_000
    assert reader.read_cloud() == cloud
    with pytest.raises(las.LasError):
        reader.read_cloud()
    # LAS chunks -> bounded streaming voxel, against the oracle on the decoded columns
    src = las.LasChunkSource(str(path), 40_000)
    cfg = StreamingVoxelConfig(0.2, 100_000, 8, SpoolOptions(str(tmp_path), 1 << 30))
    sv = StreamingVoxelSource.try_build(src, cfg)
    keys, counts = sv.keys_and_counts()
    want = oracle.stream_voxel(ref["x"], ref["y"], ref["z"], [ref["gps_time"]], leaf=0.2)
    assert np.array_equal(keys, want.keys) and np.array_equal(counts, want.counts)
    out = sv.next_chunk()
    assert out.schema == cloud.schema and out.field("classification").dtype == np.uint8
    assert np.allclose(out.field("gps_time")[:100], want.attrs[:100, 0], rtol=1e-12)


def test_errors(cuda_ctx):
    h = header_for(0, 20)
    with pytest.raises(las.LasError):
        las.decode_records(np.zeros(30, np.uint8), h)
    assert len(las.decode_records(np.zeros(0, np.uint8), h)["x"]) == 0
