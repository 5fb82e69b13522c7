"""Bounded streaming voxel on the device (srcu_stream_voxel_*) vs the oracle.

Bar: the voxel key set, order and point counts are exact; positions are the
f32 of the FP64 mean (checked within 1e-5 of the leaf, and equal to the
oracle's f32 in all but rare FP64 rounding ties); FP64 attribute means
within 1e-12 relative.  The reference's own streaming tests
(streaming.rs:1098-1171) run through the Python mirror."""
import numpy as np
import pytest

import oracle
import spatialrust_b200 as sr
from spatialrust_b200 import _native, synthetic
from spatialrust_b200.streaming import (MemoryChunkSource, SpoolOptions, StreamingVoxelConfig,
                                        StreamingVoxelSource)

pytestmark = pytest.mark.gpu
F = np.float32


def xyz_cloud(points):
    b = sr.PointCloudBuilder.xyz()
    for p in points:
        b.push_point(p)
    return b.build()


def positions(src):
    out = []
    while (c := src.next_chunk()) is not None:
        out.extend(map(list, zip(c.field("x").tolist(), c.field("y").tolist(), c.field("z").tolist())))
    return out


def check_stream(ctx, x, y, z, attrs=(), leaf=0.1, chunk=100_000, device_run=0, f64=None):
    f64 = f64 if f64 is not None else [a.dtype == np.float64 for a in attrs]
    sv = _native.StreamVoxel(ctx, leaf, f64, device_run_points=device_run)
    for lo in range(0, len(x), chunk):
        sv.push(x[lo:lo + chunk], y[lo:lo + chunk], z[lo:lo + chunk], [a[lo:lo + chunk] for a in attrs])
    info = sv.finish()
    gx, gy, gz, ga, keys, counts = sv.fetch()
    sv.close()
    ref = oracle.stream_voxel(x, y, z, [np.asarray(a, np.float64) for a in attrs], leaf=leaf)
    assert info["voxels"] == len(ref.counts)
    assert np.array_equal(keys, ref.keys)
    assert np.array_equal(counts, ref.counts)
    pos = np.stack([gx, gy, gz], 1)
    assert np.max(np.abs(pos.astype(np.float64) - ref.pos)) <= 1e-5 * leaf + 1e-6 * np.abs(ref.pos).max()
    assert np.mean(pos == ref.pos) > 0.999
    if attrs:
        assert np.allclose(ga, ref.attrs, rtol=1e-12, atol=0)
    return info


# ---- the reference's streaming tests --------------------------------------

def test_output_identical_across_chunk_and_run_sizes(tmp_path):
    # streaming.rs:1098-1130
    pts = [[1.3, 0.0, 0.0], [0.1, 0.0, 0.0], [1.1, 0.0, 0.0], [0.2, 0.0, 0.0], [2.8, 0.0, 0.0]]
    sp = SpoolOptions(str(tmp_path), 16 * 1024)
    a = StreamingVoxelSource.try_build(MemoryChunkSource(xyz_cloud(pts), 1),
                                       StreamingVoxelConfig(1.0, 2, 8, sp))
    b = StreamingVoxelSource.try_build(MemoryChunkSource(xyz_cloud(pts), 4),
                                       StreamingVoxelConfig(1.0, 3, 8, sp))
    pa, pb = positions(a), positions(b)
    assert a.spool_bytes() > 0 and a.run_count() > 1
    assert pa == pb
    assert pa == np.array([[0.15, 0, 0], [1.2, 0, 0], [2.8, 0, 0]], F).tolist()


def test_attributes_averaged_across_runs(tmp_path):
    # streaming.rs:1132-1149
    b = sr.PointCloudBuilder(sr.StandardSchemas.point_xyzi())
    for p in ([0.1, 0.0, 0.0, 10.0], [0.2, 0.0, 0.0, 20.0], [1.1, 0.0, 0.0, 50.0]):
        b.push_point(p)
    src = StreamingVoxelSource.try_build(MemoryChunkSource(b.build(), 2),
                                         StreamingVoxelConfig(1.0, 1, 4,
                                                              SpoolOptions(str(tmp_path), 4096)))
    assert src.next_chunk().intensity().tolist() == [15.0, 50.0]


def test_spool_and_run_limits_fail_closed(tmp_path):
    # streaming.rs:1151-1171
    pts = xyz_cloud([[0.0, 0.0, 0.0], [1.0, 0.0, 0.0]])
    with pytest.raises(sr.InvalidArgument):
        StreamingVoxelSource.try_build(MemoryChunkSource(pts, 2),
                                       StreamingVoxelConfig(0.1, 2, 2, SpoolOptions(str(tmp_path), 8)))
    with pytest.raises(sr.InvalidArgument):
        StreamingVoxelSource.try_build(MemoryChunkSource(pts, 2),
                                       StreamingVoxelConfig(0.1, 1, 1, SpoolOptions(str(tmp_path), 4096)))


# ---- parity on larger streams ----------------------------------------------

def test_scan_stream_parity_with_runs_and_merge(cuda_ctx):
    c = synthetic.georef_scan(600_000, seed=51)
    # shuffled, so every voxel's points are spread over many device runs
    perm = np.random.default_rng(51).permutation(len(c.x))
    x, y, z, i = c.x[perm], c.y[perm], c.z[perm], c.intensity[perm]
    info = check_stream(cuda_ctx, x, y, z, [i], leaf=0.1, chunk=70_000, device_run=50_000)
    assert info["device_runs"] == 12 and info["partial_records"] > info["voxels"]


def test_long_voxels_in_runs_and_in_the_merge(cuda_ctx):
    # 3 voxels of ~100k points: long segments in every run, and (with 1000-point
    # device runs) more than 64 partial records per voxel in the merge
    rng = np.random.default_rng(7)
    p = rng.uniform(0, 3, (300_000, 3)).astype(F)
    p[:, 1:] = F(0.5)
    gps = 1e9 + rng.uniform(0, 100, 300_000)
    info = check_stream(cuda_ctx, p[:, 0], p[:, 1], p[:, 2], [gps], leaf=1.0, chunk=25_000,
                        device_run=1000)
    assert info["voxels"] == 3 and info["device_runs"] == 300


def test_non_finite_points_are_skipped_and_negative_keys(cuda_ctx):
    rng = np.random.default_rng(8)
    p = rng.normal(0, 5, (50_000, 3)).astype(F)
    p[::7, 0] = np.nan
    p[::11, 2] = np.inf
    p[::13, 1] = -np.inf
    info = check_stream(cuda_ctx, p[:, 0], p[:, 1], p[:, 2], leaf=0.25, chunk=9_999, device_run=20_000)
    finite = np.all(np.isfinite(p), axis=1).sum()
    assert info["finite_points"] == finite and info["points"] == 50_000


def test_all_points_non_finite_or_empty(cuda_ctx):
    sv = _native.StreamVoxel(cuda_ctx, 1.0)
    sv.push(np.full(10, np.nan, F), np.zeros(10, F), np.zeros(10, F))
    assert sv.finish()["voxels"] == 0
    sv.close()
    sv = _native.StreamVoxel(cuda_ctx, 1.0)
    assert sv.finish()["voxels"] == 0
    sv.close()


def test_device_chunks_and_f32_attributes(cuda_ctx):
    import torch
    c = synthetic.shapes_scene(200_000, seed=12)
    inten = np.random.default_rng(12).random(200_000).astype(F)
    host = _native.StreamVoxel(cuda_ctx, 0.05, [False])
    dev = _native.StreamVoxel(cuda_ctx, 0.05, [False])
    for lo in range(0, 200_000, 64_000):
        sl = slice(lo, lo + 64_000)
        host.push(c.x[sl], c.y[sl], c.z[sl], [inten[sl]])
        dev.push(*[torch.from_numpy(np.ascontiguousarray(a[sl])).cuda() for a in (c.x, c.y, c.z)],
                 [torch.from_numpy(inten[sl]).cuda()])
    assert host.finish()["voxels"] == dev.finish()["voxels"]
    for a, b in zip(host.fetch(), dev.fetch()):
        assert np.array_equal(a, b)
    host.close()
    dev.close()


def test_key_range_error_and_bad_arguments(cuda_ctx):
    sv = _native.StreamVoxel(cuda_ctx, 1e-12)
    sv.push(np.array([1e30], F), np.zeros(1, F), np.zeros(1, F))
    with pytest.raises(sr.InvalidArgument, match="64-bit range"):
        sv.finish()
    sv.close()
    for leaf in (0.0, -1.0, float("nan"), float("inf")):
        with pytest.raises(sr.InvalidArgument):
            _native.StreamVoxel(cuda_ctx, leaf)
    sv = _native.StreamVoxel(cuda_ctx, 1.0, [False])
    with pytest.raises(sr.InvalidArgument):
        sv.push(np.zeros(3, F), np.zeros(3, F), np.zeros(3, F))
    with pytest.raises(sr.BufferLengthMismatch):
        sv.push(np.zeros(3, F), np.zeros(2, F), np.zeros(3, F), [np.zeros(3, F)])
    sv.close()
