"""CUDA voxel centroid downsample vs the CPU oracle (reference restatement).

Bar: the occupied voxel-key set and per-voxel counts are bit-exact, and so are
the centroids whenever every voxel is reduced in the reference's order (voxels
of <= 32 points); larger voxels are reduced by a warp in FP64 and must stay
within 1e-5 * leaf of the oracle."""
import numpy as np
import pytest

import oracle
import spatialrust_b200 as sr
from spatialrust_b200 import _native, synthetic

pytestmark = pytest.mark.gpu
F = np.float32


def build_cloud(schema, rows):
    b = sr.PointCloudBuilder(schema)
    for r in rows:
        b.push_point(r)
    return b.build()


def gpu_voxel(ctx, x, y, z, attrs=(), leaf=1.0, origin=None):
    return ctx.voxel_centroid(x, y, z, list(attrs), leaf=leaf, origin=origin, want_keys=True)


def assert_voxel_parity(ctx, x, y, z, attrs=(), leaf=1.0, origin=None, exact=True):
    cols, keys, counts = gpu_voxel(ctx, x, y, z, attrs, leaf, origin)
    ref = oracle.voxel_centroid(x, y, z, list(attrs), leaf=leaf, origin=origin)
    assert keys.shape == ref.keys.shape
    assert np.array_equal(keys, ref.keys), "voxel key set differs"
    assert np.array_equal(counts, ref.counts), "per-voxel counts differ"
    for c, (g, r) in enumerate(zip(cols, ref.fields)):
        err = np.max(np.abs(g.astype(np.float64) - r.astype(np.float64))) if len(g) else 0.0
        assert err <= 1e-5 * leaf, f"column {c}: max error {err}"
        if exact:
            assert np.array_equal(g, r), f"column {c}: {np.count_nonzero(g != r)} values differ"
    return cols, keys, counts


# ---- the reference's known-answer tests through the public API ------------

def test_centroid_downsample_reduces_points():
    # voxel.rs:1270-1288
    cloud = build_cloud(sr.StandardSchemas.point_xyz(), [[0, 0, 0], [0.1, 0, 0], [1.0, 0, 0], [1.1, 0, 0]])
    out = sr.VoxelGridDownsample(sr.VoxelGridDownsampleConfig.centroid(0.5).without_gpu_min_points()
                                 ).filter_with_policy(cloud, sr.GpuCuda)
    assert len(out) == 2
    x, _, _ = out.positions3()
    assert abs(x[0] - 0.05) < 1e-5 and abs(x[1] - 1.05) < 1e-5


def test_explicit_origin_uses_floor_for_negative_voxels():
    # voxel.rs:1290-1306
    cloud = build_cloud(sr.StandardSchemas.point_xyz(), [[-0.6, 0, 0], [-0.1, 0, 0], [0.1, 0, 0]])
    cfg = sr.VoxelGridDownsampleConfig.centroid(1.0).with_origin((0.0, 0.0, 0.0))
    out = sr.VoxelGridDownsample(cfg).filter_with_policy(cloud, sr.GpuCuda)
    x, _, _ = out.positions3()
    assert len(out) == 2
    assert abs(x[0] - -0.35) < 1e-5 and abs(x[1] - 0.1) < 1e-5


def test_default_origin_matches_explicit_min_origin():
    # voxel.rs:1308-1327
    rows = [[-1.2, 0.0, 0.0], [-1.1, 0.1, 0.0], [-0.7, 0.0, 0.0], [0.4, 1.0, 0.0], [0.6, 1.0, 0.0]]
    cloud = build_cloud(sr.StandardSchemas.point_xyz(), rows)
    a = sr.VoxelGridDownsample(sr.VoxelGridDownsampleConfig.centroid(0.5)).filter_with_policy(
        cloud, sr.GpuCuda)
    b = sr.VoxelGridDownsample(sr.VoxelGridDownsampleConfig.centroid(0.5).with_origin(
        (F(-1.2), 0.0, 0.0))).filter_with_policy(cloud, sr.GpuCuda)
    assert a == b


def test_average_intensity_in_centroid_mode():
    # voxel.rs:1342-1355 and the GPU variant voxel.rs:1389-1409
    cloud = build_cloud(sr.StandardSchemas.point_xyzi(), [[0, 0, 0, 0.2], [0.1, 0, 0, 0.8]])
    out = sr.VoxelGridDownsample(sr.VoxelGridDownsampleConfig.centroid(1.0)).filter_with_policy(
        cloud, sr.GpuCuda)
    assert len(out) == 1
    assert abs(out.intensity()[0] - 0.5) < 1e-5


def test_u8_rgb_average_matches_cpu():
    # voxel.rs:1411-1443: u8 channels averaged then rounded, exact
    cloud = build_cloud(sr.StandardSchemas.point_xyzrgb(),
                        [[0, 0, 0, 10, 20, 30], [0.1, 0, 0, 30, 40, 50]])
    out = sr.VoxelGridDownsample(sr.VoxelGridDownsampleConfig.centroid(1.0)).filter_with_policy(
        cloud, sr.GpuCuda)
    assert out.field("r").tolist() == [20] and out.field("g").tolist() == [30]
    assert out.field("b").tolist() == [40] and out.field("r").dtype == np.uint8


def test_mvp_load_voxel_downsample():
    # crates/spatialrust/tests/mvp_pipeline.rs:1-26
    x = np.arange(10, dtype=np.float32) * F(0.1)
    cloud = sr.PointCloud(sr.StandardSchemas.point_xyz(),
                          {"x": x, "y": np.zeros(10, F), "z": np.zeros(10, F)})
    out = sr.VoxelGridDownsample(sr.VoxelGridDownsampleConfig.centroid(0.5)).filter_with_policy(
        cloud, sr.Auto)
    xs, _, _ = out.positions3()
    assert len(out) == 2 and abs(xs[0] - 0.2) < 1e-5 and abs(xs[1] - 0.7) < 1e-5


def test_receipt_records_stages_and_transfers():
    cloud = build_cloud(sr.StandardSchemas.point_xyzi(), [[0, 0, 0, 0.2], [0.1, 0, 0, 0.8]])
    res = sr.VoxelGridDownsample(sr.VoxelGridDownsampleConfig.centroid(1.0)
                                 ).filter_with_policy_and_receipt(cloud, sr.GpuCuda)
    assert res.receipt.stages == ["voxel-downsample", "gpu-readback"]
    assert res.receipt.transfers[sr.TransferDirection.HostToDevice] == 2 * 16
    assert res.receipt.resolved_policy == sr.GpuCuda


# ---- parity at benchmark shapes --------------------------------------------

def test_uniform_100k_leaf4_bit_exact(cuda_ctx):
    c = synthetic.uniform_cube(100_000, seed=0)
    cols, keys, counts = assert_voxel_parity(cuda_ctx, c.x, c.y, c.z, [c.intensity], leaf=4.0)
    assert 15_500 < len(counts) <= 15_625


@pytest.mark.parametrize("leaf", [0.1, 0.5])
def test_georeferenced_2m_both_leaves(cuda_ctx, leaf):
    c = synthetic.georef_scan(2_000_000, seed=1)
    _, _, counts = assert_voxel_parity(cuda_ctx, c.x, c.y, c.z, [c.intensity], leaf=leaf,
                                       exact=False)
    assert counts.sum() == c.n


def test_georeferenced_centroids_bit_exact_when_short(cuda_ctx):
    c = synthetic.georef_scan(300_000, seed=7)
    assert_voxel_parity(cuda_ctx, c.x, c.y, c.z, [c.intensity], leaf=0.1, exact=True)


def test_large_voxels_use_warp_reduction(cuda_ctx):
    c = synthetic.uniform_cube(300_000, seed=4)
    _, _, counts = assert_voxel_parity(cuda_ctx, c.x, c.y, c.z, [c.intensity], leaf=30.0,
                                       exact=False)
    assert counts.max() > 1000


def test_single_voxel_all_points(cuda_ctx):
    rng = np.random.default_rng(9)
    p = rng.random((50_000, 3), dtype=np.float32)
    cols, keys, counts = assert_voxel_parity(cuda_ctx, p[:, 0], p[:, 1], p[:, 2], leaf=10.0,
                                             exact=False)
    assert counts.tolist() == [50_000]


@pytest.mark.parametrize("n", [1, 2, 31, 2047, 2048, 2049, 4095, 4096, 4097, 12_289])
def test_tile_boundaries(cuda_ctx, n):
    rng = np.random.default_rng(n)
    p = rng.random((n, 3), dtype=np.float32) * F(20)
    i = rng.random(n, dtype=np.float32)
    assert_voxel_parity(cuda_ctx, p[:, 0], p[:, 1], p[:, 2], [i], leaf=1.0)


def test_explicit_origin_negative_keys(cuda_ctx):
    rng = np.random.default_rng(12)
    p = (rng.random((80_000, 3), dtype=np.float32) - F(0.5)) * F(40)
    assert_voxel_parity(cuda_ctx, p[:, 0], p[:, 1], p[:, 2], [p[:, 0] * 2], leaf=0.7,
                        origin=(F(3.3), F(-2.0), F(0.25)))


def test_many_attribute_columns(cuda_ctx):
    rng = np.random.default_rng(13)
    p = rng.random((40_000, 3), dtype=np.float32) * F(10)
    attrs = [rng.random(40_000, dtype=np.float32) * F(k + 1) for k in range(6)]
    assert_voxel_parity(cuda_ctx, p[:, 0], p[:, 1], p[:, 2], attrs, leaf=0.5)


def test_nan_coordinates_follow_saturating_cast(cuda_ctx):
    # voxel_key_nonnegative: NaN `as i64` is 0; compute_bounds ignores NaN
    rng = np.random.default_rng(14)
    p = rng.random((5000, 3), dtype=np.float32) * F(10) + F(1)
    p[::97, 1] = np.nan
    cols, keys, counts = gpu_voxel(cuda_ctx, p[:, 0], p[:, 1], p[:, 2], leaf=1.0)
    ref = oracle.voxel_centroid(p[:, 0], p[:, 1], p[:, 2], leaf=1.0)
    assert np.array_equal(keys, ref.keys) and np.array_equal(counts, ref.counts)
    for g, r in zip(cols, ref.fields):
        assert np.array_equal(g, r, equal_nan=True)


def test_key_overflow_is_reported(cuda_ctx):
    x = np.array([0.0, 1e6], np.float32)
    with pytest.raises(_native.KeyOverflow):
        cuda_ctx.voxel_centroid(x, x, x, leaf=1e-4)
    # the context stays usable afterwards
    cols, _, counts = cuda_ctx.voxel_centroid(x, x, x, leaf=1.0)
    assert counts.tolist() == [1, 1]


def test_infinite_coordinate_is_reported(cuda_ctx):
    x = np.array([0.0, np.inf, 1.0], np.float32)
    with pytest.raises(_native.KeyOverflow):
        cuda_ctx.voxel_centroid(x, np.zeros(3, F), np.zeros(3, F), leaf=1.0)


def test_repeated_calls_of_varying_size(cuda_ctx):
    for n, seed in ((70_000, 1), (1_000, 2), (250_000, 3), (70_000, 1)):
        c = synthetic.uniform_cube(n, seed=seed, extent=50.0)
        assert_voxel_parity(cuda_ctx, c.x, c.y, c.z, [c.intensity], leaf=2.0)


def test_device_resident_inputs_match_host_inputs(cuda_ctx):
    import torch
    c = synthetic.uniform_cube(60_000, seed=21)
    host = gpu_voxel(cuda_ctx, c.x, c.y, c.z, [c.intensity], leaf=3.0)
    dev = [torch.from_numpy(a).cuda() for a in (c.x, c.y, c.z, c.intensity)]
    devr = gpu_voxel(cuda_ctx, dev[0], dev[1], dev[2], [dev[3]], leaf=3.0)
    for a, b in zip(host[0], devr[0]):
        assert np.array_equal(a, b)
    assert np.array_equal(host[1], devr[1]) and np.array_equal(host[2], devr[2])


# ---- ApproximateFirst and the First attribute policy (general path) ---------

def assert_general_parity(ctx, x, y, z, attrs, leaf, approximate, attribute_first, origin=None):
    cols, keys, counts = ctx.voxel_centroid(x, y, z, list(attrs), leaf=leaf, origin=origin,
                                            want_keys=True, approximate=approximate,
                                            attribute_first=attribute_first)
    ref = oracle.voxel_general(x, y, z, list(attrs), leaf=leaf, origin=origin,
                               approximate=approximate, attribute_first=attribute_first)
    assert np.array_equal(keys, ref.keys) and np.array_equal(counts, ref.counts)
    for c, (g, r) in enumerate(zip(cols, ref.fields)):
        assert np.array_equal(g, r), f"column {c}: {np.count_nonzero(g != r)} values differ"


def test_approximate_keeps_first_point_in_voxel():
    # voxel.rs:1329-1339
    cloud = build_cloud(sr.StandardSchemas.point_xyzi(), [[0, 0, 0, 0.2], [0.1, 0, 0, 0.9]])
    out = sr.VoxelGridDownsample(sr.VoxelGridDownsampleConfig.approximate(1.0)).filter_with_policy(
        cloud, sr.GpuCuda)
    assert len(out) == 1 and out.intensity()[0] == F(0.2)


def test_approximate_first_matches_cpu_four_points():
    # voxel.rs:1446-1471: x from the first point of each voxel, intensities exact
    cloud = build_cloud(sr.StandardSchemas.point_xyzi(),
                        [[0, 0, 0, 0.2], [0.1, 0, 0, 0.9], [1.0, 0, 0, 10], [1.1, 0, 0, 20]])
    out = sr.VoxelGridDownsample(sr.VoxelGridDownsampleConfig.approximate(0.5)).filter_with_policy(
        cloud, sr.GpuCuda)
    x, _, _ = out.positions3()
    assert x.tolist() == [0.0, 1.0]
    assert out.intensity().tolist() == [F(0.2), F(10.0)]


@pytest.mark.parametrize("approximate,attribute_first", [(True, True), (True, False), (False, True)])
def test_general_modes_bit_exact(cuda_ctx, approximate, attribute_first):
    # short voxels (thread path) and long voxels (warp path), with attributes
    c = synthetic.georef_scan(300_000, seed=12)
    extra = np.random.default_rng(3).random(c.n, dtype=np.float32)
    for leaf in (0.1, 2.0):
        assert_general_parity(cuda_ctx, c.x, c.y, c.z, [c.intensity, extra], leaf, approximate,
                              attribute_first)
    assert_general_parity(cuda_ctx, c.x, c.y, c.z, [c.intensity], 0.25, approximate,
                          attribute_first, origin=(-3.0, -3.0, -1.0))


def test_u8_rgb_approximate_first_exact():
    rows = [[0.0, 0.0, 0.0, 10, 20, 30], [0.2, 0.0, 0.0, 200, 100, 0], [1.5, 0.0, 0.0, 7, 8, 9]]
    cloud = build_cloud(sr.StandardSchemas.point_xyzrgb(), rows)
    out = sr.VoxelGridDownsample(sr.VoxelGridDownsampleConfig.approximate(1.0)).filter_with_policy(
        cloud, sr.GpuCuda)
    assert out.field("r").tolist() == [10, 7] and out.field("b").tolist() == [30, 9]


def test_modes_per_cloud_in_one_batch():
    import torch
    clouds = [synthetic.georef_scan(n, seed=30 + i) for i, n in enumerate([40_000, 9_000, 25_000])]
    modes = [(True, True), (False, False), (False, True)]
    cols = [torch.from_numpy(np.concatenate([getattr(c, k) for c in clouds])).cuda()
            for k in ("x", "y", "z", "intensity")]
    offsets = np.concatenate([[0], np.cumsum([c.n for c in clouds])]).astype(np.int64)
    keep = _native._Keep()
    pts = _native.make_cloud(cols[0], cols[1], cols[2], [cols[3]], keep)
    ctx = _native.Context(0)
    ctx.batch_voxel_normals_enqueue(pts, offsets, [0.2] * 3, [1.0] * 3, modes=modes)
    voff = ctx.batch_voxel_offsets()
    out = ctx.frame_fetch(int(offsets[-1]), n_attrs=1)
    for b, (c, (a, f)) in enumerate(zip(clouds, modes)):
        lo, hi = int(voff[b]), int(voff[b + 1])
        if a or f:
            ref = oracle.voxel_general(c.x, c.y, c.z, [c.intensity], leaf=0.2, approximate=a,
                                       attribute_first=f)
        else:
            ref = oracle.voxel_centroid(c.x, c.y, c.z, [c.intensity], leaf=0.2)
        assert np.array_equal(out["counts"][lo:hi], ref.counts)
        for g, r in zip(out["columns"], ref.fields):
            assert np.array_equal(g[lo:hi], r), f"cloud {b}"
    ctx.close()


def test_approximate_first_xyzinormal():
    # voxel.rs:1474-1500: point_xyzinormal, approximate(0.5); CPU semantics take
    # every field (intensity and normals too) from each voxel's first point
    rows = [[0.0, 0.0, 0.0, 0.2, 0.0, 0.0, 1.0], [0.1, 0.0, 0.0, 0.9, 0.1, 0.0, 1.0],
            [1.0, 0.0, 0.0, 10.0, 0.0, 1.0, 0.0], [1.1, 0.0, 0.0, 20.0, 0.0, 0.0, 1.0]]
    cloud = build_cloud(sr.StandardSchemas.point_xyzinormal(), rows)
    out = sr.VoxelGridDownsample(sr.VoxelGridDownsampleConfig.approximate(0.5)).filter_with_policy(
        cloud, sr.GpuCuda)
    assert out.field("x").tolist() == [0.0, 1.0]
    assert out.field("intensity").tolist() == [F(0.2), F(10.0)]
    assert out.field("normal_y").tolist() == [0.0, 1.0]
    assert out.field("normal_z").tolist() == [1.0, 0.0]


def test_voxel_centroid_enqueue_matches_sync(cuda_ctx):
    # the voxel stage alone, device-resident, against the synchronous call
    import torch
    c = synthetic.georef_scan(250_000, seed=14)
    sync_cols, _, sync_counts = cuda_ctx.voxel_centroid(c.x, c.y, c.z, [c.intensity], leaf=0.1)
    dev = [torch.from_numpy(a).cuda() for a in (c.x, c.y, c.z, c.intensity)]
    keep = _native._Keep()
    cloud = _native.make_cloud(dev[0], dev[1], dev[2], [dev[3]], keep)
    cuda_ctx.voxel_centroid_enqueue(cloud, 0.1)
    v, _ = cuda_ctx.frame_check()
    assert v == len(sync_counts)
    got = cuda_ctx.frame_fetch(c.n, n_attrs=1)
    assert np.array_equal(got["counts"], sync_counts)
    for a, b in zip(got["columns"], sync_cols):
        assert np.array_equal(a, b)
