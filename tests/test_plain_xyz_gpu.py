"""The reference's plain-xyz voxel path on the device (SRCU_VOXEL_CENTROID_XYZ)
against the oracle's restatement of filter_cpu_xyz_centroid_fast
(crates/spatialrust-filtering/src/voxel.rs:550-636).

Bar: bit-exact -- the same voxels in the same first-seen order, the same
counts, and positions equal bit for bit (f32 sums in input order,
sum * (1 / count) in f32)."""
import numpy as np
import pytest

import oracle
import spatialrust_b200 as sr
from spatialrust_b200 import _native, synthetic

pytestmark = pytest.mark.gpu
F = np.float32


def bits(a):
    return np.asarray(a, F).view(np.uint32)


def check(ctx, x, y, z, leaf, origin=None):
    cols, keys, counts = ctx.voxel_centroid(x, y, z, (), leaf=leaf, origin=origin, want_keys=True,
                                            plain_xyz=True)
    ref = oracle.voxel_centroid(x, y, z, leaf=leaf, origin=origin, plain_xyz=True)
    assert len(counts) == len(ref.counts)
    assert np.array_equal(keys, ref.keys)
    assert np.array_equal(counts, ref.counts)
    for g, r in zip(cols, (ref.x, ref.y, ref.z)):
        nan = np.isnan(r)
        assert np.array_equal(np.isnan(g), nan)
        assert np.array_equal(bits(g)[~nan], bits(r)[~nan])
    return cols, keys, counts


def shuffled_scan(n, seed):
    c = synthetic.georef_scan(n, seed=seed)
    p = np.random.default_rng(seed).permutation(n)
    return c.x[p], c.y[p], c.z[p]


@pytest.mark.parametrize("leaf", [0.1, 0.5])
def test_shuffled_scan_bit_exact(cuda_ctx, leaf):
    x, y, z = shuffled_scan(300_000, 31)
    _, _, counts = check(cuda_ctx, x, y, z, leaf)
    assert counts.max() > 1


def test_explicit_origin_negative_keys(cuda_ctx):
    x, y, z = shuffled_scan(200_000, 32)
    check(cuda_ctx, x - F(50), y - F(80), z, 0.25, origin=(0.0, 0.0, 0.0))


def test_long_voxels_sum_sequentially(cuda_ctx):
    # two voxels of ~100k points each (one f32 running sum per voxel, in input
    # order) and a sprinkle of small ones, interleaved
    rng = np.random.default_rng(33)
    n = 200_000
    x = rng.uniform(0, 2, n).astype(F)
    y = rng.uniform(0, 1, n).astype(F)
    z = rng.uniform(0, 1, n).astype(F)
    x[::97] = rng.uniform(5, 50, x[::97].shape).astype(F)
    check(cuda_ctx, x, y, z, 1.0)


def test_nan_points_and_tiny_clouds(cuda_ctx):
    x, y, z = shuffled_scan(50_000, 34)
    x = x.copy()
    x[::101] = np.nan
    check(cuda_ctx, x, y, z, 0.2)
    for n in (1, 2, 3, 4097):
        xs, ys, zs = shuffled_scan(max(n, 2), 35)
        check(cuda_ctx, xs[:n], ys[:n], zs[:n], 0.3)


def test_mirror_follows_the_reference_dispatch(cuda_ctx):
    x, y, z = shuffled_scan(100_000, 36)
    cloud = sr.PointCloud(sr.StandardSchemas.point_xyz(), {"x": x, "y": y, "z": z})
    out = sr.VoxelGridDownsample(sr.VoxelGridDownsampleConfig.centroid(0.2)).filter(cloud)
    ref = oracle.voxel_centroid(x, y, z, leaf=0.2, plain_xyz=True)
    for name, r in zip("xyz", (ref.x, ref.y, ref.z)):
        assert np.array_equal(bits(out.field(name)), bits(r))
    # any other schema or aggregation takes the general key-ordered path
    inten = np.zeros_like(x)
    xyzi = sr.PointCloud(sr.StandardSchemas.point_xyzi(), {"x": x, "y": y, "z": z, "intensity": inten})
    out_i = sr.VoxelGridDownsample(sr.VoxelGridDownsampleConfig.centroid(0.2)).filter(xyzi)
    gen = oracle.voxel_centroid(x, y, z, [inten], leaf=0.2)
    assert np.array_equal(bits(out_i.field("x")), bits(gen.x))


def test_fused_voxel_normals_in_first_seen_order(cuda_ctx):
    x, y, z = shuffled_scan(250_000, 37)
    out = cuda_ctx.voxel_normals(x, y, z, (), leaf=0.1, radius=0.5, viewpoint=(0, 0, 100),
                                 want_keys=True, plain_xyz=True)
    ref = oracle.voxel_centroid(x, y, z, leaf=0.1, plain_xyz=True)
    assert np.array_equal(out["keys"], ref.keys) and np.array_equal(out["counts"], ref.counts)
    for g, r in zip(out["columns"], (ref.x, ref.y, ref.z)):
        assert np.array_equal(bits(g), bits(r))
    # the normals are those of the first-seen centroids, row for row
    nx, ny, nz, curv, cnt, _ = cuda_ctx.radius_normals(ref.x, ref.y, ref.z, 0.5,
                                                       viewpoint=(0, 0, 100))
    assert np.array_equal(out["neighbor_counts"], cnt)
    for g, r in ((out["nx"], nx), (out["ny"], ny), (out["nz"], nz), (out["curvature"], curv)):
        assert np.array_equal(np.isnan(g), np.isnan(r))
        assert np.array_equal(bits(g)[~np.isnan(g)], bits(r)[~np.isnan(r)])


def test_mode_is_refused_where_it_does_not_apply(cuda_ctx):
    x, y, z = shuffled_scan(1000, 38)
    with pytest.raises(sr.InvalidArgument, match="x, y, z only"):
        cuda_ctx.voxel_centroid(x, y, z, [x], leaf=0.2, plain_xyz=True)
    import ctypes
    import torch
    keep = _native._Keep()
    cloud = _native.make_cloud(*[torch.from_numpy(a).cuda() for a in (x, y, z)], (), keep)
    vp = _native._voxel_params(0.2, None, plain_xyz=True)
    np_ = _native._normal_params(0.5, 3, None, False)
    st = cuda_ctx._lib.srcu_voxel_normals_enqueue(cuda_ctx._h, ctypes.byref(cloud), ctypes.byref(vp),
                                                  ctypes.byref(np_))
    assert st == _native.SRCU_ERR_INVALID_ARGUMENT
    # the context is still good for the key-ordered path
    cols, _, _ = cuda_ctx.voxel_centroid(x, y, z, (), leaf=0.2)
    assert len(cols[0]) > 0
