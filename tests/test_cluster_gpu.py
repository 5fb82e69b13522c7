"""Euclidean cluster roots on the GPU (srcu_euclidean_cluster_roots) vs the
reference's grid union-find restated in the oracle.

Bar: bit-exact roots.  The answer is unique -- every point's root is the
smallest index of its component under the f32 predicate -- so any correct
union order gives the same array."""
import numpy as np
import pytest

import oracle
import spatialrust_b200 as sr
from spatialrust_b200 import synthetic

pytestmark = pytest.mark.gpu
F = np.float32


def three_clusters():
    b = sr.PointCloudBuilder(sr.StandardSchemas.point_xyz())
    for cx, cy in ((0.0, 0.0), (10.0, 0.0), (0.0, 10.0)):
        for dx in range(3):
            for dy in range(3):
                b.push_point([cx + dx, cy + dy, 0.0])
    return b.build()


def test_gpu_finds_three_separated_clusters():
    # cluster_gpu.rs:90-101
    cfg = sr.EuclideanClusterConfig(cluster_tolerance=1.5, min_cluster_size=3)
    res = sr.GpuEuclideanClusterExtractor(cfg).extract(three_clusters())
    assert res.cluster_count == 3 and res.cluster_sizes == [9, 9, 9]
    assert res.cloud.field("label").tolist() == [0] * 9 + [1] * 9 + [2] * 9


def test_policy_arm_and_minimum_size():
    # cluster.rs:385-400: two points, min size 3 -> no cluster; Gpu(Cuda) now runs
    b = sr.PointCloudBuilder(sr.StandardSchemas.point_xyz())
    b.push_point([0.0, 0.0, 0.0])
    b.push_point([0.1, 0.0, 0.0])
    cfg = sr.EuclideanClusterConfig(cluster_tolerance=0.5, min_cluster_size=3)
    out = sr.EuclideanClusterExtractor(cfg).extract_with_policy_and_receipt(b.build(), sr.GpuCuda)
    assert out.output.cluster_count == 0
    assert out.output.cloud.field("label").tolist() == [-1, -1]
    assert "euclidean-clustering" in out.receipt.stages


def test_long_chain_is_one_component(cuda_ctx):
    # uniform_grid.rs:564-576 and cluster_gpu.rs:113-128
    x = np.arange(300, dtype=F)
    zero = np.zeros(300, F)
    assert np.all(cuda_ctx.euclidean_cluster_roots(x, zero, zero, 1.5) == 0)


@pytest.mark.parametrize("tol", [0.05, 0.2, 0.6])
def test_roots_bit_exact_on_scan(cuda_ctx, tol):
    c = synthetic.georef_scan(150_000, seed=41)
    got = cuda_ctx.euclidean_cluster_roots(c.x, c.y, c.z, tol)
    # 200 m at these tolerances exceeds the dense grid's cell cap: the sparse-cell path
    ref = oracle.euclidean_roots(c.x, c.y, c.z, tol, sparse=True)
    assert np.array_equal(got, ref), f"{np.count_nonzero(got != ref)} roots differ"


def test_roots_bit_exact_on_shapes_and_lattice(cuda_ctx):
    c = synthetic.shapes_scene(120_000, seed=8)
    assert np.array_equal(cuda_ctx.euclidean_cluster_roots(c.x, c.y, c.z, 0.1),
                          oracle.euclidean_roots(c.x, c.y, c.z, 0.1, sparse=True))
    # a lattice at exactly the tolerance: every edge is on the shell
    g = synthetic.unit_plane_grid(60, 60, 0.25)
    assert np.array_equal(cuda_ctx.euclidean_cluster_roots(g.x, g.y, g.z, 0.25),
                          oracle.euclidean_roots(g.x, g.y, g.z, 0.25))


def test_giant_component_under_contention(cuda_ctx):
    # ~13 neighbours per point: one component spans most of the cube, so many
    # lanes hook into the same roots at once
    c = synthetic.uniform_cube(200_000, seed=3, extent=20.0)
    got = cuda_ctx.euclidean_cluster_roots(c.x, c.y, c.z, 0.5)
    ref = oracle.euclidean_roots(c.x, c.y, c.z, 0.5)
    assert np.array_equal(got, ref)
    assert np.bincount(ref).max() > 100_000


def test_non_finite_points_are_singletons(cuda_ctx):
    rng = np.random.default_rng(2)
    p = (rng.random((5000, 3)) * 5).astype(F)
    p[[3, 100, 2500], 0] = np.nan
    p[[7, 4000], 2] = np.inf
    got = cuda_ctx.euclidean_cluster_roots(p[:, 0], p[:, 1], p[:, 2], 0.3)
    ref = oracle.euclidean_roots(p[:, 0], p[:, 1], p[:, 2], 0.3)
    assert np.array_equal(got, ref)
    for i in (3, 100, 2500, 7, 4000):
        assert got[i] == i


def test_device_inputs_and_repeated_calls(cuda_ctx):
    import torch
    c = synthetic.georef_scan(60_000, seed=5)
    ref = oracle.euclidean_roots(c.x, c.y, c.z, 0.3, sparse=True)
    dev = [torch.from_numpy(a).cuda() for a in (c.x, c.y, c.z)]
    for _ in range(2):
        got = cuda_ctx.euclidean_cluster_roots(*dev, 0.3)
        assert np.array_equal(got.cpu().numpy().view(np.uint32), ref)
    small = synthetic.uniform_cube(1000, seed=1, extent=3.0)
    assert np.array_equal(cuda_ctx.euclidean_cluster_roots(small.x, small.y, small.z, 0.2),
                          oracle.euclidean_roots(small.x, small.y, small.z, 0.2))


def test_argument_errors(cuda_ctx):
    x = np.zeros(4, F)
    for bad in (0.0, -1.0, float("nan"), float("inf")):
        with pytest.raises(sr.InvalidArgument):
            cuda_ctx.euclidean_cluster_roots(x, x, x, bad)
    assert len(cuda_ctx.euclidean_cluster_roots(x[:0], x[:0], x[:0], 1.0)) == 0


def test_column_hash_path_on_huge_extent(cuda_ctx):
    # blobs 100 km apart: too many columns for the dense table (column hash)
    rng = np.random.default_rng(13)
    centres = rng.uniform(0, 100_000, (50, 3))
    p = np.concatenate([c + rng.normal(0, 0.3, (200, 3)) for c in centres]).astype(F)
    x, y, z = (np.ascontiguousarray(p[:, k]) for k in range(3))
    assert np.array_equal(cuda_ctx.euclidean_cluster_roots(x, y, z, 0.25),
                          oracle.euclidean_roots(x, y, z, 0.25, sparse=True))
