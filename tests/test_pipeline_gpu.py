"""MvpPipeline (voxel -> normals -> RANSAC plane -> clusters) through the CUDA
arms, against the reference's pipeline test and stage by stage against the
oracle (crates/spatialrust-pipeline/src/mvp.rs:173-284)."""
import numpy as np
import pytest

import oracle
import spatialrust_b200 as sr
from spatialrust_b200 import synthetic

pytestmark = pytest.mark.gpu
F = np.float32


def sample_cloud():
    # mvp.rs:316-327: a 10 x 10 grid (step 0.1) at z = 0 and two points at z = 0.5
    b = sr.PointCloudBuilder.xyz()
    for x in range(10):
        for y in range(10):
            b.push_point([x * 0.1, y * 0.1, 0.0])
    b.push_point([0.0, 0.0, 0.5])
    b.push_point([0.1, 0.0, 0.5])
    return b.build()


def test_reference_pipeline_runs_every_stage():
    # mvp.rs:329-370 (without its CPU-only receipt assertions)
    cfg = sr.MvpPipelineConfig(
        voxel=sr.VoxelGridDownsampleConfig.centroid(0.2),
        normals=sr.NormalEstimationConfig(k_neighbors=8, min_neighbors=3, viewpoint=(0, 0, 10)),
        plane=sr.RansacPlaneConfig(distance_threshold=0.05, max_iterations=500, min_inliers=10,
                                   seed=17),
        cluster=sr.EuclideanClusterConfig(cluster_tolerance=0.3, min_cluster_size=1))
    res = sr.MvpPipeline(cfg).run(sample_cloud())
    assert not res.downsampled.is_empty()
    assert "normal_x" in res.with_normals.columns
    assert res.plane.inlier_count >= 10
    assert res.clusters.cluster_count >= 1
    assert "label" in res.output.columns
    assert res.registration is None
    assert res.receipt.plane.stages[0] == "plane-segmentation"
    assert res.receipt.clusters.stages[0] == "euclidean-clustering"
    assert res.receipt.host_to_device_bytes() > 0


def test_icp_step_is_refused():
    with pytest.raises(sr.InvalidArgument):
        sr.MvpPipeline(sr.MvpPipelineConfig(icp=object())).run(sample_cloud())


def test_stages_match_the_oracle_on_a_scan():
    c = synthetic.georef_scan(120_000, seed=70)
    cloud = sr.PointCloud(sr.StandardSchemas.point_xyzi(),
                          {"x": c.x, "y": c.y, "z": c.z, "intensity": c.intensity})
    cfg = sr.MvpPipelineConfig(
        voxel=sr.VoxelGridDownsampleConfig.centroid(0.2),
        normals=sr.NormalEstimationConfig(viewpoint=(0, 0, 100)),
        plane=sr.RansacPlaneConfig(distance_threshold=0.05, max_iterations=200, seed=5),
        cluster=sr.EuclideanClusterConfig(cluster_tolerance=0.5, min_cluster_size=3))
    res = sr.MvpPipeline(cfg).run(cloud)
    # the fused voxel -> normals call gives what the two stages give one after the other
    two = sr.NormalEstimator(sr.NormalEstimationConfig.radius(0.4, viewpoint=(0, 0, 100))) \
        .estimate(sr.VoxelGridDownsample(cfg.voxel).filter(cloud))
    assert res.with_normals == two
    v = oracle.voxel_centroid(c.x, c.y, c.z, [c.intensity], leaf=0.2)
    assert np.array_equal(res.downsampled.field("x"), v.x)
    assert np.array_equal(res.downsampled.field("intensity"), v.fields[3])
    ref = oracle.ransac_plane(v.x, v.y, v.z, 0.05, 200, 3, 5)
    assert res.plane.inlier_count == ref["inlier_count"]
    assert np.array_equal(res.plane.outliers.field("x"), v.x[~ref["mask"]])
    ox, oy, oz = (v.x[~ref["mask"]], v.y[~ref["mask"]], v.z[~ref["mask"]])
    roots = oracle.euclidean_roots(ox, oy, oz, 0.5, sparse=True)
    sizes = np.bincount(np.unique(roots, return_inverse=True)[1])
    assert res.clusters.cluster_count == int((sizes >= 3).sum())


def _voxel_normals_into(ctx, cloud, vcols, ncols, counts, ncounts):
    """srcu_voxel_normals into caller buffers (numpy or pinned torch tensors)."""
    import ctypes
    from spatialrust_b200 import _native
    keep = _native._Keep()
    addr = _native._addr
    attr_out = keep.add((ctypes.c_void_p * 1)(addr(vcols[3])))
    vout = _native.SrcuVoxelOut(addr(vcols[0]), addr(vcols[1]), addr(vcols[2]),
                                ctypes.cast(attr_out, ctypes.c_void_p), 0, addr(counts), 0)
    nout = _native.SrcuNormalOut(*[addr(c) for c in ncols], addr(ncounts), 0)
    vp = _native._voxel_params(0.1, None)
    np_ = _native._normal_params(0.5, 3, (0.0, 0.0, 100.0), False)
    nv = ctypes.c_uint64(0)
    stats = _native.SrcuNormalStats()
    ctx._check(ctx._lib.srcu_voxel_normals(ctx.handle, ctypes.byref(cloud), ctypes.byref(vp),
                                           ctypes.byref(np_), ctypes.byref(vout),
                                           ctypes.byref(nout), ctypes.byref(nv), ctypes.byref(stats)))
    return int(nv.value)


def test_pageable_host_buffers_match_pinned(cuda_ctx):
    # Pageable host columns (numpy) are staged through the context's pinned ring
    # in 4 MB chunks (3.2M points: 12.8 MB per column, four chunks) in both
    # directions; every output must be bit-identical to pinned host buffers'.
    import torch
    from spatialrust_b200 import _native
    c = synthetic.georef_scan(3_200_000, seed=61)
    n = c.n
    out = {}
    for kind in ("pageable", "pinned"):
        keep = _native._Keep()
        if kind == "pinned":
            cols = [torch.from_numpy(a.copy()).pin_memory() for a in (c.x, c.y, c.z, c.intensity)]
            mk = lambda dt: torch.empty(n, dtype=dt).pin_memory()
        else:
            cols = [a.copy() for a in (c.x, c.y, c.z, c.intensity)]
            mk = lambda dt: np.empty(n, {torch.float32: np.float32, torch.int32: np.uint32}[dt])
        cloud = _native.make_cloud(cols[0], cols[1], cols[2], [cols[3]], keep)
        vcols = [mk(torch.float32) for _ in range(4)]
        ncols = [mk(torch.float32) for _ in range(4)]
        counts, ncounts = mk(torch.int32), mk(torch.int32)
        v = _voxel_normals_into(cuda_ctx, cloud, vcols, ncols, counts, ncounts)
        out[kind] = [np.asarray(a)[:v].view(np.uint32).copy() for a in vcols + ncols + [counts, ncounts]]
    assert len(out["pageable"][0]) > 2_000_000
    for a, b in zip(out["pageable"], out["pinned"]):
        assert np.array_equal(a, b)
