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
