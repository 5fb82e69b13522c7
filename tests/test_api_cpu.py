"""Host-side logic of the reference-API mirror that runs without a GPU:
policy resolution, validation order, dtype narrowing, schema handling, and the
synthetic workload generators."""
import numpy as np
import pytest

import spatialrust_b200 as sr
from spatialrust_b200 import synthetic
from spatialrust_b200.filtering import narrow, resolve_cuda_policy


def xyz_cloud(pts):
    b = sr.PointCloudBuilder(sr.StandardSchemas.point_xyz())
    for p in pts:
        b.push_point(p)
    return b.build()


def test_policy_resolution():
    assert resolve_cuda_policy(sr.GpuCuda, "x") == sr.GpuCuda
    assert resolve_cuda_policy(sr.Auto, "x") == sr.GpuCuda
    with pytest.raises(sr.InvalidArgument):
        resolve_cuda_policy(sr.ExecutionPolicy.gpu(sr.DeviceKind.Cpu), "x")
    with pytest.raises(sr.InvalidArgument):
        resolve_cuda_policy(sr.ExecutionPolicy.gpu(sr.DeviceKind.Wgpu), "x")
    with pytest.raises(sr.InvalidArgument):
        resolve_cuda_policy(sr.CpuSingle, "x")
    with pytest.raises(sr.InvalidArgument):
        resolve_cuda_policy(sr.CpuParallel, "x")


def test_voxel_validation_before_device():
    cloud = xyz_cloud([[0.0, 0.0, 0.0]])
    f = sr.VoxelGridDownsample(sr.VoxelGridDownsampleConfig.centroid(0.0))
    with pytest.raises(sr.InvalidArgument):  # voxel.rs:1357-1364
        f.filter_with_policy(cloud, sr.GpuCuda)
    empty = xyz_cloud([])
    out = sr.VoxelGridDownsample(sr.VoxelGridDownsampleConfig.centroid(1.0)).filter_with_policy(
        empty, sr.GpuCuda)
    assert len(out) == 0 and out.schema == empty.schema
    # ApproximateFirst has a CUDA arm too; empty input returns before the device
    approx = sr.VoxelGridDownsample(sr.VoxelGridDownsampleConfig.approximate(1.0))
    assert len(approx.filter_with_policy(empty, sr.GpuCuda)) == 0


def test_normals_validation_before_device():
    cloud = xyz_cloud([[0.0, 0.0, 0.0]])
    est = sr.NormalEstimator(sr.NormalEstimationConfig(search_radius=-1.0))
    with pytest.raises(sr.InvalidArgument):  # normal.rs:109-111
        est.estimate_with_policy(cloud, sr.GpuCuda)
    knn = sr.NormalEstimator(sr.NormalEstimationConfig())
    with pytest.raises(sr.InvalidArgument):
        knn.estimate_with_policy(cloud, sr.GpuCuda)
    # normal.rs:705-712 rejected Gpu(Cuda) before this arm existed; an unknown
    # device kind is still rejected
    with pytest.raises(sr.InvalidArgument):
        knn.estimate_with_policy(cloud, sr.ExecutionPolicy.gpu(sr.DeviceKind.Wgpu))
    empty = xyz_cloud([])
    out, res = sr.NormalEstimator(sr.NormalEstimationConfig.radius(0.5)).estimate_with_diagnostics(empty)
    assert len(out) == 0 and res.valid_count == 0


def test_narrow_rounds_half_away_and_saturates():
    # push_field (voxel.rs:1241-1259): value.round() as u8 / i32 with Rust's
    # half-away-from-zero rounding and saturating casts
    v = np.array([0.5, 1.5, 2.5, 254.6, 300.0, -3.0, np.nan, 0.49999997], np.float32)
    assert narrow(v, sr.DType.U8).tolist() == [1, 2, 3, 255, 255, 0, 0, 0]
    assert narrow(np.array([-2.5, 2.5], np.float32), sr.DType.I32).tolist() == [-3, 3]
    assert narrow(v[:2], sr.DType.F64).dtype == np.float64


def test_build_output_cloud_appends_fields_once():
    cloud = sr.PointCloud(sr.StandardSchemas.point_xyzinormal(),
                          {k: np.zeros(2, np.float32) for k in
                           ["x", "y", "z", "intensity", "normal_x", "normal_y", "normal_z"]})
    out = sr.build_output_cloud(cloud, np.ones(2), np.ones(2), np.ones(2), np.zeros(2))
    assert out.schema.names() == ["x", "y", "z", "intensity", "normal_x", "normal_y", "normal_z",
                                  "curvature"]
    assert out.field("normal_x").tolist() == [1.0, 1.0]


def test_synthetic_generators_are_deterministic():
    a = synthetic.uniform_cube(1000, seed=0)
    b = synthetic.uniform_cube(1000, seed=0)
    assert np.array_equal(a.x, b.x) and np.array_equal(a.intensity, b.intensity)
    assert a.x.dtype == np.float32 and a.x.min() >= 0 and a.x.max() < 100
    g = synthetic.georef_scan(20_000, seed=1)
    assert g.x.dtype == np.float32 and np.allclose(g.origin, synthetic.GEO_OFFSET)
    assert -5 < g.x.min() and g.x.max() < 205  # boxes may overhang the square by half a side
    assert 0 < g.intensity.min() and g.intensity.max() < 1
    s = synthetic.shapes_scene(20_000, seed=2)
    assert s.n == 20_000 and np.all(np.abs(s.xyz()) < 100.5)
    clouds, leaves, radii = synthetic.batched_uneven(8, seed=3, scale=0.01)
    assert len(clouds) == 8 and set(np.unique(leaves)).issubset({np.float32(0.05), np.float32(0.1),
                                                                 np.float32(0.2)})
    assert np.allclose(radii, leaves * 5)


def test_c0_occupancy_matches_expectation(oracle_lib):
    c = synthetic.uniform_cube(100_000, seed=0)
    r = oracle_lib.voxel_centroid(c.x, c.y, c.z, [c.intensity], leaf=4.0)
    # 25^3 voxels, 6.4 points each on average: ~15.6k occupied
    assert 15_500 < len(r.x) <= 15_625
    assert int(r.counts.sum()) == 100_000


def test_plain_xyz_dispatch_follows_the_reference():
    from spatialrust_b200 import _native
    from spatialrust_b200.filtering import uses_plain_xyz_path
    cfg = sr.VoxelGridDownsampleConfig.centroid(0.5)
    assert uses_plain_xyz_path(sr.StandardSchemas.point_xyz(), cfg)
    assert not uses_plain_xyz_path(sr.StandardSchemas.point_xyzi(), cfg)
    assert not uses_plain_xyz_path(sr.StandardSchemas.point_xyz(),
                                   sr.VoxelGridDownsampleConfig.approximate(0.5))
    assert _native._voxel_params(0.5, None, plain_xyz=True).mode == _native.SRCU_VOXEL_CENTROID_XYZ
    assert _native._voxel_params(0.5, None).mode == _native.SRCU_VOXEL_CENTROID
