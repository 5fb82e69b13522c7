"""Interleaved (AoSoA) input records, srcu_cloud.stride > 1: the reference's
AoSoA chunk layouts (tensor_aoso.rs:10-66) give exactly the results of the same
points as packed columns, from host and from device memory."""
import numpy as np
import pytest

from spatialrust_b200 import _native, synthetic

pytestmark = pytest.mark.gpu


def records(c, extra=()):
    return np.ascontiguousarray(np.stack([c.x, c.y, c.z, c.intensity, *extra], axis=1))


def test_voxel_centroid_from_xyzi_records(cuda_ctx):
    c = synthetic.georef_scan(80_000, seed=61)
    rec = records(c)  # [x, y, z, intensity], stride 4
    keep = _native._Keep()
    cloud = _native.make_interleaved_cloud(rec, (0, 1, 2), (3,), keep)
    got = cuda_ctx.voxel_centroid(cloud, None, None, want_keys=True, leaf=0.1)
    ref = cuda_ctx.voxel_centroid(c.x, c.y, c.z, [c.intensity], want_keys=True, leaf=0.1)
    for g, r in zip(got[0], ref[0]):
        assert np.array_equal(g, r)
    assert np.array_equal(got[1], ref[1]) and np.array_equal(got[2], ref[2])


def test_voxel_normals_from_device_xyzinormal_records(cuda_ctx):
    import torch
    c = synthetic.georef_scan(60_000, seed=62)
    rng = np.random.default_rng(1)
    nrm = [rng.random(c.n, dtype=np.float32) for _ in range(3)]
    rec = torch.from_numpy(records(c, nrm)).cuda()  # stride 7
    keep = _native._Keep()
    cloud = _native.make_interleaved_cloud(rec, (0, 1, 2), (3, 4, 5, 6), keep)
    got = cuda_ctx.voxel_normals(cloud, None, None, leaf=0.1, radius=0.5)
    ref = cuda_ctx.voxel_normals(c.x, c.y, c.z, [c.intensity, *nrm], leaf=0.1, radius=0.5)
    for g, r in zip(got["columns"], ref["columns"]):
        assert np.array_equal(g, r)
    for k in ("nx", "ny", "nz", "curvature", "neighbor_counts"):
        assert np.array_equal(got[k], ref[k], equal_nan=True)


def test_radius_normals_and_clusters_from_xyz_records(cuda_ctx):
    import torch
    c = synthetic.shapes_scene(50_000, seed=3)
    rec = np.ascontiguousarray(np.stack([c.x, c.y, c.z], axis=1))  # stride 3
    keep = _native._Keep()
    got = cuda_ctx.radius_normals(_native.make_interleaved_cloud(rec, keep=keep), None, None, 0.3)
    ref = cuda_ctx.radius_normals(c.x, c.y, c.z, 0.3)
    for g, r in zip(got[:5], ref[:5]):
        assert np.array_equal(g, r, equal_nan=True)
    dev = torch.from_numpy(np.ascontiguousarray(np.stack([c.x, c.y, c.z, c.x, c.y, c.z], 1))).cuda()
    roots = cuda_ctx.euclidean_cluster_roots(_native.make_interleaved_cloud(dev, keep=keep),
                                             None, None, 0.1)
    assert np.array_equal(roots.cpu().numpy().view(np.uint32),
                          cuda_ctx.euclidean_cluster_roots(c.x, c.y, c.z, 0.1))


def test_host_columns_must_share_one_record_array(cuda_ctx):
    c = synthetic.uniform_cube(1000, seed=2)
    keep = _native._Keep()
    cloud = _native.make_cloud(c.x, c.y, c.z, [], keep)
    cloud.stride = 4  # separate arrays cannot be records of one block
    with pytest.raises(_native.InvalidArgument):
        cuda_ctx.voxel_centroid(cloud, None, None, leaf=1.0)


def test_server_accepts_records():
    c = synthetic.lidar_frame(seed=3, beams=16, azimuths=512)
    rec = records(c)
    srv = _native.Server(0, hbm_budget_bytes=2 << 30, frame_slots=1, bulk_slots=1,
                         frame_batch_points=20_000, bulk_threshold_points=10_000,
                         bulk_max_points=20_000, host_arena_bytes=64 << 20)
    lib = _native.load()
    import ctypes
    keep = _native._Keep()
    cloud = _native.make_interleaved_cloud(rec, (0, 1, 2), (3,), keep)
    vp = _native._voxel_params(0.2, None)
    np_ = _native._normal_params(0.6, 3, None, False)
    assert lib.srcu_server_submit(srv._h, 1, ctypes.byref(cloud), ctypes.byref(vp),
                                  ctypes.byref(np_)) == 0
    assert srv.submit(2, c.x, c.y, c.z, c.intensity, leaf=0.2, radius=0.6)
    got = {}
    while len(got) < 2:
        r = srv.poll(wait_us=100_000)
        if r is not None:
            got[r["req_id"]] = r
    for k in ("x", "y", "z", "intensity", "nx", "ny", "nz", "curvature", "counts"):
        assert np.array_equal(got[1][k], got[2][k], equal_nan=True)
    srv.close()
