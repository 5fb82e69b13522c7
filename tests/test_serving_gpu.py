"""The serving loop (srcu_server_*): requests of mixed sizes submitted together,
packed into batched chains and bulk slots, give exactly the results each
request gives alone (a single-cloud srcu_voxel_normals call) -- centroids,
counts, normals and curvature bit-identical -- and admission control answers
BUSY instead of queueing past its limits."""
import time

import numpy as np
import pytest

from spatialrust_b200 import _native, synthetic

pytestmark = pytest.mark.gpu

LEAF, RADIUS = 0.2, 0.6


def small_frames(k, seed0=0):
    scene = synthetic.lidar_scene(seed=4, n_boxes=100)
    return [synthetic.lidar_frame(seed=seed0 + i, scene=scene, beams=16, azimuths=512)
            for i in range(k)]


def drain(srv, count, timeout_s=60.0):
    out = {}
    t_end = time.time() + timeout_s
    while len(out) < count and time.time() < t_end:
        r = srv.poll(wait_us=10_000)
        if r is not None:
            out[r["req_id"]] = r
    assert len(out) == count, f"only {len(out)} of {count} requests finished"
    return out


def check_same_as_alone(ctx, cloud, r, leaf=LEAF, radius=RADIUS, viewpoint=None):
    ref = ctx.voxel_normals(cloud.x, cloud.y, cloud.z, [cloud.intensity], leaf=leaf, radius=radius,
                            viewpoint=viewpoint)
    assert r["status"] == 0
    assert r["voxels"] == len(ref["counts"])
    assert np.array_equal(r["counts"], ref["counts"])
    for k, col in zip(("x", "y", "z", "intensity"), ref["columns"]):
        assert np.array_equal(r[k], col), k
    for k in ("nx", "ny", "nz", "curvature"):
        assert np.array_equal(r[k], ref[k], equal_nan=True), k


def test_mixed_requests_equal_alone():
    frames = small_frames(24)
    full = synthetic.lidar_frame(seed=99)  # one full 64 x 2048 frame
    chunk = synthetic.map_chunk(300_000, seed=7)  # above the bulk threshold below
    srv = _native.Server(0, hbm_budget_bytes=8 << 30, frame_slots=2, bulk_slots=1,
                         frame_batch_points=200_000, bulk_threshold_points=150_000,
                         bulk_max_points=400_000, host_arena_bytes=256 << 20)
    reqs = frames[:12] + [chunk, full] + frames[12:]
    for i, c in enumerate(reqs):
        assert srv.submit(i, c.x, c.y, c.z, c.intensity, leaf=LEAF, radius=RADIUS)
    got = drain(srv, len(reqs))
    st = srv.stats()
    assert st["completed"] == len(reqs) and st["failed"] == 0
    assert st["batches"] < len(reqs), "no two requests shared a chain"
    # each request alone through the server, then alone through a context
    ctx = _native.Context(0)
    for i, c in enumerate(reqs):
        check_same_as_alone(ctx, c, got[i])
    for i in (0, 12, 13):
        assert srv.submit(1000 + i, reqs[i].x, reqs[i].y, reqs[i].z, reqs[i].intensity, leaf=LEAF,
                          radius=RADIUS)
        alone = drain(srv, 1)[1000 + i]
        for k in ("x", "y", "z", "nx", "ny", "nz", "curvature", "counts"):
            assert np.array_equal(alone[k], got[i][k], equal_nan=True), k
    ctx.close()
    srv.close()


def test_per_request_parameters_and_empty():
    frames = small_frames(3, seed0=40)
    srv = _native.Server(0, hbm_budget_bytes=4 << 30, frame_slots=1, bulk_slots=1,
                         frame_batch_points=200_000, bulk_threshold_points=150_000,
                         bulk_max_points=200_000, host_arena_bytes=128 << 20)
    params = [(0.1, 0.5, (0.0, 0.0, 10.0)), (0.3, 1.0, None), (0.2, 0.6, (5.0, 5.0, 5.0))]
    for i, (c, (leaf, r, vp)) in enumerate(zip(frames, params)):
        assert srv.submit(i, c.x, c.y, c.z, c.intensity, leaf=leaf, radius=r, viewpoint=vp)
    empty = np.zeros(0, np.float32)
    assert srv.submit(99, empty, empty, empty, empty, leaf=0.2, radius=0.6)
    got = drain(srv, 4)
    assert got[99]["voxels"] == 0 and got[99]["status"] == 0
    ctx = _native.Context(0)
    for i, (c, (leaf, r, vp)) in enumerate(zip(frames, params)):
        check_same_as_alone(ctx, c, got[i], leaf=leaf, radius=r, viewpoint=vp)
    ctx.close()
    srv.close()


def test_admission_and_argument_errors():
    frames = small_frames(1)
    c = frames[0]
    srv = _native.Server(0, hbm_budget_bytes=2 << 30, frame_slots=1, bulk_slots=1,
                         frame_batch_points=20_000, bulk_threshold_points=10_000,
                         bulk_max_points=20_000, max_pending_points=9_000,
                         host_arena_bytes=64 << 20)
    with pytest.raises(_native.InvalidArgument):  # leaf must be > 0
        srv.submit(1, c.x, c.y, c.z, c.intensity, leaf=0.0, radius=RADIUS)
    with pytest.raises(_native.InvalidArgument):  # larger than bulk_max_points
        big = synthetic.uniform_cube(30_000, seed=1)
        srv.submit(2, big.x, big.y, big.z, big.intensity, leaf=LEAF, radius=RADIUS)
    # 8192-point requests against a 9000-point queue: the queue holds one at a time
    accepted = 0
    busy = 0
    for i in range(20):
        if srv.submit(10 + i, c.x, c.y, c.z, c.intensity, leaf=LEAF, radius=RADIUS):
            accepted += 1
        else:
            busy += 1
    drain(srv, accepted)
    assert accepted >= 1
    assert srv.stats()["rejected"] == busy
    with pytest.raises(_native.InvalidArgument):  # an id still held is refused
        assert srv.submit(500, c.x, c.y, c.z, c.intensity, leaf=LEAF, radius=RADIUS)
        srv.submit(500, c.x, c.y, c.z, c.intensity, leaf=LEAF, radius=RADIUS)
    drain(srv, 1)
    srv.close()
    with pytest.raises(_native.OutOfBudget):  # slots larger than the HBM budget
        _native.Server(0, hbm_budget_bytes=1 << 20)
