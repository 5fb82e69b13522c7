"""CUDA radius normals vs the FP64 oracle and the reference restatement.

Bar: neighbour counts are exact (the f32 predicate is evaluated exactly as the
reference's KD-tree does, kdtree.rs:544-549); normals are within 1e-4 rad of
the FP64 oracle, sign-matched by viewpoint, for every point whose covariance
is not near-degenerate (relative eigengap >= GAP_MIN; those are counted and
reported, and their share is bounded); curvature within 1e-5 (normal_parity.py)."""
import numpy as np
import pytest

import normal_parity
import oracle
import spatialrust_b200 as sr
from spatialrust_b200 import synthetic

pytestmark = pytest.mark.gpu
F = np.float32
ANGLE_TOL = normal_parity.ANGLE_TOL
GAP_MIN = normal_parity.GAP_MIN
angle_errors = normal_parity.angle_errors


def check_normals(ctx, x, y, z, radius, min_neighbors=3, viewpoint=None, report=None,
                  include_self=False, ill_max=normal_parity.ILL_MAX):
    nx, ny, nz, curv, counts, stats = ctx.radius_normals(x, y, z, radius, min_neighbors, viewpoint,
                                                         include_self)
    ref = oracle.radius_normals_fp64(x, y, z, radius, min_neighbors, viewpoint,
                                     include_self=include_self)
    rep = normal_parity.check_against_fp64(nx, ny, nz, curv, counts, ref, x, y, z, viewpoint,
                                           stats, ill_max=ill_max, include_self=include_self)
    if report is not None:
        report.update(rep)
    return nx, ny, nz, curv, counts, stats


def grid(nx_, ny_, step, z=0.0):
    c = synthetic.unit_plane_grid(nx_, ny_, step, z)
    return c.x, c.y, c.z


# ---- the reference's known-answer tests ------------------------------------

def test_grid_planar_patch_vertical_normal():
    # normal_gpu.rs:127-152 (GpuNormalEstimator, radius 0.25, 12x12 grid step 0.1)
    x, y, z = grid(12, 12, 0.1)
    cloud = sr.PointCloud(sr.StandardSchemas.point_xyz(), {"x": x, "y": y, "z": z})
    est = sr.GpuNormalEstimator(sr.NormalEstimationConfig(search_radius=0.25, viewpoint=(0, 0, 10)))
    out = est.estimate(cloud)
    _, _, nz = out.normals3()
    assert np.all(nz > 0.99)
    assert np.all(out.field("curvature") < 1e-3)


def test_normals_grid_kernel_semantics():
    # normals_grid.rs:359-377: |nz| > 0.99, curvature < 1e-3 (no viewpoint)
    x, y, z = grid(12, 12, 0.1)
    cloud = sr.PointCloud(sr.StandardSchemas.point_xyz(), {"x": x, "y": y, "z": z})
    out = sr.GpuNormalEstimator(sr.NormalEstimationConfig(search_radius=0.25)).estimate(cloud)
    assert np.all(np.abs(out.field("normal_z")) > 0.99)
    assert np.all(out.field("curvature") < 1e-3)


def test_plane_normals_upward():
    # normal.rs:650-667 (radius covering the 8-neighbourhood)
    x, y, z = grid(5, 5, 1.0)
    cloud = sr.PointCloud(sr.StandardSchemas.point_xyz(), {"x": x, "y": y, "z": z})
    est = sr.NormalEstimator(sr.NormalEstimationConfig(search_radius=1.5, viewpoint=(0, 0, 10)))
    out, stats = est.estimate_with_diagnostics(cloud)
    assert stats.valid_count == 25 and stats.invalid_count == 0
    assert np.all(np.abs(out.field("normal_z") - 1.0) < 0.1)


def test_tilted_plane_normals():
    # normal.rs:669-686
    rows = []
    for i in range(7):
        for j in range(7):
            fx, fy = F(i) * F(0.2), F(j) * F(0.2)
            rows.append((fx, fy, F(0.2) * fx - F(0.3) * fy + F(0.1)))
    p = np.array(rows, np.float32)
    cloud = sr.PointCloud(sr.StandardSchemas.point_xyz(), {"x": p[:, 0], "y": p[:, 1], "z": p[:, 2]})
    out = sr.NormalEstimator(sr.NormalEstimationConfig(search_radius=0.45, viewpoint=(0, 0, 10))
                             ).estimate_with_policy(cloud, sr.GpuCuda)
    n = np.stack(out.normals3(), 1)
    expected = np.array([-0.2, 0.3, 1.0]) / np.linalg.norm([-0.2, 0.3, 1.0])
    assert np.all(n @ expected > 0.98)


def test_orientation_and_schema():
    x, y, z = grid(5, 5, 1.0)
    cloud = sr.PointCloud(sr.StandardSchemas.point_xyzi(),
                          {"x": x, "y": y, "z": z, "intensity": np.ones_like(x)})
    res = sr.NormalEstimator(sr.NormalEstimationConfig(search_radius=1.5, viewpoint=(0, 0, -10))
                             ).estimate_with_policy_and_receipt(cloud, sr.GpuCuda)
    out = res.output
    assert out.schema.names() == ["x", "y", "z", "intensity", "normal_x", "normal_y", "normal_z",
                                  "curvature"]
    assert np.all(out.field("normal_z") < -0.9)
    assert res.receipt.stages == ["normal-estimation", "gpu-readback"]


def test_min_neighbors_invalid_is_nan(cuda_ctx):
    x = np.array([0.0, 10.0, 20.0, 20.5], np.float32)
    nx, ny, nz, curv, counts, stats = cuda_ctx.radius_normals(x, np.zeros(4, F), np.zeros(4, F), 1.0)
    assert stats["invalid_count"] == 4 and np.all(np.isnan(nx)) and np.all(curv == 0)
    assert counts.tolist() == [0, 0, 1, 1]


def test_include_self_semantics(cuda_ctx):
    # normals_grid.rs: self included, fewer than 3 -> (0, 0, 1), curvature 0
    x = np.array([0.0, 10.0, 10.5], np.float32)
    nx, ny, nz, curv, counts, _ = cuda_ctx.radius_normals(x, np.zeros(3, F), np.zeros(3, F), 1.0,
                                                          include_self=True)
    assert nx.tolist() == [0, 0, 0] and nz.tolist() == [1, 1, 1] and curv.tolist() == [0, 0, 0]
    assert counts.tolist() == [1, 2, 2]
    # GpuNormalEstimator turns the fallback toward the viewpoint too (normal_gpu.rs:63-70)
    nx, ny, nz, curv, counts, _ = cuda_ctx.radius_normals(x, np.zeros(3, F), np.zeros(3, F), 1.0,
                                                          viewpoint=(0, 0, -5), include_self=True)
    assert nz.tolist() == [-1, -1, -1] and curv.tolist() == [0, 0, 0]


def test_include_self_georeferenced_scan(cuda_ctx):
    # the wgpu grid semantics on a 300k-point scan against the FP64 oracle's
    # include_self mode: counts = oracle counts (query included), the fallback
    # set and its (0, 0, +-1) exact, normals within 1e-4 rad
    # (r 0.6 on a sparse scan: ~9 points per neighbourhood, 36k fallbacks,
    # 642 ill-conditioned neighbourhoods of 3-5 nearly collinear points)
    c = synthetic.georef_scan(300_000, seed=9)
    rep = {}
    check_normals(cuda_ctx, c.x, c.y, c.z, 0.6, viewpoint=(0, 0, 100), include_self=True,
                  report=rep, ill_max=3.5e-3)
    assert 250_000 < rep["solved"] < c.n  # both branches exercised
    print("include_self scan:", rep)


def test_include_self_shapes_crop_no_viewpoint(cuda_ctx):
    c = synthetic.shapes_scene(5_000_000, seed=2)
    xyz = c.xyz()
    lo = xyz[7] - 8.0
    p = xyz[np.all((xyz >= lo) & (xyz < lo + 16), axis=1)]
    assert p.shape[0] > 20_000
    rep = {}
    check_normals(cuda_ctx, p[:, 0].copy(), p[:, 1].copy(), p[:, 2].copy(), 0.3,
                  include_self=True, report=rep)
    print("include_self shapes crop:", rep)


def test_zero_radius_counts_duplicates(cuda_ctx):
    # r = 0 is allowed (normal.rs:109): only exact duplicates are neighbours
    x = np.array([1.0, 1.0, 1.0, 2.0, 2.0, 3.0], np.float32)
    nx, ny, nz, curv, counts, _ = cuda_ctx.radius_normals(x, x, x, 0.0, min_neighbors=1)
    assert counts.tolist() == [2, 2, 2, 1, 1, 0]


# ---- parity vs the FP64 oracle ---------------------------------------------

def test_uniform_counts_and_normals(cuda_ctx):
    rng = np.random.default_rng(31)
    p = rng.random((30_000, 3), dtype=np.float32) * F(10)
    check_normals(cuda_ctx, p[:, 0], p[:, 1], p[:, 2], 0.6, viewpoint=(5, 5, 50))


def test_noisy_planes_no_viewpoint(cuda_ctx):
    rng = np.random.default_rng(32)
    n = 40_000
    uv = rng.uniform(-5, 5, (n, 2))
    z = 0.4 * uv[:, 0] - 0.1 * uv[:, 1] + rng.normal(0, 0.005, n)
    p = np.stack([uv[:, 0], uv[:, 1], z], 1).astype(np.float32)
    check_normals(cuda_ctx, p[:, 0], p[:, 1], p[:, 2], 0.15)


def test_shapes_scene_crop(cuda_ctx):
    # the 5M-point radius workload at full density, cropped to a 12 m cube
    c = synthetic.shapes_scene(5_000_000, seed=2)
    xyz = c.xyz()
    for centre in xyz[:3]:  # 12 m cubes around three random surface points
        lo = centre - 6.0
        m = np.all((xyz >= lo) & (xyz < lo + 12), axis=1)
        p = xyz[m]
        assert p.shape[0] > 5_000
        rep = {}
        check_normals(cuda_ctx, p[:, 0].copy(), p[:, 1].copy(), p[:, 2].copy(), 0.3,
                      viewpoint=(50, 50, 150), report=rep)
        print("shapes crop:", p.shape[0], rep)


def test_georeferenced_centroid_normals(cuda_ctx):
    c = synthetic.georef_scan(400_000, seed=1)
    vox = oracle.voxel_centroid(c.x, c.y, c.z, [c.intensity], leaf=0.5)
    rep = {}
    check_normals(cuda_ctx, vox.x, vox.y, vox.z, 0.5, viewpoint=(0, 0, 100), report=rep)
    print("georef centroids:", len(vox.x), rep)


def test_duplicates_and_shell_points(cuda_ctx):
    # exact duplicates are neighbours; points exactly on the shell are counted
    base = np.array([[0, 0, 0], [0.5, 0, 0], [0, 0.5, 0], [0, 0, 0.5], [0.25, 0.25, 0]], np.float32)
    p = np.concatenate([base, base[:2]], 0)
    nx, ny, nz, curv, counts, stats = cuda_ctx.radius_normals(p[:, 0], p[:, 1], p[:, 2], 0.5)
    ref = oracle.radius_normals_fp64(p[:, 0], p[:, 1], p[:, 2], 0.5)
    assert np.array_equal(counts, ref.counts)
    assert stats["shell_points"] == int(ref.shell.sum())


# ---- chained voxel -> normals (MvpPipeline) ----------------------------------

def test_voxel_then_normals_chain(cuda_ctx):
    c = synthetic.georef_scan(300_000, seed=5)
    out = cuda_ctx.voxel_normals(c.x, c.y, c.z, [c.intensity], leaf=0.1, radius=0.5,
                                 viewpoint=(0, 0, 100), want_keys=True)
    vox = oracle.voxel_centroid(c.x, c.y, c.z, [c.intensity], leaf=0.1)
    assert np.array_equal(out["keys"], vox.keys) and np.array_equal(out["counts"], vox.counts)
    for g, r in zip(out["columns"], vox.fields):
        assert np.max(np.abs(g - r)) <= 1e-6
    gx, gy, gz = out["columns"][:3]  # the normals stage's own input
    ref = oracle.radius_normals_fp64(gx, gy, gz, 0.5, 3, (0, 0, 100))
    normal_parity.check_against_fp64(out["nx"], out["ny"], out["nz"], out["curvature"],
                                     out["neighbor_counts"], ref, gx, gy, gz, (0, 0, 100),
                                     out["stats"], label="chain")


def test_device_enqueue_matches_sync_path(cuda_ctx):
    import torch
    from spatialrust_b200 import _native
    c = synthetic.georef_scan(200_000, seed=6)
    sync = cuda_ctx.voxel_normals(c.x, c.y, c.z, [c.intensity], leaf=0.2, radius=0.6,
                                  viewpoint=(0, 0, 100))
    dev = [torch.from_numpy(a).cuda() for a in (c.x, c.y, c.z, c.intensity)]
    keep = _native._Keep()
    cloud = _native.make_cloud(dev[0], dev[1], dev[2], [dev[3]], keep)
    for _ in range(3):  # repeated enqueues reuse the buffers
        cuda_ctx.voxel_normals_enqueue(cloud, 0.2, None, 0.6, 3, (0, 0, 100))
    v, stats = cuda_ctx.frame_check()
    assert v == len(sync["counts"])
    got = cuda_ctx.frame_fetch(c.n, n_attrs=1)
    for a, b in zip(got["columns"], sync["columns"]):
        assert np.array_equal(a, b)
    for k in ("nx", "ny", "nz"):
        assert np.array_equal(got[k], sync[k], equal_nan=True)
    assert np.array_equal(got["curvature"], sync["curvature"])
    assert np.array_equal(got["neighbor_counts"], sync["neighbor_counts"])
    assert got["stats"] == sync["stats"] == stats


def test_column_hash_path_on_huge_extent(cuda_ctx):
    # 100 km across at r = 0.5: the dense column table would need ~4e10
    # slots, so the chain uses the column hash; counts must still be exact
    rng = np.random.default_rng(12)
    blobs = rng.uniform(0, 100_000, (40, 2))
    pts = []
    for cx, cy in blobs:
        p = rng.normal(0, 0.4, (250, 3))
        p[:, 0] += cx
        p[:, 1] += cy
        pts.append(p)
    p = np.concatenate(pts).astype(np.float32)
    x, y, z = (np.ascontiguousarray(p[:, k]) for k in range(3))
    nx, ny, nz, curv, counts, stats = cuda_ctx.radius_normals(x, y, z, 0.5, 3)
    ref = oracle.brute_radius_counts(x, y, z, 0.5)
    assert np.array_equal(counts, ref)
    assert stats["valid_count"] + stats["invalid_count"] == len(x)
