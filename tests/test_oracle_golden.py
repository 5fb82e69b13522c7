"""Pins the CPU oracle (oracle/srcu_oracle.c) to the reference's own
known-answer tests for this path.  The reference is Rust and cannot be built
here, so these golden values are transcribed from its unit tests (file:line
cited per test) and the oracle must reproduce them exactly as stated there."""
import math

import numpy as np
import pytest

import oracle


@pytest.fixture(scope="module", autouse=True)
def _built():
    oracle.build()


F = np.float32


def test_centroid_downsample_reduces_points():
    # crates/spatialrust-filtering/src/voxel.rs:1270-1288 (point_xyz, leaf 0.5)
    r = oracle.voxel_centroid([0.0, 0.1, 1.0, 1.1], [0] * 4, [0] * 4, leaf=0.5, plain_xyz=True)
    assert len(r.x) == 2
    assert abs(r.x[0] - 0.05) < 1e-5
    assert abs(r.x[1] - 1.05) < 1e-5


def test_explicit_origin_uses_floor_for_negative_voxels():
    # voxel.rs:1290-1306
    r = oracle.voxel_centroid([-0.6, -0.1, 0.1], [0] * 3, [0] * 3, leaf=1.0, origin=(0, 0, 0),
                              plain_xyz=True)
    assert len(r.x) == 2
    assert abs(r.x[0] - -0.35) < 1e-5
    assert abs(r.x[1] - 0.1) < 1e-5
    assert r.keys.tolist() == [[-1, 0, 0], [0, 0, 0]]


def test_default_origin_matches_explicit_min_origin():
    # voxel.rs:1308-1327: default origin output == explicit min-corner origin output
    pts = np.array([[-1.2, 0.0, 0.0], [-1.1, 0.1, 0.0], [-0.7, 0.0, 0.0], [0.4, 1.0, 0.0],
                    [0.6, 1.0, 0.0]], np.float32)
    a = oracle.voxel_centroid(pts[:, 0], pts[:, 1], pts[:, 2], leaf=0.5, plain_xyz=True)
    b = oracle.voxel_centroid(pts[:, 0], pts[:, 1], pts[:, 2], leaf=0.5,
                              origin=(F(-1.2), 0.0, 0.0), plain_xyz=True)
    for fa, fb in zip(a.fields, b.fields):
        assert np.array_equal(fa, fb)


def test_average_intensity_in_centroid_mode():
    # voxel.rs:1342-1355 (point_xyzi -> generic f64 path)
    r = oracle.voxel_centroid([0.0, 0.1], [0, 0], [0, 0], [[0.2, 0.8]], leaf=1.0)
    assert len(r.x) == 1
    assert abs(r.fields[3][0] - 0.5) < 1e-5


def test_rejects_non_positive_leaf_size():
    # voxel.rs:1357-1364
    with pytest.raises(oracle.OracleError):
        oracle.voxel_centroid([0.0], [0.0], [0.0], leaf=0.0)


def test_mvp_load_voxel_downsample():
    # crates/spatialrust/tests/mvp_pipeline.rs:1-26: 10 pts x = i*0.1, leaf 0.5 -> 0.2, 0.7
    x = np.arange(10, dtype=np.float32) * F(0.1)
    r = oracle.voxel_centroid(x, np.zeros(10), np.zeros(10), leaf=0.5, plain_xyz=True)
    assert len(r.x) == 2
    assert abs(r.x[0] - 0.2) < 1e-5 and abs(r.x[1] - 0.7) < 1e-5


def test_voxel_segments_counts():
    # crates/spatialrust-gpu/src/kernels/voxel_segments.rs test: keys
    # [(0,0,0),(1,0,0),(0,0,0),(1,0,0)] -> counts [2, 2]
    x = np.array([0.1, 1.1, 0.2, 1.2], np.float32)
    r = oracle.voxel_centroid(x, np.zeros(4), np.zeros(4), leaf=1.0, origin=(0, 0, 0))
    assert r.counts.tolist() == [2, 2]
    assert r.keys.tolist() == [[0, 0, 0], [1, 0, 0]]


def test_generic_path_sorted_by_key_and_fp64_means():
    # voxel.rs:522-536: point_xyzi output sorted by (ix,iy,iz); value (sum*(1/count)) as f32
    rng = np.random.default_rng(5)
    pts = rng.random((2000, 3), dtype=np.float32) * F(10)
    inten = rng.random(2000, dtype=np.float32)
    r = oracle.voxel_centroid(pts[:, 0], pts[:, 1], pts[:, 2], [inten], leaf=1.0)
    keys = [tuple(k) for k in r.keys.tolist()]
    assert keys == sorted(keys)
    # numpy restatement of the same arithmetic
    o = pts.min(axis=0)
    k = (((pts - o) * (F(1.0) / F(1.0))).astype(np.float32)).astype(np.int64)
    for row, key in enumerate(keys[:50]):
        m = np.all(k == np.array(key), axis=1)
        assert r.counts[row] == m.sum()
        expect = np.float32(np.sum(pts[m, 0].astype(np.float64)) * (1.0 / m.sum()))
        assert r.x[row] == expect


def test_approximate_keeps_first_point_in_voxel():
    # voxel.rs:1329-1339: approximate(1.0) on two points in one voxel keeps the first
    x = np.array([0.0, 0.1], F)
    zero = np.zeros(2, F)
    r = oracle.voxel_general(x, zero, zero, [np.array([0.2, 0.9], F)], leaf=1.0, approximate=True)
    assert len(r.x) == 1 and r.fields[3][0] == F(0.2) and r.x[0] == F(0.0)


def test_approximate_first_four_points():
    # voxel.rs:1446-1471 (CPU side): approximate(0.5), x = 0, 0.1, 1.0, 1.1, i = 0.2, 0.9, 10, 20
    x = np.array([0.0, 0.1, 1.0, 1.1], F)
    zero = np.zeros(4, F)
    inten = np.array([0.2, 0.9, 10.0, 20.0], F)
    r = oracle.voxel_general(x, zero, zero, [inten], leaf=0.5, approximate=True)
    assert r.x.tolist() == [0.0, 1.0]
    assert r.fields[3].tolist() == [F(0.2), F(10.0)]
    assert r.counts.tolist() == [2, 2]


def test_centroid_first_policy_divides_and_keeps_first_attribute():
    # voxel.rs:1123-1165: Centroid + First: positions (f64 sum / count) as f32,
    # attributes from the first point; the key set is the fast path's
    rng = np.random.default_rng(9)
    pts = (rng.random((3000, 3), dtype=np.float32) * F(7)).astype(np.float32)
    inten = rng.random(3000, dtype=np.float32)
    g = oracle.voxel_general(pts[:, 0], pts[:, 1], pts[:, 2], [inten], leaf=0.7,
                             attribute_first=True)
    f = oracle.voxel_centroid(pts[:, 0], pts[:, 1], pts[:, 2], [inten], leaf=0.7)
    assert np.array_equal(g.keys, f.keys) and np.array_equal(g.counts, f.counts)
    o = pts.min(axis=0)
    k = ((pts - o) * (F(1.0) / F(0.7))).astype(np.float32).astype(np.int64)
    for row in range(0, len(g.x), 97):
        m = np.nonzero(np.all(k == g.keys[row], axis=1))[0]
        assert g.x[row] == np.float32(np.sum(pts[m, 0].astype(np.float64)) / len(m))
        assert g.fields[3][row] == inten[m[0]]


def test_cluster_long_chain_is_one_component():
    # uniform_grid.rs:564-576: 300 points spaced 1.0 on x, tolerance 1.5 -> all root 0
    x = np.arange(300, dtype=F)
    zero = np.zeros(300, F)
    assert np.all(oracle.euclidean_roots(x, zero, zero, 1.5) == 0)


def test_cluster_prebuilt_segments_example():
    # uniform_grid.rs:578-597: x = 0, 0.5, 2.0, tolerance 1.0 -> roots 0, 0, 2
    x = np.array([0.0, 0.5, 2.0], F)
    zero = np.zeros(3, F)
    assert oracle.euclidean_roots(x, zero, zero, 1.0).tolist() == [0, 0, 2]


def test_cluster_three_separated_clusters():
    # cluster.rs:370-383 / cluster_gpu.rs:90-101: three 3x3 grids 10 m apart,
    # tolerance 1.5 -> three components of 9 points
    pts = [(cx + dx, cy + dy, 0.0) for cx, cy in ((0, 0), (10, 0), (0, 10))
           for dx in range(3) for dy in range(3)]
    p = np.array(pts, F)
    roots = oracle.euclidean_roots(p[:, 0], p[:, 1], p[:, 2], 1.5)
    assert sorted(np.unique(roots, return_counts=True)[1].tolist()) == [9, 9, 9]
    assert np.unique(roots).tolist() == [0, 9, 18]


def test_cluster_roots_match_brute_force_components():
    # the component structure of the f32 predicate, by brute-force flood fill
    rng = np.random.default_rng(4)
    p = (rng.random((400, 3)) * 6).astype(F)
    tol = F(0.55)
    roots = oracle.euclidean_roots(p[:, 0], p[:, 1], p[:, 2], tol)
    d = p[None, :, :] - p[:, None, :]
    adj = ((d[..., 0] * d[..., 0] + d[..., 1] * d[..., 1]) + d[..., 2] * d[..., 2]) <= tol * tol
    expect = np.full(400, -1)
    for s in range(400):
        if expect[s] >= 0:
            continue
        stack, expect[s] = [s], s
        while stack:
            i = stack.pop()
            for j in np.nonzero(adj[i])[0]:
                if expect[j] < 0:
                    expect[j] = s
                    stack.append(j)
    assert roots.tolist() == expect.tolist()
    sparse = oracle.euclidean_roots(p[:, 0], p[:, 1], p[:, 2], tol, sparse=True)
    assert sparse.tolist() == expect.tolist()


def test_cluster_rejects_non_positive_tolerance():
    x = np.zeros(3, F)
    with pytest.raises(oracle.OracleError):
        oracle.euclidean_roots(x, x, x, 0.0)


def test_plane_covariance_planar_patch_is_disk():
    # crates/spatialrust-gpu/src/kernels/covariances_grid.rs:371-395: 12x12
    # grid step 0.1 at z = 0, radius 0.25, eps 1e-3 -> c22 ~ eps, c00, c11 > 0.5
    xs, ys = np.meshgrid(np.arange(12) * 0.1, np.arange(12) * 0.1, indexing="ij")
    x, y = xs.ravel().astype(F), ys.ravel().astype(F)
    r = oracle.plane_covariances(x, y, np.zeros_like(x), 0.25, 1e-3)
    assert r.cov.shape == (144, 6)
    assert np.all(np.abs(r.cov[:, 2] - 1e-3) < 1e-2)
    assert np.all(r.cov[:, 0] > 0.5) and np.all(r.cov[:, 1] > 0.5)


def test_plane_covariance_tilted_plane_and_fallback():
    # eigenvalues (eps, 1, 1) about the plane normal: I + (eps - 1) n n^T;
    # an isolated point (1 point in its neighbourhood, < 3) -> (eps, eps, eps, 0, 0, 0)
    eps = 0.01
    u, v = np.meshgrid(np.arange(15) * 0.1, np.arange(15) * 0.1, indexing="ij")
    u, v = u.ravel(), v.ravel()
    x, y, z = u, v, 0.5 * u - 0.25 * v
    x = np.append(x, 50.0).astype(F)
    y = np.append(y, 50.0).astype(F)
    z = np.append(z, 50.0).astype(F)
    r = oracle.plane_covariances(x, y, z, 0.25, eps)
    n = np.array([0.5, -0.25, -1.0])
    n /= np.linalg.norm(n)
    want = np.eye(3) + (eps - 1.0) * np.outer(n, n)
    six = np.array([want[0, 0], want[1, 1], want[2, 2], want[0, 1], want[0, 2], want[1, 2]])
    assert np.max(np.abs(r.cov[:-1] - six[None, :])) < 1e-5
    assert np.array_equal(r.cov[-1], [eps, eps, eps, 0.0, 0.0, 0.0])
    assert r.counts[-1] == 1


def test_plane_covariance_counts_include_the_query():
    rng = np.random.default_rng(5)
    p = rng.uniform(0, 2, (800, 3)).astype(F)
    r = oracle.plane_covariances(p[:, 0], p[:, 1], p[:, 2], 0.3, 1e-3)
    brute = oracle.brute_radius_counts(p[:, 0], p[:, 1], p[:, 2], 0.3)
    assert np.array_equal(r.counts, brute + 1)
    with pytest.raises(oracle.OracleError):
        oracle.plane_covariances(p[:, 0], p[:, 1], p[:, 2], 0.0, 1e-3)


def test_plane_normals_upward_radius():
    # normal.rs:650-667 uses k=8 on a 5x5 unit grid; the radius-mode analogue
    # (r = 1.5 covers the 8-neighbourhood) must give the same upward normals.
    xs, ys = np.meshgrid(np.arange(5, dtype=np.float32), np.arange(5, dtype=np.float32), indexing="ij")
    x, y = xs.ravel(), ys.ravel()
    r = oracle.radius_normals_ref(x, y, np.zeros_like(x), 1.5, 3, (0.0, 0.0, 10.0))
    assert r.valid_count == 25 and r.invalid_count == 0
    assert np.all(np.abs(r.nz - 1.0) < 0.1)


def test_tilted_plane_normals():
    # normal.rs:669-686: z = 0.2x - 0.3y + 0.1 on a 7x7 grid, step 0.2
    pts = []
    for i in range(7):
        for j in range(7):
            fx, fy = F(i) * F(0.2), F(j) * F(0.2)
            pts.append((fx, fy, F(0.2) * fx - F(0.3) * fy + F(0.1)))
    p = np.array(pts, np.float32)
    r = oracle.radius_normals_ref(p[:, 0], p[:, 1], p[:, 2], 0.45, 3, (0.0, 0.0, 10.0))
    expected = np.array([-0.2, 0.3, 1.0]) / np.linalg.norm([-0.2, 0.3, 1.0])
    dots = r.normals @ expected
    assert np.all(dots > 0.98)


def test_orientation_towards_viewpoint():
    # normal.rs:688-695 -- exercised through a plane seen from below
    xs, ys = np.meshgrid(np.arange(5, dtype=np.float32), np.arange(5, dtype=np.float32), indexing="ij")
    x, y = xs.ravel(), ys.ravel()
    r = oracle.radius_normals_ref(x, y, np.zeros_like(x), 1.5, 3, (0.0, 0.0, -10.0))
    assert np.all(r.nz < -0.9)


def test_grid_planar_patch_vertical_normal():
    # normal_gpu.rs:127-152 and normals_grid.rs:359-377: 12x12 grid step 0.1, r 0.25
    xs, ys = np.meshgrid(np.arange(12, dtype=np.float32), np.arange(12, dtype=np.float32), indexing="ij")
    x = xs.ravel() * F(0.1)
    y = ys.ravel() * F(0.1)
    r = oracle.radius_normals_ref(x, y, np.zeros_like(x), 0.25, 3, (0.0, 0.0, 10.0))
    assert np.all(r.nz > 0.99)
    assert np.all(r.curvature < 1e-3)


def test_wgsl_restatement_grid_known_answers():
    # normals_grid.rs:359-377 (no viewpoint: |nz| > 0.99, curvature < 1e-3) and
    # normal_gpu.rs:127-152 (viewpoint (0, 0, 10): nz > 0.99) on the 12x12 grid,
    # through the restatement of the shader's own f32 arithmetic
    xs, ys = np.meshgrid(np.arange(12, dtype=np.float32), np.arange(12, dtype=np.float32), indexing="ij")
    x = xs.ravel() * F(0.1)
    y = ys.ravel() * F(0.1)
    z = np.zeros_like(x)
    r = oracle.grid_normals_wgsl(x, y, z, 0.25)
    assert np.all(np.abs(r.nz) > 0.99) and np.all(r.curvature < 1e-3)
    assert np.all(r.counts >= 5)  # the query and its 4-neighbours at least
    r = oracle.grid_normals_wgsl(x, y, z, 0.25, (0.0, 0.0, 10.0))
    assert np.all(r.nz > 0.99)
    f = oracle.radius_normals_fp64(x, y, z, 0.25, viewpoint=(0.0, 0.0, 10.0), include_self=True)
    assert np.array_equal(f.counts, r.counts) and np.all(f.nz > 0.99)


def test_include_self_semantics_of_the_oracles():
    # normals_grid.rs:129-132: fewer than 3 points (query included) -> (0, 0, 1),
    # curvature 0; turned toward the viewpoint by normal_gpu.rs:63-70
    x = np.array([0.0, 10.0, 10.5, 20.0, 20.3, 20.6, 40.0], np.float32)
    zeros = np.zeros_like(x)
    for vp, sign in ((None, 1.0), ((0.0, 0.0, -5.0), -1.0), ((0.0, 0.0, 5.0), 1.0)):
        f = oracle.radius_normals_fp64(x, zeros, zeros, 1.0, viewpoint=vp, include_self=True)
        w = oracle.grid_normals_wgsl(x, zeros, zeros, 1.0, vp)
        assert f.counts.tolist() == [1, 2, 2, 3, 3, 3, 1] == w.counts.tolist()
        for k in (0, 1, 2, 6):  # fallback points
            assert (f.nx[k], f.ny[k], f.nz[k], f.curvature[k]) == (0.0, 0.0, sign, 0.0)
            assert (w.nx[k], w.ny[k], w.nz[k], w.curvature[k]) == (0.0, 0.0, sign, 0.0)
    # a non-finite query finds nothing, itself included
    xn = np.array([0.0, 0.1, np.nan, 0.2], np.float32)
    f = oracle.radius_normals_fp64(xn, np.zeros(4, F), np.zeros(4, F), 0.5, include_self=True)
    assert f.counts.tolist() == [3, 3, 0, 3]


def test_include_self_counts_are_plain_counts_plus_one():
    rng = np.random.default_rng(17)
    p = rng.random((4000, 3), dtype=np.float32)
    a = oracle.radius_normals_fp64(p[:, 0], p[:, 1], p[:, 2], 0.08, 3)
    b = oracle.radius_normals_fp64(p[:, 0], p[:, 1], p[:, 2], 0.08, 3, include_self=True)
    w = oracle.grid_normals_wgsl(p[:, 0], p[:, 1], p[:, 2], 0.08)
    assert np.array_equal(b.counts, a.counts + 1) and np.array_equal(w.counts, b.counts)
    # where both solve, the shader's f32 Jacobi agrees with the FP64 solve on
    # well-conditioned neighbourhoods (loose: 16 f32 sweeps, f32 sums)
    ok = (b.counts >= 3) & (b.gap >= 0.1)
    cosang = np.abs(np.sum(b.normals[ok] * np.stack([w.nx, w.ny, w.nz], 1)[ok], axis=1))
    assert np.degrees(np.arccos(np.clip(cosang, -1, 1))).max() < 0.5


def test_kdtree_radius_matches_brute_force():
    # kdtree.rs:654 (radius search vs brute force)
    rng = np.random.default_rng(11)
    p = rng.random((1500, 3), dtype=np.float32)
    r = oracle.radius_normals_fp64(p[:, 0], p[:, 1], p[:, 2], 0.1, 3)
    brute = oracle.brute_radius_counts(p[:, 0], p[:, 1], p[:, 2], 0.1)
    assert np.array_equal(r.counts, brute)
    r2 = oracle.radius_normals_ref(p[:, 0], p[:, 1], p[:, 2], 0.1, 3)
    assert np.array_equal(r2.counts, brute)


def test_min_neighbors_invalid_is_nan():
    # normal.rs:331-346: fewer than min_neighbors -> NaN normal, curvature 0
    x = np.array([0.0, 10.0, 20.0], np.float32)
    r = oracle.radius_normals_ref(x, np.zeros(3), np.zeros(3), 1.0, 3)
    assert r.invalid_count == 3
    assert np.all(np.isnan(r.nx)) and np.all(r.curvature == 0)


def test_ref_and_fp64_agree_on_planes():
    rng = np.random.default_rng(3)
    n = 3000
    uv = rng.uniform(-1, 1, (n, 2))
    z = 0.3 * uv[:, 0] - 0.2 * uv[:, 1] + rng.normal(0, 0.01, n)
    p = np.stack([uv[:, 0], uv[:, 1], z], 1).astype(np.float32)
    a = oracle.radius_normals_ref(p[:, 0], p[:, 1], p[:, 2], 0.2, 3, (0, 0, 10))
    b = oracle.radius_normals_fp64(p[:, 0], p[:, 1], p[:, 2], 0.2, 3, (0, 0, 10))
    assert np.array_equal(a.counts, b.counts)
    ok = ~np.isnan(a.nx)
    cosang = np.clip(np.sum(a.normals[ok] * b.normals[ok], axis=1), -1, 1)
    assert np.degrees(np.arccos(cosang)).max() < 0.5


def test_symmetric_eigen_closed_form():
    # normal.rs:475-504 on a diagonal and a rotated covariance
    n, c = oracle.smallest_eigenpair_f32(3.0, 2.0, 1.0, 0.0, 0.0, 0.0)
    assert abs(abs(n[2]) - 1.0) < 1e-6
    assert abs(c - 1.0 / 6.0) < 1e-6
    th = 0.3
    R = np.array([[math.cos(th), -math.sin(th), 0], [math.sin(th), math.cos(th), 0], [0, 0, 1]])
    C = R @ np.diag([0.5, 2.0, 3.0]) @ R.T
    n, c = oracle.smallest_eigenpair_f32(C[0, 0], C[1, 1], C[2, 2], C[0, 1], C[0, 2], C[1, 2])
    assert abs(abs(float(np.dot(n, R[:, 0]))) - 1.0) < 1e-5


def test_parallel_worker_count():
    # crates/spatialrust-search/src/staging.rs:11-28
    assert oracle.parallel_worker_count(4095, 8) == 1
    assert oracle.parallel_worker_count(4096, 8) == 1
    assert oracle.parallel_worker_count(100_000, 8) == 6
    assert oracle.parallel_worker_count(2_000_000, 8) == 8


# ---- bounded streaming voxel (crates/spatialrust-pipeline/src/streaming.rs) --

def test_stream_voxel_identical_output_golden():
    # streaming.rs:1098-1130: leaf 1.0 -> [[0.15,0,0],[1.2,0,0],[2.8,0,0]]
    r = oracle.stream_voxel([1.3, 0.1, 1.1, 0.2, 2.8], [0] * 5, [0] * 5, leaf=1.0)
    assert r.pos.tolist() == np.array([[0.15, 0, 0], [1.2, 0, 0], [2.8, 0, 0]], F).tolist()
    assert r.keys.tolist() == [[0, 0, 0], [1, 0, 0], [2, 0, 0]]
    assert r.counts.tolist() == [2, 2, 1]


def test_stream_voxel_averages_attributes_golden():
    # streaming.rs:1132-1149: intensities 10, 20 | 50 -> [15, 50]
    r = oracle.stream_voxel([0.1, 0.2, 1.1], [0] * 3, [0] * 3,
                            attrs=[np.array([10.0, 20.0, 50.0])], leaf=1.0)
    assert r.attrs[:, 0].tolist() == [15.0, 50.0]


def test_stream_voxel_skips_non_finite_and_floors_negatives():
    r = oracle.stream_voxel([0.0, -0.5, np.nan, 2.0, -1.0], [0, 0, 0, np.inf, 0], [0] * 5, leaf=1.0)
    assert r.keys.tolist() == [[-1, 0, 0], [0, 0, 0]]
    assert r.counts.tolist() == [2, 1]
    with pytest.raises(oracle.OracleError):
        oracle.stream_voxel([1e30], [0], [0], leaf=1e-12)


def test_stream_voxel_compensated_sum_beats_plain_sum():
    # CompensatedSum (streaming.rs:240-262): 1 + 1e-16 * 1000 keeps the small terms
    x = np.full(1001, 0.5, F)
    a = np.full(1001, 1e-16)
    a[0] = 1.0
    r = oracle.stream_voxel(x, np.zeros_like(x), np.zeros_like(x), attrs=[a], leaf=1.0)
    assert r.attrs[0, 0] == (1.0 + 1e-13) / 1001


# ---- RANSAC plane (crates/spatialrust-segmentation/src/plane.rs) ------------

def plane_with_outliers():
    pts = [[x, y, 0.0] for x in range(10) for y in range(10)] + [[0, 0, 5], [1, 1, 5]]
    return np.array(pts, F)


def test_ransac_segments_dominant_plane():
    # plane.rs:372-386 (threshold 0.05, 500 iterations, min 50 inliers, seed 7)
    p = plane_with_outliers()
    r = oracle.ransac_plane(p[:, 0], p[:, 1], p[:, 2], 0.05, 500, 50, 7)
    assert r["inlier_count"] == 100
    assert int((~r["mask"]).sum()) == 2
    assert abs(r["model"][2]) > 0.9
    # extract_outliers_removes_plane (plane.rs:394-406)
    assert np.all(p[~r["mask"], 2] > 1.0)


def test_ransac_errors_follow_the_reference():
    with pytest.raises(oracle.OracleError):
        oracle.ransac_plane([], [], [], 0.05, 10, 3, 1)
    with pytest.raises(oracle.OracleError):
        oracle.ransac_plane([0, 1], [0, 0], [0, 0], 0.05, 10, 1, 1)
    p = plane_with_outliers()
    with pytest.raises(oracle.OracleError):  # min_inliers above the plane's 100
        oracle.ransac_plane(p[:, 0], p[:, 1], p[:, 2], 0.05, 50, 101, 7)
