"""RANSAC plane segmentation on the device vs the reference CPU segmenter.

Bar: the winning hypothesis, the inlier count and the inlier mask are exact
(the counts use the reference's f32 expressions); the hypothesis plane is
bit-exact; the refined model (FP64 sums in a different order) is within 1e-6
of the oracle's."""
import numpy as np
import pytest

import oracle
import spatialrust_b200 as sr
from spatialrust_b200 import gpu, synthetic

pytestmark = pytest.mark.gpu
F = np.float32


def cloud_of(p):
    return sr.PointCloud(sr.StandardSchemas.point_xyz(), {"x": p[:, 0], "y": p[:, 1], "z": p[:, 2]})


def plane_with_outliers():
    pts = [[x, y, 0.0] for x in range(10) for y in range(10)] + [[0, 0, 5], [1, 1, 5]]
    return np.array(pts, F)


def test_reference_dominant_plane_and_outliers():
    # plane.rs:372-406 and plane_gpu.rs:117-133 (threshold 0.05, 500 iterations, seed 7)
    cfg = sr.RansacPlaneConfig(distance_threshold=0.05, max_iterations=500, min_inliers=50, seed=7)
    res = sr.RansacPlaneSegmenter(cfg).segment(cloud_of(plane_with_outliers()))
    assert res.inlier_count == 100 and len(res.outliers) == 2
    assert abs(res.model.normal[2]) > 0.9
    assert np.all(res.outliers.field("z") > 1.0)
    gpu_res = sr.GpuRansacPlaneSegmenter(cfg).segment(cloud_of(plane_with_outliers()))
    assert gpu_res.inlier_count == res.inlier_count and len(gpu_res.outliers) == 2


@pytest.mark.parametrize("seed", [1, 42, 12345])
def test_parity_on_a_scan(cuda_ctx, seed):
    c = synthetic.georef_scan(40_000, seed=60 + seed)
    info, mask = cuda_ctx.ransac_plane_segment(c.x, c.y, c.z, 0.05, 300, 3, seed)
    ref = oracle.ransac_plane(c.x, c.y, c.z, 0.05, 300, 3, seed)
    assert info["best_hypothesis"] == ref["best_index"]
    assert info["inlier_count"] == ref["inlier_count"]
    assert np.array_equal(mask, ref["mask"])
    assert np.array_equal(np.array(info["hypothesis_normal"] + (info["hypothesis_d"],), F),
                          ref["hypothesis"])
    got = np.array(info["normal"] + (info["d"],), np.float64)
    assert np.max(np.abs(got - ref["model"])) <= 1e-6 * max(1.0, abs(float(ref["model"][3])))


def test_scores_match_numpy_f32(cuda_ctx):
    c = synthetic.shapes_scene(60_000, seed=13)
    rng = np.random.default_rng(13)
    hyp = rng.integers(0, 60_000, (700, 3)).astype(np.uint32)
    hyp[5] = [7, 7, 9]  # a degenerate triple scores zeros
    got = gpu.score_ransac_plane_hypotheses_gpu(c.x, c.y, c.z, hyp, 0.02)
    x, y, z = c.x, c.y, c.z
    for h in range(0, 700, 7):
        i0, i1, i2 = hyp[h]
        v1 = np.array([x[i1] - x[i0], y[i1] - y[i0], z[i1] - z[i0]], F)
        v2 = np.array([x[i2] - x[i0], y[i2] - y[i0], z[i2] - z[i0]], F)
        n = np.array([v1[1] * v2[2] - v1[2] * v2[1], v1[2] * v2[0] - v1[0] * v2[2],
                      v1[0] * v2[1] - v1[1] * v2[0]], F)
        ls = F(F(n[0] * n[0] + n[1] * n[1]) + n[2] * n[2])
        if ls < F(1e-12):
            assert got[h] == (0, (0.0, 0.0, 0.0), 0.0)
            continue
        n = (n / np.sqrt(ls)).astype(F)
        d = -F(F(n[0] * x[i0] + n[1] * y[i0]) + n[2] * z[i0])
        dist = np.abs(((n[0] * x + n[1] * y) + n[2] * z) + d)
        assert got[h][0] == int(np.count_nonzero(dist <= F(0.02))), h
        assert got[h][1] == tuple(float(v) for v in n) and got[h][2] == float(d)


def test_device_inputs_give_the_same_mask(cuda_ctx):
    import torch
    c = synthetic.georef_scan(30_000, seed=64)
    info, mask = cuda_ctx.ransac_plane_segment(c.x, c.y, c.z, 0.05, 200, 3, 9)
    dev = [torch.from_numpy(a).cuda() for a in (c.x, c.y, c.z)]
    info_d, mask_d = cuda_ctx.ransac_plane_segment(*dev, 0.05, 200, 3, 9)
    assert mask_d.is_cuda and np.array_equal(mask_d.cpu().numpy().astype(bool), mask)
    assert info_d == info


def test_errors(cuda_ctx):
    e = np.zeros(0, F)
    with pytest.raises(sr.InvalidArgument, match="empty"):
        cuda_ctx.ransac_plane_segment(e, e, e)
    with pytest.raises(sr.InvalidArgument, match="three points"):
        cuda_ctx.ransac_plane_segment(np.zeros(2, F), np.zeros(2, F), np.zeros(2, F))
    p = plane_with_outliers()
    with pytest.raises(sr.InvalidArgument, match="minimum is 101"):
        cuda_ctx.ransac_plane_segment(p[:, 0], p[:, 1], p[:, 2], 0.05, 50, 101, 7)
    line = np.arange(50, dtype=F)  # collinear: every hypothesis degenerate
    with pytest.raises(sr.InvalidArgument):
        cuda_ctx.ransac_plane_segment(line, line, line, 0.05, 20, 1, 3)
    with pytest.raises(sr.InvalidArgument):
        cuda_ctx.ransac_plane_scores(p[:, 0], p[:, 1], p[:, 2], [[0, 1, 500]], 0.05)
