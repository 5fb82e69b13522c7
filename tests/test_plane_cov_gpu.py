"""CUDA GICP plane covariances (srcu_plane_covariances) vs the FP64 oracle.

Bar: which points fall back to (eps, eps, eps, 0, 0, 0) is exact (fewer than 3
points within radius, the query included, by the reference's f32 predicate);
every other element is within COV_TOL of the FP64 oracle wherever the
neighbourhood's plane is well defined (relative eigengap >= GAP_MIN).  The
regularised matrix is I + (eps - 1) n n^T, so an element error is at most
2 |dn|: COV_TOL = 2e-4 is the 1e-4 rad normal bound."""
import numpy as np
import pytest

import oracle
from spatialrust_b200 import InvalidArgument, gpu, synthetic

pytestmark = pytest.mark.gpu
F = np.float32
COV_TOL = 2e-4
GAP_MIN = 1e-3


def check(ctx, x, y, z, radius, eps):
    got, stats = ctx.plane_covariances(x, y, z, radius, eps, with_stats=True)
    ref = oracle.plane_covariances(x, y, z, radius, eps)
    fallback = ref.counts < 3
    assert stats["valid_count"] == int((~fallback).sum())
    assert stats["invalid_count"] == int(fallback.sum())
    assert np.array_equal(got[fallback], np.tile(np.array([eps, eps, eps, 0, 0, 0], F),
                                                 (int(fallback.sum()), 1)))
    well = ~fallback & (ref.gap >= GAP_MIN)
    err = np.abs(got[well].astype(np.float64) - ref.cov[well]).max() if well.any() else 0.0
    assert err <= COV_TOL, f"max element error {err:.3e}"
    return got, ref


def test_planar_patch_is_disk():
    # covariances_grid.rs:371-395
    xs, ys = np.meshgrid(np.arange(12) * 0.1, np.arange(12) * 0.1, indexing="ij")
    x, y = xs.ravel().astype(F), ys.ravel().astype(F)
    eps = 1e-3
    cov = gpu.estimate_plane_covariances_grid_gpu(x, y, np.zeros_like(x), 0.25, eps)
    assert cov.shape == (144, 6)
    assert np.all(np.abs(cov[:, 2] - eps) < 1e-2)
    assert np.all(cov[:, 0] > 0.5) and np.all(cov[:, 1] > 0.5)


def test_parity_on_scan(cuda_ctx):
    c = synthetic.georef_scan(150_000, seed=43)
    check(cuda_ctx, c.x, c.y, c.z, 0.3, 1e-3)


def test_parity_on_shapes_with_sparse_points(cuda_ctx):
    c = synthetic.shapes_scene(120_000, seed=9)
    rng = np.random.default_rng(9)
    # isolated points: neighbourhoods of 1 and 2 points take the fallback
    far = rng.uniform(500, 5000, (300, 3)).astype(F)
    x = np.concatenate([c.x, far[:, 0], far[:150, 0] + F(0.01)])
    y = np.concatenate([c.y, far[:, 1], far[:150, 1]])
    z = np.concatenate([c.z, far[:, 2], far[:150, 2]])
    got, ref = check(cuda_ctx, x, y, z, 0.15, 0.05)
    assert int((ref.counts < 3).sum()) >= 300


def test_size_independent_properties_at_two_million(cuda_ctx):
    # eigenvalues (eps, 1, 1): trace 2 + eps and determinant eps per valid point
    c = synthetic.georef_scan(2_000_000, seed=1)
    eps = 1e-3
    cov, stats = cuda_ctx.plane_covariances(c.x, c.y, c.z, 0.5, eps, with_stats=True)
    assert cov.shape == (2_000_000, 6)
    fb = np.all(cov == np.array([eps, eps, eps, 0, 0, 0], F), axis=1)
    assert stats["invalid_count"] == int(fb.sum())
    m = cov[~fb].astype(np.float64)
    tr = m[:, 0] + m[:, 1] + m[:, 2]
    det = (m[:, 0] * (m[:, 1] * m[:, 2] - m[:, 5] ** 2) - m[:, 3] * (m[:, 3] * m[:, 2] - m[:, 5] * m[:, 4])
           + m[:, 4] * (m[:, 3] * m[:, 5] - m[:, 1] * m[:, 4]))
    assert np.max(np.abs(tr - (2 + eps))) < 1e-5
    assert np.max(np.abs(det - eps)) < 1e-5


def test_device_inputs_and_outputs(cuda_ctx):
    import torch
    c = synthetic.shapes_scene(50_000, seed=10)
    host = cuda_ctx.plane_covariances(c.x, c.y, c.z, 0.2, 1e-3)
    dev = [torch.from_numpy(a).cuda() for a in (c.x, c.y, c.z)]
    out = cuda_ctx.plane_covariances(*dev, 0.2, 1e-3)
    assert out.is_cuda and tuple(out.shape) == (50_000, 6)
    assert np.array_equal(out.cpu().numpy(), host)


def test_empty_input_and_argument_errors(cuda_ctx):
    e = np.zeros(0, F)
    assert cuda_ctx.plane_covariances(e, e, e, 0.5, 1e-3).shape == (0, 6)
    # empty input is returned before the radius is checked (covariances_grid.rs:228-233)
    assert gpu.estimate_plane_covariances_grid_gpu(e, e, e, 0.0, 1e-3).shape == (0, 6)
    x = np.zeros(4, F)
    for bad in (0.0, -1.0, float("nan"), float("inf")):
        with pytest.raises(InvalidArgument):
            cuda_ctx.plane_covariances(x, x, x, bad, 1e-3)
