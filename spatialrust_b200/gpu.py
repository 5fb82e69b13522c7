"""Free functions of spatialrust-gpu that run on the uniform radius grid,
on the CUDA library (crates/spatialrust-gpu/src/lib.rs:38-54 exports them).

    estimate_normals_grid_gpu            kernels/normals_grid.rs:208-350
    euclidean_cluster_roots_gpu          kernels/euclidean_cluster.rs:62-71
    estimate_plane_covariances_grid_gpu  kernels/covariances_grid.rs:216-364
    score_ransac_plane_hypotheses_gpu    kernels/ransac_plane.rs:104-263

The reference takes a &WgpuRuntime first; here the device index is a
keyword argument and the process-wide context of that device plays the
runtime's part (runtime.rs:72-95).  Inputs are f32 columns (numpy, or CUDA
tensors for device-resident data); outputs are numpy arrays with one row per
point in input order (CUDA tensors when the inputs were).
"""
from __future__ import annotations

import numpy as np

from . import _native
from .core import InvalidArgument


def _len(col) -> int:
    return int(col.shape[0]) if hasattr(col, "shape") else len(col)


def estimate_normals_grid_gpu(x, y, z, radius: float, device: int = 0) -> np.ndarray:
    """(n, 4) rows [nx, ny, nz, curvature] (GpuNormal, normals.rs:20-25) with
    the grid shader's semantics: self-inclusive radius neighbourhoods, fewer
    than 3 points -> (0, 0, 1, 0) (normals_grid.rs:86-197)."""
    if _len(x) and not radius > 0.0:  # normals_grid.rs:219-224: empty input first
        raise InvalidArgument("grid radius must be positive")
    nx, ny, nz, curv, _, _ = _native.shared_context(device).radius_normals(
        x, y, z, radius, include_self=True)
    return np.stack([nx, ny, nz, curv], axis=1)


def euclidean_cluster_roots_gpu(x, y, z, cluster_tolerance: float, device: int = 0):
    """Smallest point index of every point's connected component
    (uniform_grid.rs:90-139 semantics; union-find on the device)."""
    if _len(x) and not cluster_tolerance > 0.0:  # uniform_grid.rs:100-105: empty input first
        raise InvalidArgument("cluster_tolerance must be positive")
    return _native.shared_context(device).euclidean_cluster_roots(x, y, z, cluster_tolerance)


def estimate_plane_covariances_grid_gpu(x, y, z, radius: float, epsilon: float,
                                        device: int = 0):
    """(n, 6) GICP plane-regularised covariances [c00, c11, c22, c01, c02, c12]
    (GpuCovariance, covariances_grid.rs:21-23): the radius-neighbourhood
    covariance (query included) with eigenvalues replaced by (epsilon, 1, 1);
    fewer than 3 points -> (epsilon, epsilon, epsilon, 0, 0, 0)."""
    if _len(x) and not radius > 0.0:  # covariances_grid.rs:228-233: empty input first
        raise InvalidArgument("grid radius must be positive")
    return _native.shared_context(device).plane_covariances(x, y, z, radius, epsilon)


def score_ransac_plane_hypotheses_gpu(x, y, z, hypotheses, distance_threshold: float,
                                      device: int = 0):
    """[(inlier_count, (nx, ny, nz), d)] per hypothesis (GpuPlaneScore,
    ransac_plane.rs:27-37): the plane through the three indexed points and its
    inliers, in the CPU path's f32 arithmetic; a degenerate triple scores zeros."""
    hyp = np.asarray(hypotheses, np.uint32).reshape(-1, 3)
    if len(hyp) == 0:  # ransac_plane.rs:124-126
        return []
    return _native.shared_context(device).ransac_plane_scores(x, y, z, hyp, distance_threshold)
