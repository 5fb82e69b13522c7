"""Euclidean cluster extraction with the ExecutionPolicy::Gpu(DeviceKind::Cuda) arm.

Mirrors crates/spatialrust-segmentation/src/cluster.rs (EuclideanClusterConfig
:21-60, EuclideanClusterExtractor::extract_with_policy :123-235,
finalize_euclidean_clusters :244-288) and cluster_gpu.rs
(GpuEuclideanClusterExtractor :10-63).  The component roots come from the CUDA
library (srcu_euclidean_cluster_roots: grid, union-find and root compression
all on the device); the size filter and the label numbering are the
reference's own host-side finalisation.
"""
from __future__ import annotations

from dataclasses import dataclass
from typing import List, Optional

import numpy as np

from . import _native
from .core import (DeviceKind, DType, ExecutionOutput, ExecutionPolicy, ExecutionReceipt,
                   FieldSemantic, InvalidArgument, PointCloud, PointField, TransferDirection)
from .filtering import resolve_cuda_policy

USIZE_MAX = (1 << 64) - 1


@dataclass(frozen=True)
class EuclideanClusterConfig:
    cluster_tolerance: float = 0.02
    min_cluster_size: int = 1
    max_cluster_size: int = USIZE_MAX
    gpu_min_points: Optional[int] = None


@dataclass
class EuclideanClusterResult:
    cloud: PointCloud
    cluster_count: int
    cluster_sizes: List[int]


def with_labels(input: PointCloud, field_name: str, labels: np.ndarray) -> PointCloud:
    """with_labels (cloud.rs:44-74): the input columns plus an i32 label column."""
    schema = input.schema
    if schema.find_semantic(FieldSemantic.Label) is None:
        schema = schema.with_field(PointField.scalar(field_name, FieldSemantic.Label, DType.I32))
    cols = {k: v.copy() for k, v in input.columns.items()}
    cols[field_name] = np.asarray(labels, np.int32)
    return PointCloud(schema, cols, input.metadata)


def finalize_euclidean_clusters(input: PointCloud, roots: np.ndarray,
                                config: EuclideanClusterConfig) -> EuclideanClusterResult:
    """finalize_euclidean_clusters (cluster.rs:244-288): components whose size
    lies in [min_cluster_size, max_cluster_size] are numbered in ascending root
    order; every other point gets label -1."""
    if len(roots) != len(input):
        raise InvalidArgument("component root labels must match point count")
    uniq, inverse, sizes = np.unique(roots, return_inverse=True, return_counts=True)
    keep = (sizes >= config.min_cluster_size) & (sizes <= config.max_cluster_size)
    ids = np.full(len(uniq), -1, np.int64)
    ids[keep] = np.arange(int(keep.sum()))
    labels = ids[inverse].astype(np.int32) if len(roots) else np.zeros(0, np.int32)
    cluster_sizes = [int(s) for s in sizes[keep]]
    return EuclideanClusterResult(with_labels(input, "label", labels), len(cluster_sizes),
                                  cluster_sizes)


class GpuEuclideanClusterExtractor:
    """GpuEuclideanClusterExtractor (cluster_gpu.rs:10-63) on the CUDA library."""

    def __init__(self, config: EuclideanClusterConfig, device: int = 0):
        self._config = config
        self._device = device

    def config(self) -> EuclideanClusterConfig:
        return self._config

    def name(self) -> str:
        return "GpuEuclideanClusterExtractor"

    def extract(self, input: PointCloud) -> EuclideanClusterResult:
        return self.extract_with_receipt(input)[0]

    def extract_with_receipt(self, input: PointCloud):
        if input.is_empty():
            return EuclideanClusterResult(input.clone(), 0, []), {}
        tol = float(self._config.cluster_tolerance)
        if not tol > 0.0:  # uniform_grid.rs:103-105
            raise InvalidArgument("cluster_tolerance must be positive")
        x, y, z = input.positions3()
        ctx = _native.shared_context(self._device)
        roots = ctx.euclidean_cluster_roots(x, y, z, tol)
        n = len(input)
        transfers = {TransferDirection.HostToDevice: n * 12, TransferDirection.DeviceToHost: n * 4}
        return finalize_euclidean_clusters(input, roots, self._config), transfers


class EuclideanClusterExtractor:
    """EuclideanClusterExtractor (cluster.rs:62-235): the Gpu(Cuda) arm, which
    the reference rejects today (cluster.rs:233-235)."""

    def __init__(self, config: EuclideanClusterConfig, device: int = 0):
        self._config = config
        self._device = device

    def config(self) -> EuclideanClusterConfig:
        return self._config

    def name(self) -> str:
        return "EuclideanClusterExtractor"

    def extract(self, input: PointCloud) -> EuclideanClusterResult:
        """The reference runs CpuSingle here; this package's only backend is
        CUDA, so it runs Gpu(Cuda)."""
        return self.extract_with_policy(input, ExecutionPolicy.gpu(DeviceKind.Cuda))

    def extract_with_policy(self, input: PointCloud,
                            policy: ExecutionPolicy) -> EuclideanClusterResult:
        return self.extract_with_policy_and_receipt(input, policy).into_output()

    def extract_with_policy_and_receipt(self, input: PointCloud,
                                        policy: ExecutionPolicy) -> ExecutionOutput:
        resolved = resolve_cuda_policy(policy, "Euclidean clustering")
        out, transfers = GpuEuclideanClusterExtractor(self._config, self._device) \
            .extract_with_receipt(input)
        receipt = ExecutionReceipt(policy, resolved)
        receipt.record_stage("euclidean-clustering")
        if transfers:
            for direction, nbytes in transfers.items():
                receipt.record_transfer(direction, nbytes)
            receipt.record_stage("gpu-sparse-grid")
        return ExecutionOutput(out, receipt)



# ---- RANSAC plane segmentation (plane.rs, plane_gpu.rs, cloud.rs) -------------

DEFAULT_GPU_MIN_POINTS_PLANE = 2_000  # plane.rs:50


@dataclass(frozen=True)
class PlaneModel:
    """PlaneModel (plane.rs:15-42): unit normal and offset, n.p + d = 0."""

    normal: tuple
    d: float

    def signed_distance(self, p) -> float:
        n = np.asarray(self.normal, np.float32)
        return float(np.float32(n[0] * np.float32(p[0]) + n[1] * np.float32(p[1])
                                + n[2] * np.float32(p[2]) + np.float32(self.d)))

    def distance(self, p) -> float:
        return abs(self.signed_distance(p))


@dataclass(frozen=True)
class RansacPlaneConfig:
    """RansacPlaneConfig (plane.rs:55-105)."""

    distance_threshold: float = 0.01
    max_iterations: int = 1_000
    min_inliers: int = 3
    seed: int = 42
    gpu_min_points: Optional[int] = DEFAULT_GPU_MIN_POINTS_PLANE

    @staticmethod
    def with_distance_threshold(distance_threshold: float) -> "RansacPlaneConfig":
        return RansacPlaneConfig(distance_threshold=distance_threshold)

    def without_gpu_min_points(self) -> "RansacPlaneConfig":
        return RansacPlaneConfig(self.distance_threshold, self.max_iterations, self.min_inliers,
                                 self.seed, None)


@dataclass
class RansacPlaneSegmentation:
    """RansacPlaneSegmentation (plane.rs:108-119)."""

    model: PlaneModel
    inliers: PointCloud
    outliers: PointCloud
    inlier_count: int


def extract_mask(input: PointCloud, mask: np.ndarray) -> PointCloud:
    """extract_mask (cloud.rs:29-42): the selected points, in order, same schema
    and metadata."""
    mask = np.asarray(mask, bool)
    if len(mask) != len(input):
        raise InvalidArgument(f"mask length {len(mask)} does not match point count {len(input)}")
    return PointCloud(input.schema, {k: v[mask] for k, v in input.columns.items()}, input.metadata)


class GpuRansacPlaneSegmenter:
    """GpuRansacPlaneSegmenter (plane_gpu.rs:16-91) on the CUDA library, with the
    CPU segmenter's results (srcu_ransac_plane_segment)."""

    def __init__(self, config: RansacPlaneConfig, device: int = 0):
        self._config = config
        self._device = device

    def config(self) -> RansacPlaneConfig:
        return self._config

    def name(self) -> str:
        return "GpuRansacPlaneSegmenter"

    def segment(self, input: PointCloud) -> RansacPlaneSegmentation:
        return self.segment_with_info(input)[0]

    def segment_with_info(self, input: PointCloud):
        if input.is_empty():  # plane.rs:267-271
            raise InvalidArgument("cannot segment plane from empty point cloud")
        x, y, z = input.positions3()
        if len(input) < 3:
            raise InvalidArgument("plane segmentation requires at least three points")
        c = self._config
        info, mask = _native.shared_context(self._device).ransac_plane_segment(
            x, y, z, c.distance_threshold, c.max_iterations, c.min_inliers, c.seed)
        model = PlaneModel(tuple(float(v) for v in info["normal"]), float(info["d"]))
        return RansacPlaneSegmentation(model, extract_mask(input, mask), extract_mask(input, ~mask),
                                       info["inlier_count"]), info


class RansacPlaneSegmenter:
    """RansacPlaneSegmenter (plane.rs:121-306): the Gpu(Cuda) arm, which the
    reference rejects today (plane.rs:259-261)."""

    def __init__(self, config: RansacPlaneConfig, device: int = 0):
        self._config = config
        self._device = device

    def config(self) -> RansacPlaneConfig:
        return self._config

    def name(self) -> str:
        return "RansacPlaneSegmenter"

    def segment(self, input: PointCloud) -> RansacPlaneSegmentation:
        """The reference runs CpuSingle here; this package's only backend is
        CUDA, so it runs Gpu(Cuda)."""
        return self.segment_with_policy(input, ExecutionPolicy.gpu(DeviceKind.Cuda))

    def segment_with_policy(self, input: PointCloud,
                            policy: ExecutionPolicy) -> RansacPlaneSegmentation:
        return self.segment_with_policy_and_receipt(input, policy).into_output()

    def segment_with_policy_and_receipt(self, input: PointCloud,
                                        policy: ExecutionPolicy) -> ExecutionOutput:
        resolved = resolve_cuda_policy(policy, "plane segmentation")
        out, info = GpuRansacPlaneSegmenter(self._config, self._device).segment_with_info(input)
        receipt = ExecutionReceipt(policy, resolved)
        receipt.record_stage("plane-segmentation")
        # plane.rs:172-187: points up, hypotheses up, scores down
        receipt.record_transfer(TransferDirection.HostToDevice, len(input) * 12)
        receipt.record_transfer(TransferDirection.HostToDevice, info["hypotheses"] * 16)
        receipt.record_transfer(TransferDirection.DeviceToHost, info["hypotheses"] * 20)
        receipt.record_stage("gpu-score-readback")
        return ExecutionOutput(out, receipt)

    def extract_outliers(self, input: PointCloud) -> PointCloud:
        return self.segment(input).outliers
