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

