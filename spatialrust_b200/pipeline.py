"""MvpPipeline on the CUDA library.

Mirrors crates/spatialrust-pipeline/src/mvp.rs (MvpPipelineConfig :54-102,
MvpPipelineResult / MvpPipelineReceipt :104-171, MvpPipeline::run :173-284):
voxel downsample -> radius normals on the centroids -> RANSAC plane ->
Euclidean clusters of the plane's outliers, every stage through its
Gpu(Cuda) arm.  As in the reference's GPU path, a normals config without
search_radius gets `leaf_size * normal_gpu_radius_scale` (at least 1e-4,
mvp.rs:198-211).  The optional ICP registration step is registration, which
this library does not provide: a config with `icp` is refused.
"""
from __future__ import annotations

from dataclasses import dataclass, field, replace
from typing import Optional

from .core import (Auto, ExecutionPolicy, ExecutionReceipt, InvalidArgument, PointCloud,
                   TransferDirection)
from .features import NormalEstimationConfig, NormalEstimator
from .filtering import VoxelGridDownsample, VoxelGridDownsampleConfig
from .segmentation import (EuclideanClusterConfig, EuclideanClusterExtractor,
                           EuclideanClusterResult, RansacPlaneConfig, RansacPlaneSegmentation,
                           RansacPlaneSegmenter)


@dataclass
class MvpPipelineConfig:
    """MvpPipelineConfig (mvp.rs:54-102)."""

    voxel: VoxelGridDownsampleConfig = field(
        default_factory=lambda: VoxelGridDownsampleConfig.centroid(0.05))
    normals: NormalEstimationConfig = field(default_factory=NormalEstimationConfig)
    plane: RansacPlaneConfig = field(default_factory=RansacPlaneConfig)
    cluster: EuclideanClusterConfig = field(default_factory=EuclideanClusterConfig)
    icp: Optional[object] = None
    voxel_policy: ExecutionPolicy = Auto
    plane_policy: ExecutionPolicy = Auto
    normal_policy: ExecutionPolicy = Auto
    normal_gpu_radius_scale: float = 2.0
    cluster_policy: ExecutionPolicy = Auto

    @staticmethod
    def with_voxel_leaf_size(leaf_size: float) -> "MvpPipelineConfig":
        return MvpPipelineConfig(voxel=VoxelGridDownsampleConfig.centroid(leaf_size))


@dataclass
class MvpPipelineReceipt:
    """MvpPipelineReceipt (mvp.rs:122-171)."""

    voxel: ExecutionReceipt
    normals: ExecutionReceipt
    plane: ExecutionReceipt
    clusters: ExecutionReceipt
    registration: Optional[ExecutionReceipt] = None

    def _total(self, direction: TransferDirection) -> int:
        return sum(r.transfers.get(direction, 0)
                   for r in (self.voxel, self.normals, self.plane, self.clusters))

    def host_to_device_bytes(self) -> int:
        return self._total(TransferDirection.HostToDevice)

    def device_to_device_bytes(self) -> int:
        return self._total(TransferDirection.DeviceToDevice)

    def device_to_host_bytes(self) -> int:
        return self._total(TransferDirection.DeviceToHost)


@dataclass
class MvpPipelineResult:
    """MvpPipelineResult (mvp.rs:104-120)."""

    downsampled: PointCloud
    with_normals: PointCloud
    plane: RansacPlaneSegmentation
    clusters: EuclideanClusterResult
    output: PointCloud
    receipt: MvpPipelineReceipt
    registration: Optional[object] = None


class MvpPipeline:
    """MvpPipeline (mvp.rs:173-284)."""

    def __init__(self, config: MvpPipelineConfig, device: int = 0):
        self._config = config
        self._device = device

    def config(self) -> MvpPipelineConfig:
        return self._config

    def run(self, input: PointCloud) -> MvpPipelineResult:
        c = self._config
        if c.icp is not None:
            raise InvalidArgument("the ICP registration step is not part of this library's CUDA "
                                  "arms; run it in SpatialRust's registration crate")
        voxel = VoxelGridDownsample(c.voxel, self._device).filter_with_policy_and_receipt(
            input, c.voxel_policy)
        downsampled, voxel_receipt = voxel.output, voxel.receipt
        normal_config = c.normals
        if normal_config.search_radius is None:  # mvp.rs:198-211
            radius = max(c.voxel.leaf_size * c.normal_gpu_radius_scale, 1e-4)
            normal_config = replace(normal_config, search_radius=float(radius))
        normals = NormalEstimator(normal_config, self._device).estimate_with_policy_and_receipt(
            downsampled, c.normal_policy)
        with_normals, normals_receipt = normals.output, normals.receipt
        plane = RansacPlaneSegmenter(c.plane, self._device).segment_with_policy_and_receipt(
            with_normals, c.plane_policy)
        clusters = EuclideanClusterExtractor(c.cluster, self._device) \
            .extract_with_policy_and_receipt(plane.output.outliers, c.cluster_policy)
        return MvpPipelineResult(
            downsampled=downsampled, with_normals=with_normals, plane=plane.output,
            clusters=clusters.output, output=clusters.output.cloud,
            receipt=MvpPipelineReceipt(voxel_receipt, normals_receipt, plane.receipt,
                                       clusters.receipt))
