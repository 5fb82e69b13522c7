"""MvpPipeline on the CUDA library.

Mirrors crates/spatialrust-pipeline/src/mvp.rs (MvpPipelineConfig :54-102,
MvpPipelineResult / MvpPipelineReceipt :104-171, MvpPipeline::run :173-284):
voxel downsample -> radius normals on the centroids -> RANSAC plane ->
Euclidean clusters of the plane's outliers, every stage through its
Gpu(Cuda) arm; with the Centroid + Average voxel mode the first two stages
are one device-resident call (srcu_voxel_normals).  As in the reference's GPU
path, a normals config without search_radius gets
`leaf_size * normal_gpu_radius_scale` (at least 1e-4, mvp.rs:198-211).  The optional ICP registration step is registration, which
this library does not provide: a config with `icp` is refused.
"""
from __future__ import annotations

from dataclasses import dataclass, field, replace
from typing import Optional

from . import _native
from .core import (POSITION_SEMANTICS, Auto, ExecutionPolicy, ExecutionReceipt, FieldSemantic,
                   InvalidArgument, PointCloud, TransferDirection)
from .features import NormalEstimationConfig, NormalEstimator, build_output_cloud
from .filtering import (AttributeAggregation, VoxelAggregationMode, VoxelGridDownsample,
                        VoxelGridDownsampleConfig, _widen, narrow, resolve_cuda_policy,
                        uses_plain_xyz_path)
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

    def _voxel_normals(self, input: PointCloud, normal_config: NormalEstimationConfig):
        """Voxel centroids and their normals in one device-resident call
        (srcu_voxel_normals): the same columns as the two stages run one after
        the other, without the centroids' round trip through the host."""
        c = self._config
        v_resolved = resolve_cuda_policy(c.voxel_policy, "voxel downsampling")
        n_resolved = resolve_cuda_policy(c.normal_policy, "normal estimation")
        if c.voxel.leaf_size <= 0.0:
            raise InvalidArgument("leaf_size must be greater than zero")
        if normal_config.search_radius < 0.0:
            raise InvalidArgument("search_radius must be non-negative")
        x, y, z = input.positions3()
        attr_fields = [f for f in input.schema.fields if f.semantic not in POSITION_SEMANTICS]
        attrs = [_widen(input.columns[f.name]) for f in attr_fields]
        out = _native.shared_context(self._device).voxel_normals(
            x, y, z, attrs, leaf=c.voxel.leaf_size, origin=c.voxel.origin,
            radius=normal_config.search_radius, min_neighbors=normal_config.min_neighbors,
            viewpoint=normal_config.viewpoint, plain_xyz=uses_plain_xyz_path(input.schema, c.voxel))
        cols = out["columns"]
        pos = {f.semantic: f.name for f in input.schema.fields if f.semantic in POSITION_SEMANTICS}
        vcols = {pos[FieldSemantic.PositionX]: cols[0], pos[FieldSemantic.PositionY]: cols[1],
                 pos[FieldSemantic.PositionZ]: cols[2]}
        for f, col in zip(attr_fields, cols[3:]):
            vcols[f.name] = narrow(col, f.dtype)
        downsampled = PointCloud(input.schema, vcols, input.metadata)
        with_normals = build_output_cloud(downsampled, out["nx"], out["ny"], out["nz"],
                                          out["curvature"])
        n, v = len(input), len(cols[0])
        vr = ExecutionReceipt(c.voxel_policy, v_resolved)
        vr.record_stage("voxel-downsample")
        vr.record_transfer(TransferDirection.HostToDevice, n * 4 * (3 + len(attrs)))
        vr.record_transfer(TransferDirection.DeviceToHost, v * 4 * (3 + len(attrs)))
        vr.record_stage("gpu-readback")
        nr = ExecutionReceipt(c.normal_policy, n_resolved)
        nr.record_stage("normal-estimation")
        nr.record_transfer(TransferDirection.DeviceToHost, v * 16)
        nr.record_stage("gpu-readback")
        return downsampled, with_normals, vr, nr

    def run(self, input: PointCloud) -> MvpPipelineResult:
        c = self._config
        if c.icp is not None:
            raise InvalidArgument("the ICP registration step is not part of this library's CUDA "
                                  "arms; run it in SpatialRust's registration crate")
        normal_config = c.normals
        if normal_config.search_radius is None:  # mvp.rs:198-211
            radius = max(c.voxel.leaf_size * c.normal_gpu_radius_scale, 1e-4)
            normal_config = replace(normal_config, search_radius=float(radius))
        if (c.voxel.mode == VoxelAggregationMode.Centroid
                and c.voxel.attribute_policy == AttributeAggregation.Average
                and not input.is_empty()):
            downsampled, with_normals, voxel_receipt, normals_receipt = self._voxel_normals(
                input, normal_config)
        else:
            voxel = VoxelGridDownsample(c.voxel, self._device).filter_with_policy_and_receipt(
                input, c.voxel_policy)
            downsampled, voxel_receipt = voxel.output, voxel.receipt
            normals = NormalEstimator(normal_config, self._device) \
                .estimate_with_policy_and_receipt(downsampled, c.normal_policy)
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
