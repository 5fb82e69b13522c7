"""VoxelGridDownsample with the ExecutionPolicy::Gpu(DeviceKind::Cuda) arm.

Mirrors crates/spatialrust-filtering/src/voxel.rs: the config
(VoxelGridDownsampleConfig, voxel.rs:112-183), the filter entry points
(filter_with_policy / filter_with_policy_and_receipt, voxel.rs:213-237) and
the validation of filter_internal (voxel.rs:251-275).  Execution goes through
the CUDA library (include/srcuda.h); this package has no CPU implementation,
so explicit CPU policies are rejected rather than silently served elsewhere.
"""
from __future__ import annotations

import enum
from dataclasses import dataclass, replace
from typing import Optional, Tuple

import numpy as np

from . import _native
from .core import (POSITION_SEMANTICS, DeviceKind, DType, ExecutionOutput, ExecutionPolicy,
                   ExecutionReceipt, FieldSemantic, InvalidArgument, PointCloud, TransferDirection,
                   UnsupportedDType)

DEFAULT_GPU_MIN_POINTS = None  # the CUDA arm has no crossover threshold; Auto selects CUDA


class VoxelAggregationMode(enum.Enum):
    Centroid = "centroid"
    ApproximateFirst = "approximate_first"


class AttributeAggregation(enum.Enum):
    Average = "average"
    First = "first"


@dataclass(frozen=True)
class VoxelGridDownsampleConfig:
    leaf_size: float
    origin: Optional[Tuple[float, float, float]] = None
    mode: VoxelAggregationMode = VoxelAggregationMode.Centroid
    attribute_policy: AttributeAggregation = AttributeAggregation.Average
    gpu_min_points: Optional[int] = None

    @staticmethod
    def centroid(leaf_size: float) -> "VoxelGridDownsampleConfig":
        return VoxelGridDownsampleConfig(float(leaf_size))

    @staticmethod
    def approximate(leaf_size: float) -> "VoxelGridDownsampleConfig":
        return VoxelGridDownsampleConfig(float(leaf_size), None,
                                         VoxelAggregationMode.ApproximateFirst,
                                         AttributeAggregation.First)

    def without_gpu_min_points(self) -> "VoxelGridDownsampleConfig":
        return replace(self, gpu_min_points=None)

    def with_origin(self, origin) -> "VoxelGridDownsampleConfig":
        return replace(self, origin=tuple(float(v) for v in origin))


def resolve_cuda_policy(policy: ExecutionPolicy, what: str) -> ExecutionPolicy:
    """Policy resolution of the CUDA arm.  An explicit GPU request never falls
    back (voxel.rs:209-212); Auto resolves to CUDA because this package has no
    other backend."""
    policy.validate()
    if policy.kind == "gpu":
        if policy.device == DeviceKind.Cuda:
            return policy
        raise InvalidArgument(f"unsupported GPU device kind for {what}: {policy.device.name}")
    if policy.kind == "auto":
        return ExecutionPolicy.gpu(DeviceKind.Cuda)
    raise InvalidArgument(
        f"{policy!r} {what} runs in SpatialRust's own CPU code; this library provides the "
        "Gpu(Cuda) arm only")


def _widen(col: np.ndarray) -> np.ndarray:
    """read_buffer_f32 (voxel.rs:692-701): every numeric column read as f32."""
    return np.ascontiguousarray(col, dtype=np.float32)


def _round_half_away(v: np.ndarray) -> np.ndarray:
    """f64::round: half away from zero.  The fraction d - trunc(d) is exact, so
    this does not round 0.49999999999999994 up as trunc(d + 0.5) would."""
    d = np.asarray(v, np.float64)
    t = np.trunc(d)
    with np.errstate(invalid="ignore"):
        up = np.abs(d - t) >= 0.5
    return t + np.where(up, np.sign(d), 0.0)


def narrow(values: np.ndarray, dtype: DType) -> np.ndarray:
    """push_field (voxel.rs:1241-1259): round() then a saturating cast for integer fields."""
    if dtype in (DType.F32, DType.F16):
        return values.astype(np.float32)
    if dtype == DType.F64:
        return values.astype(np.float32).astype(np.float64)
    info = np.iinfo(dtype.numpy)
    r = _round_half_away(values)
    r = np.where(np.isnan(r), 0.0, np.clip(r, info.min, info.max))
    return r.astype(dtype.numpy)


def is_plain_xyz_f32_schema(schema) -> bool:
    """voxel.rs:670-688: exactly three fields, F32 or F16, the three positions."""
    fields = list(schema.fields)
    return (len(fields) == 3 and all(f.dtype in (DType.F32, DType.F16) for f in fields)
            and {f.semantic for f in fields} == set(POSITION_SEMANTICS))


def uses_plain_xyz_path(schema, config: "VoxelGridDownsampleConfig") -> bool:
    """Whether the reference's CPU dispatch (voxel.rs:314-330 -> 474-485) takes
    filter_cpu_xyz_centroid_fast: Centroid + Average on a plain-xyz cloud.
    The CUDA arm follows it (SRCU_VOXEL_CENTROID_XYZ): f32 sums, first-seen
    voxel order."""
    return (config.mode == VoxelAggregationMode.Centroid
            and config.attribute_policy == AttributeAggregation.Average
            and is_plain_xyz_f32_schema(schema))


class VoxelGridDownsample:
    """Voxel-grid downsampling filter (voxel.rs:185-248)."""

    def __init__(self, config: VoxelGridDownsampleConfig, device: int = 0):
        self._config = config
        self._device = device

    def config(self) -> VoxelGridDownsampleConfig:
        return self._config

    def name(self) -> str:
        return "VoxelGridDownsample"

    def filter(self, input: PointCloud) -> PointCloud:
        """PointCloudFilter::filter.  The reference runs CpuSingle here; this
        package's only backend is CUDA, so it runs Gpu(Cuda)."""
        return self.filter_with_policy(input, ExecutionPolicy.gpu(DeviceKind.Cuda))

    def filter_with_policy(self, input: PointCloud, policy: ExecutionPolicy) -> PointCloud:
        return self.filter_with_policy_and_receipt(input, policy).into_output()

    def filter_with_policy_and_receipt(self, input: PointCloud,
                                       policy: ExecutionPolicy) -> ExecutionOutput:
        resolved = resolve_cuda_policy(policy, "voxel downsampling")
        receipt = ExecutionReceipt(policy, resolved)
        output = self._filter_cuda(input, receipt)
        receipt.stages.insert(0, "voxel-downsample")
        return ExecutionOutput(output, receipt)

    def _filter_cuda(self, input: PointCloud, receipt: ExecutionReceipt) -> PointCloud:
        cfg = self._config
        if input.is_empty():
            return input.clone()
        if cfg.leaf_size <= 0.0:
            raise InvalidArgument("leaf_size must be greater than zero")
        x, y, z = input.positions3()
        attr_fields = [f for f in input.schema.fields if f.semantic not in POSITION_SEMANTICS]
        attrs = [_widen(input.columns[f.name]) for f in attr_fields]
        ctx = _native.shared_context(self._device)
        cols, _, _ = ctx.voxel_centroid(
            x, y, z, attrs, leaf=cfg.leaf_size, origin=cfg.origin,
            approximate=cfg.mode == VoxelAggregationMode.ApproximateFirst,
            attribute_first=cfg.attribute_policy == AttributeAggregation.First,
            plain_xyz=uses_plain_xyz_path(input.schema, cfg))
        out = {}
        pos_names = {f.semantic: f.name for f in input.schema.fields if f.semantic in POSITION_SEMANTICS}
        out[pos_names[FieldSemantic.PositionX]] = cols[0]
        out[pos_names[FieldSemantic.PositionY]] = cols[1]
        out[pos_names[FieldSemantic.PositionZ]] = cols[2]
        for f, c in zip(attr_fields, cols[3:]):
            out[f.name] = narrow(c, f.dtype)
        n, v = len(input), cols[0].shape[0]
        receipt.record_transfer(TransferDirection.HostToDevice, n * 4 * (3 + len(attrs)))
        receipt.record_transfer(TransferDirection.DeviceToHost, v * 4 * (3 + len(attrs)))
        receipt.record_stage("gpu-readback")
        return PointCloud(input.schema, out, input.metadata)
