"""Point-cloud data model, execution policy and errors, mirroring spatialrust-core.

Only what the uniform-grid path needs: SoA columns with a schema
(crates/spatialrust-core/src/pointcloud.rs, schema.rs), the
ExecutionPolicy / DeviceKind / ExecutionReceipt contract (execution.rs,
device.rs) and the SpatialError variants (error.rs:8-37).
"""
from __future__ import annotations

import enum
from dataclasses import dataclass, field
from typing import Dict, List, Optional, Sequence

import numpy as np


# ---- errors (crates/spatialrust-core/src/error.rs:8-37) ----------------------

class SpatialError(Exception):
    """Base of every error this package raises."""


class MissingField(SpatialError):
    pass


class SchemaValidation(SpatialError):
    pass


class InvalidArgument(SpatialError):
    pass


class BufferLengthMismatch(SpatialError):
    pass


class UnsupportedDType(SpatialError):
    pass


# ---- schema (crates/spatialrust-core/src/schema.rs) --------------------------

class DType(enum.Enum):
    F32 = "f32"
    F64 = "f64"
    F16 = "f16"
    U8 = "u8"
    U16 = "u16"
    U32 = "u32"
    I32 = "i32"

    @property
    def numpy(self):
        return {DType.F32: np.float32, DType.F64: np.float64, DType.F16: np.float32,
                DType.U8: np.uint8, DType.U16: np.uint16, DType.U32: np.uint32,
                DType.I32: np.int32}[self]


class FieldSemantic(enum.Enum):
    PositionX = "position_x"
    PositionY = "position_y"
    PositionZ = "position_z"
    Intensity = "intensity"
    NormalX = "normal_x"
    NormalY = "normal_y"
    NormalZ = "normal_z"
    Curvature = "curvature"
    ColorR = "r"
    ColorG = "g"
    ColorB = "b"
    Label = "label"
    TimeOffset = "time_offset"
    Custom = "custom"


POSITION_SEMANTICS = (FieldSemantic.PositionX, FieldSemantic.PositionY, FieldSemantic.PositionZ)


@dataclass(frozen=True)
class PointField:
    name: str
    semantic: FieldSemantic
    dtype: DType

    @staticmethod
    def scalar(name: str, semantic: FieldSemantic, dtype: DType) -> "PointField":
        return PointField(name, semantic, dtype)


@dataclass(frozen=True)
class PointSchema:
    fields: tuple = ()

    def with_field(self, f: PointField) -> "PointSchema":
        return PointSchema(self.fields + (f,))

    def find_semantic(self, semantic: FieldSemantic) -> Optional[PointField]:
        for f in self.fields:
            if f.semantic == semantic:
                return f
        return None

    def names(self) -> List[str]:
        return [f.name for f in self.fields]

    def __len__(self):
        return len(self.fields)


class StandardSchemas:
    """StandardSchemas (schema.rs:170-214)."""

    @staticmethod
    def point_xyz() -> PointSchema:
        return (PointSchema()
                .with_field(PointField.scalar("x", FieldSemantic.PositionX, DType.F32))
                .with_field(PointField.scalar("y", FieldSemantic.PositionY, DType.F32))
                .with_field(PointField.scalar("z", FieldSemantic.PositionZ, DType.F32)))

    @staticmethod
    def point_xyzi() -> PointSchema:
        return StandardSchemas.point_xyz().with_field(
            PointField.scalar("intensity", FieldSemantic.Intensity, DType.F32))

    @staticmethod
    def point_xyzrgb() -> PointSchema:
        return (StandardSchemas.point_xyz()
                .with_field(PointField.scalar("r", FieldSemantic.ColorR, DType.U8))
                .with_field(PointField.scalar("g", FieldSemantic.ColorG, DType.U8))
                .with_field(PointField.scalar("b", FieldSemantic.ColorB, DType.U8)))

    @staticmethod
    def point_xyzinormal() -> PointSchema:
        return (StandardSchemas.point_xyzi()
                .with_field(PointField.scalar("normal_x", FieldSemantic.NormalX, DType.F32))
                .with_field(PointField.scalar("normal_y", FieldSemantic.NormalY, DType.F32))
                .with_field(PointField.scalar("normal_z", FieldSemantic.NormalZ, DType.F32)))


# ---- point cloud (crates/spatialrust-core/src/pointcloud.rs) -----------------

class PointCloud:
    """Columnar point cloud: one numpy column per schema field, plus metadata."""

    def __init__(self, schema: PointSchema, columns: Dict[str, np.ndarray],
                 metadata: Optional[dict] = None):
        n = None
        cols = {}
        for f in schema.fields:
            if f.name not in columns:
                raise MissingField(f.name)
            c = np.ascontiguousarray(columns[f.name], dtype=f.dtype.numpy)
            if n is None:
                n = c.shape[0]
            elif c.shape[0] != n:
                raise BufferLengthMismatch(f"expected {n}, found {c.shape[0]}")
            cols[f.name] = c
        self.schema = schema
        self.columns = cols
        self.metadata = dict(metadata or {})
        self._len = int(n or 0)

    @staticmethod
    def from_columns(schema: PointSchema, **columns) -> "PointCloud":
        return PointCloud(schema, columns)

    def __len__(self):
        return self._len

    def is_empty(self) -> bool:
        return self._len == 0

    def field(self, name: str) -> np.ndarray:
        if name not in self.columns:
            raise MissingField(name)
        return self.columns[name]

    def positions3(self):
        """HasPositions3::positions3 (capabilities.rs:22-29): F32 x, y, z columns."""
        out = []
        for sem in POSITION_SEMANTICS:
            f = self.schema.find_semantic(sem)
            if f is None:
                raise MissingField(sem.value)
            if f.dtype not in (DType.F32, DType.F16):
                raise UnsupportedDType(f.dtype)
            out.append(self.columns[f.name])
        return tuple(out)

    def normals3(self):
        out = []
        for sem in (FieldSemantic.NormalX, FieldSemantic.NormalY, FieldSemantic.NormalZ):
            f = self.schema.find_semantic(sem)
            if f is None:
                raise MissingField(sem.value)
            out.append(self.columns[f.name])
        return tuple(out)

    def intensity(self) -> np.ndarray:
        f = self.schema.find_semantic(FieldSemantic.Intensity)
        if f is None:
            raise MissingField("intensity")
        return self.columns[f.name]

    def clone(self) -> "PointCloud":
        return PointCloud(self.schema, {k: v.copy() for k, v in self.columns.items()},
                          self.metadata)

    def __eq__(self, other):
        if not isinstance(other, PointCloud):
            return NotImplemented
        return (self.schema == other.schema and self.metadata == other.metadata
                and all(np.array_equal(self.columns[k], other.columns[k], equal_nan=True)
                        for k in self.columns))


class PointCloudBuilder:
    """PointCloudBuilder: push rows of field values in schema order."""

    def __init__(self, schema: PointSchema):
        self.schema = schema
        self.rows: List[Sequence[float]] = []

    @staticmethod
    def xyz() -> "PointCloudBuilder":
        return PointCloudBuilder(StandardSchemas.point_xyz())

    def push_point(self, values: Sequence[float]) -> "PointCloudBuilder":
        if len(values) != len(self.schema):
            raise BufferLengthMismatch(f"expected {len(self.schema)}, found {len(values)}")
        self.rows.append(tuple(values))
        return self

    def build(self) -> PointCloud:
        cols = {}
        for i, f in enumerate(self.schema.fields):
            cols[f.name] = np.array([r[i] for r in self.rows], dtype=f.dtype.numpy)
        return PointCloud(self.schema, cols)


# ---- execution policy (execution.rs, device.rs) -------------------------------

class DeviceKind(enum.Enum):
    Cpu = "cpu"
    Wgpu = "wgpu"
    Cuda = "cuda"

    def is_gpu(self) -> bool:
        return self in (DeviceKind.Wgpu, DeviceKind.Cuda)


@dataclass(frozen=True)
class ExecutionPolicy:
    """ExecutionPolicy::{CpuSingle, CpuParallel, Gpu(DeviceKind), Auto}."""

    kind: str
    device: Optional[DeviceKind] = None

    @staticmethod
    def cpu_single() -> "ExecutionPolicy":
        return ExecutionPolicy("cpu_single")

    @staticmethod
    def cpu_parallel() -> "ExecutionPolicy":
        return ExecutionPolicy("cpu_parallel")

    @staticmethod
    def gpu(device: DeviceKind) -> "ExecutionPolicy":
        return ExecutionPolicy("gpu", device)

    @staticmethod
    def auto() -> "ExecutionPolicy":
        return ExecutionPolicy("auto")

    def validate(self):
        """execution.rs:19-26"""
        if self.kind == "gpu" and self.device == DeviceKind.Cpu:
            raise InvalidArgument("GPU execution policy cannot target the CPU device")

    def requests_gpu(self) -> bool:
        return self.kind == "gpu" and self.device is not None and self.device.is_gpu()

    def allows_fallback(self) -> bool:
        return self.kind == "auto"

    def __repr__(self):
        return f"Gpu({self.device.name})" if self.kind == "gpu" else self.kind


CpuSingle = ExecutionPolicy.cpu_single()
CpuParallel = ExecutionPolicy.cpu_parallel()
Auto = ExecutionPolicy.auto()
GpuCuda = ExecutionPolicy.gpu(DeviceKind.Cuda)


class TransferDirection(enum.Enum):
    HostToDevice = "h2d"
    DeviceToDevice = "d2d"
    DeviceToHost = "d2h"


@dataclass
class ExecutionReceipt:
    """ExecutionReceipt (execution.rs:69-143): policies, stages, transfer bytes."""

    requested_policy: ExecutionPolicy
    resolved_policy: ExecutionPolicy
    stages: List[str] = field(default_factory=list)
    transfers: Dict[TransferDirection, int] = field(default_factory=dict)

    def record_stage(self, name: str):
        self.stages.append(name)

    def record_transfer(self, direction: TransferDirection, nbytes: int):
        self.transfers[direction] = self.transfers.get(direction, 0) + int(nbytes)


@dataclass
class ExecutionOutput:
    output: object
    receipt: ExecutionReceipt

    def into_output(self):
        return self.output
