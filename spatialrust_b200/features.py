"""Radius-mode normal estimation with the ExecutionPolicy::Gpu(DeviceKind::Cuda) arm.

Mirrors crates/spatialrust-features/src/normal.rs (NormalEstimationConfig
:17-71, NormalEstimator :84-308, build_output_cloud :575-599) and
normal_gpu.rs (GpuNormalEstimator :15-83).  NormalEstimator keeps the CPU
semantics of the reference (query excluded from its own neighbourhood, NaN
normal below min_neighbors); GpuNormalEstimator keeps the wgpu grid semantics
(query included, fewer than 3 points -> (0, 0, 1), normals_grid.rs:86-197).
"""
from __future__ import annotations

from dataclasses import dataclass, replace
from typing import Optional, Tuple

import numpy as np

from . import _native
from .core import (DType, ExecutionOutput, ExecutionPolicy, ExecutionReceipt, FieldSemantic,
                   InvalidArgument, PointCloud, PointField, TransferDirection)
from .filtering import resolve_cuda_policy

DEFAULT_GPU_MIN_POINTS_NORMAL = 10_000


@dataclass(frozen=True)
class NormalEstimationConfig:
    k_neighbors: int = 20
    search_radius: Optional[float] = None
    min_neighbors: int = 3
    viewpoint: Optional[Tuple[float, float, float]] = None
    gpu_min_points: Optional[int] = DEFAULT_GPU_MIN_POINTS_NORMAL

    @staticmethod
    def radius(search_radius: float, **kw) -> "NormalEstimationConfig":
        return NormalEstimationConfig(search_radius=float(search_radius), **kw)

    def without_gpu_min_points(self) -> "NormalEstimationConfig":
        return replace(self, gpu_min_points=None)


@dataclass
class NormalEstimationResult:
    valid_count: int = 0
    invalid_count: int = 0
    shell_points: int = 0
    fp64_eigensolves: int = 0


def _ensure_field(schema, name, semantic):
    if schema.find_semantic(semantic) is None:
        schema = schema.with_field(PointField.scalar(name, semantic, DType.F32))
    return schema


def build_output_cloud(input: PointCloud, nx, ny, nz, curvature) -> PointCloud:
    """build_output_cloud (normal.rs:575-599): input columns + normal_x/y/z, curvature."""
    schema = input.schema
    for name, sem in (("normal_x", FieldSemantic.NormalX), ("normal_y", FieldSemantic.NormalY),
                      ("normal_z", FieldSemantic.NormalZ), ("curvature", FieldSemantic.Curvature)):
        schema = _ensure_field(schema, name, sem)
    cols = {k: v.copy() for k, v in input.columns.items()}
    cols["normal_x"] = np.asarray(nx, np.float32)
    cols["normal_y"] = np.asarray(ny, np.float32)
    cols["normal_z"] = np.asarray(nz, np.float32)
    cols["curvature"] = np.asarray(curvature, np.float32)
    # a schema that already had the semantics under other names keeps them
    for f in schema.fields:
        if f.semantic in (FieldSemantic.NormalX, FieldSemantic.NormalY, FieldSemantic.NormalZ,
                          FieldSemantic.Curvature) and f.name not in ("normal_x", "normal_y",
                                                                       "normal_z", "curvature"):
            cols[f.name] = cols[{FieldSemantic.NormalX: "normal_x", FieldSemantic.NormalY: "normal_y",
                                 FieldSemantic.NormalZ: "normal_z",
                                 FieldSemantic.Curvature: "curvature"}[f.semantic]]
    return PointCloud(schema, cols, input.metadata)


class NormalEstimator:
    """Covariance-based normal estimator, radius mode on CUDA."""

    def __init__(self, config: NormalEstimationConfig, device: int = 0):
        self._config = config
        self._device = device

    def config(self) -> NormalEstimationConfig:
        return self._config

    def name(self) -> str:
        return "NormalEstimator"

    def _run(self, input: PointCloud, include_self: bool):
        cfg = self._config
        if cfg.search_radius is None:
            raise InvalidArgument(
                "the CUDA arm implements radius-mode normal estimation; set search_radius")
        if cfg.search_radius < 0.0:
            raise InvalidArgument("search_radius must be non-negative")
        x, y, z = input.positions3()
        ctx = _native.shared_context(self._device)
        nx, ny, nz, curv, counts, stats = ctx.radius_normals(
            x, y, z, cfg.search_radius, cfg.min_neighbors, cfg.viewpoint, include_self)
        result = NormalEstimationResult(stats["valid_count"], stats["invalid_count"],
                                        stats["shell_points"], stats["fp64_eigensolves"])
        return build_output_cloud(input, nx, ny, nz, curv), result, counts

    def estimate_with_diagnostics(self, input: PointCloud):
        """normal.rs:102-164 on the CUDA arm: (cloud, NormalEstimationResult)."""
        if input.is_empty():
            return input.clone(), NormalEstimationResult()
        cloud, result, _ = self._run(input, include_self=False)
        return cloud, result

    def estimate(self, input: PointCloud) -> PointCloud:
        return self.estimate_with_diagnostics(input)[0]

    def estimate_with_policy(self, input: PointCloud, policy: ExecutionPolicy) -> PointCloud:
        return self.estimate_with_policy_and_receipt(input, policy).into_output()

    def estimate_with_policy_and_receipt(self, input: PointCloud,
                                         policy: ExecutionPolicy) -> ExecutionOutput:
        resolved = resolve_cuda_policy(policy, "normal estimation")
        receipt = ExecutionReceipt(policy, resolved)
        receipt.record_stage("normal-estimation")
        output = self.estimate(input)
        n = len(input)
        receipt.record_transfer(TransferDirection.HostToDevice, n * 12)
        receipt.record_transfer(TransferDirection.DeviceToHost, len(output) * 16)
        receipt.record_stage("gpu-readback")
        return ExecutionOutput(output, receipt)


class GpuNormalEstimator:
    """GpuNormalEstimator (normal_gpu.rs:15-83), radius mode on CUDA with the
    grid kernel's semantics: the query point counts toward its own
    neighbourhood and fewer than 3 points give (0, 0, 1) with curvature 0."""

    def __init__(self, config: NormalEstimationConfig, device: int = 0):
        self._config = config
        self._inner = NormalEstimator(config, device)

    def config(self) -> NormalEstimationConfig:
        return self._config

    def estimate(self, input: PointCloud) -> PointCloud:
        if input.is_empty():
            return input.clone()
        return self._inner._run(input, include_self=True)[0]
