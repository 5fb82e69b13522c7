"""Bounded streaming voxel centroids on the CUDA library.

Mirrors crates/spatialrust-pipeline/src/streaming.rs (StreamingVoxelConfig
:334-390, StreamingVoxelSource :392-676) and the spool contract it is
configured with (SpoolOptions, crates/spatialrust-io/src/spool.rs:12-47).
The points never gather on the host: every chunk goes to the device, where
runs are sorted and reduced (srcu_stream_voxel_*, include/srcuda.h); the
reduced runs held in device memory take the place of the disk spool, whose
size and run-count limits are still enforced exactly as the reference
computes them.

A source is anything with ``next_chunk() -> PointCloud | None`` (and
optionally ``chunk_points``), or any iterable of PointClouds; MemoryChunkSource
plays the part of RecyclingMemoryChunkSource in the reference's tests.
"""
from __future__ import annotations

import itertools
import os
from dataclasses import dataclass
from typing import Iterable, Optional

import numpy as np

from . import _native
from .core import (DType, MissingField, PointCloud, SpatialError, UnsupportedDType,
                   POSITION_SEMANTICS)
from .filtering import _round_half_away

DEFAULT_CHUNK_POINTS = 65_536


class RecordsError(SpatialError):
    """RecordsError (spatialrust-records): invalid configuration or chunk."""


@dataclass(frozen=True)
class SpoolOptions:
    """SpoolOptions::new (spool.rs:21-33): a directory and a byte limit."""

    directory: str
    limit_bytes: int

    def __post_init__(self):
        if self.limit_bytes == 0:
            raise RecordsError("spool limit must be positive")
        if not os.path.isdir(self.directory):
            raise RecordsError(f"spool directory does not exist: {self.directory}")


class StreamingVoxelConfig:
    """StreamingVoxelConfig::new (streaming.rs:345-363)."""

    def __init__(self, leaf_size: float, run_points: int, max_runs: int, spool: SpoolOptions):
        leaf = float(np.float32(leaf_size))
        if not np.isfinite(leaf) or leaf <= 0.0:
            raise RecordsError("streaming voxel leaf size must be positive and finite")
        if run_points == 0 or max_runs == 0:
            raise RecordsError("streaming voxel run_points and max_runs must be positive")
        self._leaf = leaf
        self._run_points = int(run_points)
        self._max_runs = int(max_runs)
        self._spool = spool

    def leaf_size(self) -> float:
        return self._leaf

    def run_points(self) -> int:
        return self._run_points

    def max_runs(self) -> int:
        return self._max_runs

    def spool(self) -> SpoolOptions:
        return self._spool


class MemoryChunkSource:
    """A cloud served as consecutive chunks of chunk_points points."""

    def __init__(self, cloud: PointCloud, chunk_points: int):
        if chunk_points <= 0:
            raise RecordsError("chunk_points must be positive")
        self.cloud = cloud
        self.schema = cloud.schema
        self.chunk_points = int(chunk_points)
        self._next = 0

    def next_chunk(self) -> Optional[PointCloud]:
        n = len(self.cloud)
        if self._next >= n:
            return None
        lo, hi = self._next, min(n, self._next + self.chunk_points)
        self._next = hi
        return PointCloud(self.schema, {k: v[lo:hi] for k, v in self.cloud.columns.items()},
                          self.cloud.metadata)


def _chunks(source) -> Iterable[PointCloud]:
    if hasattr(source, "next_chunk"):
        while True:
            c = source.next_chunk()
            if c is None:
                return
            yield c
    else:
        yield from source


def push_scalar(values: np.ndarray, dtype: DType) -> np.ndarray:
    """push_scalar (streaming.rs:922-938): as f32 / f64, or round() then clamp
    into the integer type."""
    if dtype in (DType.F32, DType.F16):
        return values.astype(np.float32)
    if dtype == DType.F64:
        return values.astype(np.float64)
    info = np.iinfo(dtype.numpy)
    lo = 0 if dtype in (DType.U8, DType.U16, DType.U32) else info.min
    r = np.clip(_round_half_away(values), lo, info.max)
    return np.where(np.isnan(r), 0, r).astype(dtype.numpy)


# columns averaged in FP64 on the device: f32 cannot carry them exactly
_F64_DTYPES = (DType.F64, DType.U32, DType.I32)


class StreamingVoxelSource:
    """Bounded source of globally aggregated voxel centroids (streaming.rs:392-676)."""

    def __init__(self, schema, fields, sv: "_native.StreamVoxel", metadata, chunk_points: int):
        self.schema = schema
        self._fields = fields  # attribute fields, in schema order
        self._sv = sv
        self.metadata = metadata
        self.chunk_points = chunk_points
        self._next = 0
        self._info = sv.info

    @staticmethod
    def try_build(source, config: StreamingVoxelConfig, device: int = 0) -> "StreamingVoxelSource":
        chunks = _chunks(source)
        schema = getattr(source, "schema", None)
        first = None
        if schema is None:
            first = next(chunks, None)
            schema = first.schema if first is not None else None
        if schema is None:
            raise RecordsError("the stream has no schema")
        pos_fields = []
        for sem in POSITION_SEMANTICS:
            f = schema.find_semantic(sem)
            if f is None:  # positions() (streaming.rs:860-880)
                raise MissingField(sem.value)
            if f.dtype not in (DType.F32, DType.F16):
                raise UnsupportedDType(f.dtype)
            pos_fields.append(f)
        attrs = [f for f in schema.fields if f not in pos_fields]
        ctx = _native.shared_context(device)
        sv = _native.StreamVoxel(ctx, config.leaf_size(), [f.dtype in _F64_DTYPES for f in attrs],
                                 config.run_points(), config.max_runs(), config.spool().limit_bytes)
        metadata = None
        try:
            for c in itertools.chain([first] if first is not None else [], chunks):
                if metadata is None:
                    metadata = c.metadata
                sv.push(*[c.columns[f.name] for f in pos_fields],
                        [c.columns[f.name] for f in attrs])
            sv.finish()
        except Exception:
            sv.close()
            raise
        chunk_points = int(getattr(source, "chunk_points", DEFAULT_CHUNK_POINTS))
        return StreamingVoxelSource(schema, (pos_fields, attrs), sv, metadata or {}, chunk_points)

    def run_count(self) -> int:
        """Runs the reference's spill would hold: ceil(finite points / run_points)."""
        return self._info["runs"]

    def spool_bytes(self) -> int:
        """The reference's spool extent for those runs."""
        return self._info["spool_bytes"]

    def info(self) -> dict:
        return dict(self._info)

    def next_chunk(self) -> Optional[PointCloud]:
        total = self._info["voxels"]
        if self._next >= total:
            return None
        count = min(self.chunk_points, total - self._next)
        x, y, z, a, _, _ = self._sv.fetch(self._next, count)
        self._next += count
        pos_fields, attrs = self._fields
        cols = {pos_fields[0].name: x, pos_fields[1].name: y, pos_fields[2].name: z}
        for i, f in enumerate(attrs):
            cols[f.name] = push_scalar(a[:, i], f.dtype)
        return PointCloud(self.schema, cols, self.metadata)

    def keys_and_counts(self):
        """(ix, iy, iz) and point count of every voxel, in output order."""
        _, _, _, _, keys, counts = self._sv.fetch(0, self._info["voxels"])
        return keys, counts

    def close(self):
        self._sv.close()
