"""ctypes binding of libsrcuda.so (the C ABI declared in include/srcuda.h).

The CUDA library is the product path: there is no CPU fallback.  Importing this
module fails loudly when libsrcuda.so is missing.
"""
from __future__ import annotations

import ctypes
import os
from typing import Sequence

import numpy as np

from .core import (BufferLengthMismatch, InvalidArgument, MissingField, SpatialError,
                   UnsupportedDType)

_LIB_PATH = os.path.join(os.path.dirname(os.path.abspath(__file__)), "libsrcuda.so")

SRCU_OK = 0
SRCU_ERR_INVALID_ARGUMENT = 1
SRCU_ERR_LENGTH_MISMATCH = 2
SRCU_ERR_UNSUPPORTED_DTYPE = 3
SRCU_ERR_MISSING_FIELD = 4
SRCU_ERR_OUT_OF_BUDGET = 5
SRCU_ERR_CUDA = 6
SRCU_ERR_TIMEOUT = 7
SRCU_ERR_KEY_OVERFLOW = 8
SRCU_ERR_NO_DEVICE = 9
SRCU_ERR_BUSY = 10

STATUS_NAMES = {
    SRCU_OK: "SRCU_OK",
    SRCU_ERR_INVALID_ARGUMENT: "SRCU_ERR_INVALID_ARGUMENT",
    SRCU_ERR_LENGTH_MISMATCH: "SRCU_ERR_LENGTH_MISMATCH",
    SRCU_ERR_UNSUPPORTED_DTYPE: "SRCU_ERR_UNSUPPORTED_DTYPE",
    SRCU_ERR_MISSING_FIELD: "SRCU_ERR_MISSING_FIELD",
    SRCU_ERR_OUT_OF_BUDGET: "SRCU_ERR_OUT_OF_BUDGET",
    SRCU_ERR_CUDA: "SRCU_ERR_CUDA",
    SRCU_ERR_TIMEOUT: "SRCU_ERR_TIMEOUT",
    SRCU_ERR_KEY_OVERFLOW: "SRCU_ERR_KEY_OVERFLOW",
    SRCU_ERR_NO_DEVICE: "SRCU_ERR_NO_DEVICE",
    SRCU_ERR_BUSY: "SRCU_ERR_BUSY",
}

MAX_ATTRS = 9


class CudaError(SpatialError):
    """A CUDA-side failure (maps to SpatialError::InvalidArgument text in the reference)."""

    def __init__(self, status: int, message: str):
        super().__init__(f"{STATUS_NAMES.get(status, status)}: {message}")
        self.status = status


class OutOfBudget(CudaError):
    pass


class DeviceTimeout(CudaError):
    pass


class KeyOverflow(CudaError):
    pass


class NoDevice(CudaError):
    pass


c_float3 = ctypes.c_float * 3


class SrcuCloud(ctypes.Structure):
    _fields_ = [("x", ctypes.c_void_p), ("y", ctypes.c_void_p), ("z", ctypes.c_void_p),
                ("attrs", ctypes.c_void_p), ("n_attrs", ctypes.c_uint32),
                ("on_device", ctypes.c_int32), ("n", ctypes.c_uint64),
                ("stride", ctypes.c_uint32), ("reserved", ctypes.c_uint32)]


SRCU_VOXEL_CENTROID = 0
SRCU_VOXEL_APPROXIMATE_FIRST = 1
SRCU_VOXEL_CENTROID_XYZ = 2  # the reference's plain-xyz fast path (voxel.rs:550-636)
SRCU_ATTRIBUTE_AVERAGE = 0
SRCU_ATTRIBUTE_FIRST = 1


class SrcuVoxelParams(ctypes.Structure):
    _fields_ = [("leaf_size", ctypes.c_float), ("has_origin", ctypes.c_int32),
                ("origin", c_float3), ("mode", ctypes.c_int32), ("attribute_policy", ctypes.c_int32)]


class SrcuVoxelOut(ctypes.Structure):
    _fields_ = [("x", ctypes.c_void_p), ("y", ctypes.c_void_p), ("z", ctypes.c_void_p),
                ("attrs", ctypes.c_void_p), ("keys", ctypes.c_void_p), ("counts", ctypes.c_void_p),
                ("on_device", ctypes.c_int32)]


class SrcuNormalParams(ctypes.Structure):
    _fields_ = [("radius", ctypes.c_float), ("min_neighbors", ctypes.c_uint32),
                ("has_viewpoint", ctypes.c_int32), ("viewpoint", c_float3),
                ("include_self", ctypes.c_int32), ("count_shell", ctypes.c_int32)]


class SrcuNormalOut(ctypes.Structure):
    _fields_ = [("nx", ctypes.c_void_p), ("ny", ctypes.c_void_p), ("nz", ctypes.c_void_p),
                ("curvature", ctypes.c_void_p), ("neighbor_counts", ctypes.c_void_p),
                ("on_device", ctypes.c_int32)]


class SrcuNormalStats(ctypes.Structure):
    _fields_ = [("valid_count", ctypes.c_uint64), ("invalid_count", ctypes.c_uint64),
                ("shell_points", ctypes.c_uint64), ("fp64_eigensolves", ctypes.c_uint64)]


class SrcuFrameView(ctypes.Structure):
    _fields_ = [("x", ctypes.c_void_p), ("y", ctypes.c_void_p), ("z", ctypes.c_void_p),
                ("attrs", ctypes.c_void_p), ("nx", ctypes.c_void_p), ("ny", ctypes.c_void_p),
                ("nz", ctypes.c_void_p), ("curvature", ctypes.c_void_p),
                ("counts", ctypes.c_void_p), ("voxel_count", ctypes.c_void_p),
                ("n_attrs", ctypes.c_uint32)]


class SrcuChainInfo(ctypes.Structure):
    _fields_ = [("points", ctypes.c_uint64), ("voxels", ctypes.c_uint64), ("cells", ctypes.c_uint64),
                ("voxel_key_bits", ctypes.c_uint32), ("cell_key_bits", ctypes.c_uint32),
                ("voxel_sort_passes", ctypes.c_uint32), ("cell_sort_passes", ctypes.c_uint32),
                ("cell_size", ctypes.c_double)]


class SrcuKernelStat(ctypes.Structure):
    _fields_ = [("name", ctypes.c_char * 32), ("launches", ctypes.c_uint64),
                ("timed_regions", ctypes.c_uint64), ("total_ms", ctypes.c_double)]


class SrcuServerConfig(ctypes.Structure):
    _fields_ = [("device", ctypes.c_int), ("hbm_budget_bytes", ctypes.c_uint64),
                ("frame_slots", ctypes.c_uint32), ("bulk_slots", ctypes.c_uint32),
                ("frame_batch_points", ctypes.c_uint64), ("bulk_threshold_points", ctypes.c_uint64),
                ("bulk_max_points", ctypes.c_uint64), ("max_pending_points", ctypes.c_uint64),
                ("host_arena_bytes", ctypes.c_uint64)]


class SrcuRequestResult(ctypes.Structure):
    _fields_ = [("req_id", ctypes.c_uint64), ("status", ctypes.c_int), ("points", ctypes.c_uint64),
                ("voxels", ctypes.c_uint64), ("x", ctypes.c_void_p), ("y", ctypes.c_void_p),
                ("z", ctypes.c_void_p), ("intensity", ctypes.c_void_p), ("nx", ctypes.c_void_p),
                ("ny", ctypes.c_void_p), ("nz", ctypes.c_void_p), ("curvature", ctypes.c_void_p),
                ("counts", ctypes.c_void_p), ("latency_ms", ctypes.c_double)]


class SrcuServerStats(ctypes.Structure):
    _fields_ = [(k, ctypes.c_uint64) for k in
                ("submitted", "rejected", "completed", "failed", "batches", "points")] + [
                (k, ctypes.c_double) for k in
                ("frame_p50_ms", "frame_p99_ms", "bulk_p50_ms", "bulk_p99_ms", "all_p50_ms",
                 "all_p99_ms", "elapsed_s")]


class SrcuStreamVoxelParams(ctypes.Structure):
    _fields_ = [("leaf_size", ctypes.c_float), ("n_attrs", ctypes.c_uint32),
                ("attr_f64_mask", ctypes.c_uint32), ("device_run_points", ctypes.c_uint32),
                ("run_points", ctypes.c_uint64), ("max_runs", ctypes.c_uint64),
                ("spool_limit_bytes", ctypes.c_uint64)]


class SrcuStreamVoxelInfo(ctypes.Structure):
    _fields_ = [(k, ctypes.c_uint64) for k in
                ("points", "finite_points", "runs", "spool_bytes", "device_runs",
                 "partial_records", "voxels")]


class SrcuStreamVoxelOut(ctypes.Structure):
    _fields_ = [("x", ctypes.c_void_p), ("y", ctypes.c_void_p), ("z", ctypes.c_void_p),
                ("attrs", ctypes.c_void_p), ("keys", ctypes.c_void_p), ("counts", ctypes.c_void_p),
                ("on_device", ctypes.c_int32)]


class SrcuLasFormat(ctypes.Structure):
    _fields_ = [("point_format", ctypes.c_uint32), ("record_length", ctypes.c_uint32),
                ("scale", ctypes.c_double * 3), ("offset", ctypes.c_double * 3),
                ("has_origin", ctypes.c_int32), ("reserved", ctypes.c_int32),
                ("origin", ctypes.c_double * 3)]


class SrcuLasOut(ctypes.Structure):
    _fields_ = [(k, ctypes.c_void_p) for k in
                ("x", "y", "z", "intensity", "classification", "gps_time", "red", "green", "blue")] + [
                ("on_device", ctypes.c_int32)]


class SrcuPlaneScore(ctypes.Structure):
    _fields_ = [("inlier_count", ctypes.c_uint32), ("normal", ctypes.c_float * 3),
                ("d", ctypes.c_float)]


class SrcuRansacParams(ctypes.Structure):
    _fields_ = [("distance_threshold", ctypes.c_float), ("max_iterations", ctypes.c_uint32),
                ("min_inliers", ctypes.c_uint64), ("seed", ctypes.c_uint64)]


class SrcuRansacResult(ctypes.Structure):
    _fields_ = [("normal", ctypes.c_float * 3), ("d", ctypes.c_float),
                ("inlier_count", ctypes.c_uint64), ("hypotheses", ctypes.c_uint32),
                ("best_hypothesis", ctypes.c_uint32), ("hypothesis_normal", ctypes.c_float * 3),
                ("hypothesis_d", ctypes.c_float)]


KERNEL_IDS = ["begin", "bounds", "voxel_plan", "voxel_hist", "voxel_sort", "voxel_segments",
              "unpack_keys", "cell_plan", "cell_hist", "cell_sort", "cells", "hash", "ranges",
              "normals", "cluster", "las_decode", "ransac"]


# Every symbol include/srcuda.h declares, with its ctypes signature.
_P = ctypes.c_void_p
SIGNATURES = {
    "srcu_abi_version": ([], ctypes.c_int),
    "srcu_create": ([ctypes.c_int, ctypes.c_uint64, ctypes.POINTER(ctypes.c_void_p)], ctypes.c_int),
    "srcu_destroy": ([_P], None),
    "srcu_last_error": ([_P], ctypes.c_char_p),
    "srcu_set_stream": ([_P, _P], ctypes.c_int),
    "srcu_synchronize": ([_P], ctypes.c_int),
    "srcu_device_bytes": ([_P], ctypes.c_uint64),
    "srcu_voxel_centroid": ([_P, ctypes.POINTER(SrcuCloud), ctypes.POINTER(SrcuVoxelParams),
                             ctypes.POINTER(SrcuVoxelOut), ctypes.POINTER(ctypes.c_uint64)],
                            ctypes.c_int),
    "srcu_radius_normals": ([_P, ctypes.POINTER(SrcuCloud), ctypes.POINTER(SrcuNormalParams),
                             ctypes.POINTER(SrcuNormalOut), ctypes.POINTER(SrcuNormalStats)],
                            ctypes.c_int),
    "srcu_voxel_normals": ([_P, ctypes.POINTER(SrcuCloud), ctypes.POINTER(SrcuVoxelParams),
                            ctypes.POINTER(SrcuNormalParams), ctypes.POINTER(SrcuVoxelOut),
                            ctypes.POINTER(SrcuNormalOut), ctypes.POINTER(ctypes.c_uint64),
                            ctypes.POINTER(SrcuNormalStats)], ctypes.c_int),
    "srcu_voxel_normals_enqueue": ([_P, ctypes.POINTER(SrcuCloud), ctypes.POINTER(SrcuVoxelParams),
                                    ctypes.POINTER(SrcuNormalParams)], ctypes.c_int),
    "srcu_voxel_centroid_enqueue": ([_P, ctypes.POINTER(SrcuCloud), ctypes.POINTER(SrcuVoxelParams)],
                                    ctypes.c_int),
    "srcu_frame_view_get": ([_P, ctypes.POINTER(SrcuFrameView)], ctypes.c_int),
    "srcu_frame_check": ([_P, ctypes.POINTER(ctypes.c_uint64), ctypes.POINTER(SrcuNormalStats)],
                         ctypes.c_int),
    "srcu_frame_fetch": ([_P, ctypes.POINTER(SrcuVoxelOut), ctypes.POINTER(SrcuNormalOut),
                          ctypes.POINTER(ctypes.c_uint64), ctypes.POINTER(SrcuNormalStats)],
                         ctypes.c_int),
    "srcu_chain_info_get": ([_P, ctypes.POINTER(SrcuChainInfo)], ctypes.c_int),
    "srcu_batch_voxel_normals_enqueue": ([_P, ctypes.POINTER(SrcuCloud), ctypes.POINTER(ctypes.c_uint64),
                                          ctypes.c_uint32, ctypes.POINTER(SrcuVoxelParams),
                                          ctypes.POINTER(SrcuNormalParams)], ctypes.c_int),
    "srcu_batch_voxel_offsets": ([_P, ctypes.POINTER(ctypes.c_uint64)], ctypes.c_int),
    "srcu_chain_graph_create": ([_P, ctypes.POINTER(SrcuCloud), ctypes.POINTER(ctypes.c_uint64),
                                 ctypes.c_uint32, ctypes.POINTER(SrcuVoxelParams),
                                 ctypes.POINTER(SrcuNormalParams), ctypes.POINTER(ctypes.c_void_p)],
                                ctypes.c_int),
    "srcu_graph_launch": ([_P, _P], ctypes.c_int),
    "srcu_graph_destroy": ([_P], None),
    "srcu_profile_enable": ([_P, ctypes.c_uint64], ctypes.c_int),
    "srcu_voxel_centroid_noalloc": ([ctypes.POINTER(SrcuCloud), ctypes.POINTER(SrcuVoxelParams),
                                     ctypes.POINTER(SrcuVoxelOut), ctypes.POINTER(ctypes.c_uint64),
                                     _P], ctypes.c_int),
    "srcu_profile_read": ([_P, ctypes.POINTER(SrcuKernelStat), ctypes.c_int, ctypes.c_int],
                          ctypes.c_int),
    "srcu_euclidean_cluster_roots": ([_P, ctypes.POINTER(SrcuCloud), ctypes.c_float,
                                      ctypes.c_void_p], ctypes.c_int),
    "srcu_plane_covariances": ([_P, ctypes.POINTER(SrcuCloud), ctypes.c_float, ctypes.c_float,
                                ctypes.c_void_p, ctypes.POINTER(SrcuNormalStats)], ctypes.c_int),
    "srcu_stream_voxel_create": ([_P, ctypes.POINTER(SrcuStreamVoxelParams),
                                  ctypes.POINTER(ctypes.c_void_p)], ctypes.c_int),
    "srcu_stream_voxel_push": ([_P, ctypes.POINTER(SrcuCloud)], ctypes.c_int),
    "srcu_stream_voxel_finish": ([_P, ctypes.POINTER(SrcuStreamVoxelInfo)], ctypes.c_int),
    "srcu_stream_voxel_fetch": ([_P, ctypes.c_uint64, ctypes.c_uint64,
                                 ctypes.POINTER(SrcuStreamVoxelOut)], ctypes.c_int),
    "srcu_stream_voxel_destroy": ([_P], None),
    "srcu_selftest_bounded_wait": ([_P, ctypes.c_uint32], ctypes.c_int),
    "srcu_sort_configs": ([ctypes.c_void_p, ctypes.c_int], ctypes.c_int),
    "srcu_set_neighbor_staging": ([_P, ctypes.c_int32], ctypes.c_int),
    "srcu_get_neighbor_staging": ([_P], ctypes.c_int32),
    "srcu_set_sort_tuning": ([_P, ctypes.c_int32, ctypes.POINTER(ctypes.c_uint64), ctypes.POINTER(ctypes.c_int32),
                              ctypes.c_uint32], ctypes.c_int),
    "srcu_get_sort_tuning": ([_P, ctypes.c_int32, ctypes.POINTER(ctypes.c_uint64), ctypes.POINTER(ctypes.c_int32),
                              ctypes.POINTER(ctypes.c_uint32)], ctypes.c_int),
    "srcu_ransac_plane_scores": ([_P, ctypes.POINTER(SrcuCloud), ctypes.c_void_p, ctypes.c_uint32,
                                  ctypes.c_float, ctypes.POINTER(SrcuPlaneScore)], ctypes.c_int),
    "srcu_ransac_plane_segment": ([_P, ctypes.POINTER(SrcuCloud), ctypes.POINTER(SrcuRansacParams),
                                   ctypes.POINTER(SrcuRansacResult), ctypes.c_void_p], ctypes.c_int),
    "srcu_las_decode": ([_P, ctypes.c_void_p, ctypes.c_uint64, ctypes.c_int32,
                         ctypes.POINTER(SrcuLasFormat), ctypes.POINTER(SrcuLasOut)], ctypes.c_int),
    "srcu_server_create": ([ctypes.POINTER(SrcuServerConfig), ctypes.POINTER(ctypes.c_void_p)],
                           ctypes.c_int),
    "srcu_server_destroy": ([_P], None),
    "srcu_server_submit": ([_P, ctypes.c_uint64, ctypes.POINTER(SrcuCloud),
                            ctypes.POINTER(SrcuVoxelParams), ctypes.POINTER(SrcuNormalParams)],
                           ctypes.c_int),
    "srcu_server_poll": ([_P, ctypes.POINTER(SrcuRequestResult), ctypes.c_uint32], ctypes.c_int),
    "srcu_server_release": ([_P, ctypes.c_uint64], ctypes.c_int),
    "srcu_server_stats_get": ([_P, ctypes.POINTER(SrcuServerStats)], ctypes.c_int),
    "srcu_server_stats_reset": ([_P], ctypes.c_int),
    "srcu_last_length_mismatch": ([_P, ctypes.POINTER(ctypes.c_uint64),
                                   ctypes.POINTER(ctypes.c_uint64)], ctypes.c_int),
    "srcu_debug_set_epoch": ([_P, ctypes.c_uint32], ctypes.c_int),
    "srcu_debug_get_epoch": ([_P, ctypes.POINTER(ctypes.c_uint32), ctypes.POINTER(ctypes.c_uint64)],
                             ctypes.c_int),
    "srcu_noalloc_debug_set_epoch": ([ctypes.c_uint32], ctypes.c_int),
    "srcu_noalloc_debug_get_epoch": ([ctypes.POINTER(ctypes.c_uint32),
                                      ctypes.POINTER(ctypes.c_uint64)], ctypes.c_int),
}

_lib = None

SORT_TUNING_MAX = 32
# SRCU_SORT_VOXEL_KEYS .. SRCU_SORT_BATCH_CELL_KEYS: one table per sort kind,
# the batch kinds for chains of more than one cloud
SORT_KINDS = {"voxel": 0, "cell": 1, "batch_voxel": 2, "batch_cell": 3}


class SrcuSortConfig(ctypes.Structure):
    _fields_ = [("items_per_thread", ctypes.c_uint32), ("blocks_per_sm", ctypes.c_uint32),
                ("digit_bits", ctypes.c_uint32), ("threads_per_block", ctypes.c_uint32)]


def sort_configs() -> list:
    """The sort launch shapes the library was built with, by index."""
    lib = load()
    arr = (SrcuSortConfig * 16)()
    n = lib.srcu_sort_configs(arr, 16)
    return [{f: int(getattr(arr[k], f)) for f, _ in SrcuSortConfig._fields_} for k in range(min(n, 16))]


def library_path() -> str:
    return _LIB_PATH


def load() -> ctypes.CDLL:
    """Loads libsrcuda.so; raises ImportError if it has not been built."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(_LIB_PATH):
        raise ImportError(
            f"{_LIB_PATH} is missing: build it with `python -m spatialrust_b200.csrc.build` "
            "(the CUDA library is required; there is no CPU fallback)")
    lib = ctypes.CDLL(_LIB_PATH)
    for name, (args, res) in SIGNATURES.items():
        fn = getattr(lib, name)
        fn.argtypes = args
        fn.restype = res
    _lib = lib
    return lib


def _raise(status: int, message: str):
    if status == SRCU_ERR_INVALID_ARGUMENT:
        raise InvalidArgument(message)
    if status == SRCU_ERR_LENGTH_MISMATCH:
        raise BufferLengthMismatch(message)
    if status == SRCU_ERR_UNSUPPORTED_DTYPE:
        raise UnsupportedDType(message)
    if status == SRCU_ERR_MISSING_FIELD:
        raise MissingField(message)
    if status == SRCU_ERR_OUT_OF_BUDGET:
        raise OutOfBudget(status, message)
    if status == SRCU_ERR_TIMEOUT:
        raise DeviceTimeout(status, message)
    if status == SRCU_ERR_KEY_OVERFLOW:
        raise KeyOverflow(status, message)
    if status == SRCU_ERR_NO_DEVICE:
        raise NoDevice(status, message)
    raise CudaError(status, message)


def _is_device(a) -> bool:
    return hasattr(a, "data_ptr") and getattr(a, "is_cuda", False)


def _addr(a) -> int:
    if a is None:
        return 0
    if hasattr(a, "data_ptr"):
        return int(a.data_ptr())
    return int(a.ctypes.data)


def _as_f32_host(a) -> np.ndarray:
    return np.ascontiguousarray(a, dtype=np.float32)


class _Keep:
    """Keeps ctypes arrays and converted buffers alive for one call."""

    def __init__(self):
        self.items = []

    def add(self, x):
        self.items.append(x)
        return x


def make_interleaved_cloud(records, position_offsets=(0, 1, 2), attr_offsets=(),
                           keep: _Keep | None = None) -> SrcuCloud:
    """A cloud over interleaved f32 records (n, stride): numpy (host) or a CUDA
    tensor (device), e.g. the reference's AoSoA [x, y, z, intensity] chunks."""
    keep = keep or _Keep()
    on_dev = _is_device(records)
    if not on_dev:
        records = keep.add(np.ascontiguousarray(records, dtype=np.float32))
    if records.ndim != 2:
        raise InvalidArgument("interleaved records must be a 2-D (n, stride) array")
    n, stride = int(records.shape[0]), int(records.shape[1])
    offs = list(position_offsets) + list(attr_offsets)
    if any(o < 0 or o >= stride for o in offs):
        raise InvalidArgument("field offsets must lie inside one record")
    base = _addr(records)
    ptrs = [base + 4 * o for o in offs]
    attr_arr = keep.add((ctypes.c_void_p * max(len(attr_offsets), 1))(*ptrs[3:]))
    return SrcuCloud(ptrs[0], ptrs[1], ptrs[2], ctypes.cast(attr_arr, ctypes.c_void_p),
                     len(attr_offsets), int(on_dev), n, stride, 0)


def make_cloud(x, y, z, attrs: Sequence = (), keep: _Keep | None = None) -> SrcuCloud:
    """SoA columns -> SrcuCloud; a SrcuCloud passed as x is returned as is
    (e.g. one from make_interleaved_cloud)."""
    if isinstance(x, SrcuCloud):
        return x
    keep = keep or _Keep()
    on_dev = _is_device(x)
    cols = [x, y, z, *attrs]
    if on_dev:
        import torch
        for c in cols:
            if not _is_device(c) or c.dtype != torch.float32 or not c.is_contiguous():
                raise InvalidArgument("device columns must be contiguous float32 CUDA tensors")
    else:
        cols = [keep.add(_as_f32_host(c)) for c in cols]
    n = int(cols[0].shape[0])
    for c in cols:
        if int(c.shape[0]) != n:
            raise BufferLengthMismatch(f"expected {n}, found {int(c.shape[0])}")
    if len(attrs) > MAX_ATTRS:
        raise InvalidArgument(f"at most {MAX_ATTRS} attribute columns are supported")
    attr_arr = keep.add((ctypes.c_void_p * max(len(attrs), 1))(*[_addr(c) for c in cols[3:]]))
    return SrcuCloud(_addr(cols[0]), _addr(cols[1]), _addr(cols[2]),
                     ctypes.cast(attr_arr, ctypes.c_void_p), len(attrs), int(on_dev), n)


class Context:
    """One srcu_ctx: a CUDA device, a stream and the HBM-budgeted buffer pool."""

    def __init__(self, device: int = 0, hbm_budget_bytes: int = 0):
        self._lib = load()
        h = ctypes.c_void_p()
        st = self._lib.srcu_create(device, hbm_budget_bytes, ctypes.byref(h))
        if st != SRCU_OK:
            _raise(st, f"srcu_create(device={device}) failed")
        self._h = h
        self.device = device

    def close(self):
        if getattr(self, "_h", None):
            self._lib.srcu_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def _check(self, st: int):
        if st != SRCU_OK:
            msg = self._lib.srcu_last_error(self._h)
            _raise(st, msg.decode() if msg else "")

    @property
    def handle(self) -> ctypes.c_void_p:
        return self._h

    def set_stream(self, stream_handle: int | None):
        self._check(self._lib.srcu_set_stream(self._h, ctypes.c_void_p(stream_handle or 0)))

    def synchronize(self):
        self._check(self._lib.srcu_synchronize(self._h))

    def device_bytes(self) -> int:
        return int(self._lib.srcu_device_bytes(self._h))

    def chain_info(self) -> dict:
        info = SrcuChainInfo()
        self._check(self._lib.srcu_chain_info_get(self._h, ctypes.byref(info)))
        return {name: getattr(info, name) for name, _ in SrcuChainInfo._fields_}

    def profile_enable(self, kernels=()):
        """Times the named kernel groups (see KERNEL_IDS) with CUDA events."""
        mask = 0
        for k in kernels:
            mask |= 1 << KERNEL_IDS.index(k)
        self._check(self._lib.srcu_profile_enable(self._h, mask))

    def profile_read(self, reset: bool = True) -> dict:
        """{group: {name, launches, timed_regions, total_ms}} since the last reset."""
        arr = (SrcuKernelStat * len(KERNEL_IDS))()
        n = self._lib.srcu_profile_read(self._h, arr, len(KERNEL_IDS), int(reset))
        if n < 0:
            self._check(-n)
        return {KERNEL_IDS[i]: dict(name=arr[i].name.decode(), launches=int(arr[i].launches),
                                    timed_regions=int(arr[i].timed_regions),
                                    total_ms=float(arr[i].total_ms)) for i in range(n)}

    # ---- one cloud --------------------------------------------------------

    def voxel_centroid(self, x, y, z, attrs=(), leaf: float = 1.0, origin=None,
                       want_keys: bool = False, approximate: bool = False,
                       attribute_first: bool = False, plain_xyz: bool = False):
        """Returns (columns [x, y, z, attrs...], keys (V,3) int64 or None, counts) as numpy.
        approximate / attribute_first select the reference's ApproximateFirst mode
        and First attribute policy (srcu_voxel_params)."""
        keep = _Keep()
        cloud = make_cloud(x, y, z, attrs, keep)
        n = int(cloud.n)
        ncol = 3 + int(cloud.n_attrs)
        outs = [np.empty(max(n, 1), np.float32) for _ in range(ncol)]
        counts = np.empty(max(n, 1), np.uint32)
        keys = np.empty((max(n, 1), 3), np.int64) if want_keys else None
        attr_out = keep.add((ctypes.c_void_p * max(ncol - 3, 1))(*[o.ctypes.data for o in outs[3:]]))
        vout = SrcuVoxelOut(outs[0].ctypes.data, outs[1].ctypes.data, outs[2].ctypes.data,
                            ctypes.cast(attr_out, ctypes.c_void_p),
                            keys.ctypes.data if keys is not None else 0, counts.ctypes.data, 0)
        vp = _voxel_params(leaf, origin, approximate, attribute_first, plain_xyz)
        nv = ctypes.c_uint64(0)
        self._check(self._lib.srcu_voxel_centroid(self._h, ctypes.byref(cloud), ctypes.byref(vp),
                                                  ctypes.byref(vout), ctypes.byref(nv)))
        v = int(nv.value)
        return ([o[:v] for o in outs], keys[:v] if keys is not None else None, counts[:v])

    def radius_normals(self, x, y, z, radius: float, min_neighbors: int = 3, viewpoint=None,
                       include_self: bool = False):
        """Returns (nx, ny, nz, curvature, neighbor_counts, stats dict) as numpy, input order."""
        keep = _Keep()
        cloud = make_cloud(x, y, z, (), keep)
        n = int(cloud.n)
        outs = [np.empty(max(n, 1), np.float32) for _ in range(4)]
        counts = np.empty(max(n, 1), np.uint32)
        nout = SrcuNormalOut(*[o.ctypes.data for o in outs], counts.ctypes.data, 0)
        np_ = _normal_params(radius, min_neighbors, viewpoint, include_self)
        stats = SrcuNormalStats()
        self._check(self._lib.srcu_radius_normals(self._h, ctypes.byref(cloud), ctypes.byref(np_),
                                                  ctypes.byref(nout), ctypes.byref(stats)))
        return (*[o[:n] for o in outs], counts[:n], _stats(stats))

    def euclidean_cluster_roots(self, x, y, z, cluster_tolerance: float):
        """Smallest point index of every point's component (numpy in and out,
        or CUDA tensors in and a CUDA tensor out)."""
        keep = _Keep()
        cloud = make_cloud(x, y, z, (), keep)
        n = int(cloud.n)
        if cloud.on_device:
            import torch
            roots = torch.empty(max(n, 1), dtype=torch.int32, device=torch.device("cuda", self.device))
            addr = roots.data_ptr()
        else:
            roots = np.empty(max(n, 1), np.uint32)
            addr = roots.ctypes.data
        self._check(self._lib.srcu_euclidean_cluster_roots(self._h, ctypes.byref(cloud),
                                                           ctypes.c_float(cluster_tolerance), addr))
        return roots[:n]

    def sort_tuning(self, kind: str | None = None):
        """[(max_points, launch shape index)] this context sorts `kind` keys
        with ("voxel", "cell", "batch_voxel" or "batch_cell"); all of them as a
        dict when kind is None."""
        if kind is None:
            return {k: self.sort_tuning(k) for k in SORT_KINDS}
        cap = SORT_TUNING_MAX
        mp = (ctypes.c_uint64 * cap)()
        cf = (ctypes.c_int32 * cap)()
        cnt = ctypes.c_uint32(cap)
        self._check(self._lib.srcu_get_sort_tuning(self._h, SORT_KINDS[kind], mp, cf,
                                                   ctypes.byref(cnt)))
        return [(int(mp[k]), int(cf[k])) for k in range(cnt.value)]

    def set_sort_tuning(self, table, kind: str | None = None) -> None:
        """Installs [(max_points, launch shape index)], ascending sizes, for
        the `kind` sort ("voxel", "cell", "batch_voxel" or "batch_cell"; all
        four when None); the last entry also covers larger sorts.  An empty
        table restores the built-in one."""
        if kind is None:
            for k in SORT_KINDS:
                self.set_sort_tuning(table, k)
            return
        table = list(table)
        mp = (ctypes.c_uint64 * max(1, len(table)))(*[int(m) for m, _ in table])
        cf = (ctypes.c_int32 * max(1, len(table)))(*[int(c) for _, c in table])
        self._check(self._lib.srcu_set_sort_tuning(self._h, SORT_KINDS[kind], mp, cf, len(table)))

    def set_neighbor_staging(self, mode: int) -> None:
        """1: the normals kernel stages candidate records in shared memory by
        bulk copies; 0: it reads them through L1; -1: the built-in choice."""
        self._check(self._lib.srcu_set_neighbor_staging(self._h, int(mode)))

    def neighbor_staging(self) -> int:
        return int(self._lib.srcu_get_neighbor_staging(self._h))

    def debug_set_epoch(self, epoch: int) -> None:
        """Test hook: places the look-back epoch (a multiple of 64)."""
        self._check(self._lib.srcu_debug_set_epoch(self._h, int(epoch)))

    def debug_epoch(self) -> tuple:
        """(epoch, restarts) after synchronising."""
        e = ctypes.c_uint32(0)
        r = ctypes.c_uint64(0)
        self._check(self._lib.srcu_debug_get_epoch(self._h, ctypes.byref(e), ctypes.byref(r)))
        return int(e.value), int(r.value)

    def selftest_bounded_wait(self, max_polls: int = 1000):
        """Runs a device wait that must give up: raises DeviceTimeout."""
        self._check(self._lib.srcu_selftest_bounded_wait(self._h, int(max_polls)))

    def ransac_plane_segment(self, x, y, z, distance_threshold: float = 0.01,
                             max_iterations: int = 1000, min_inliers: int = 3, seed: int = 42):
        """(result dict, inlier mask): the CPU segmenter's answer, scored on the
        device.  The mask is a numpy bool array (a CUDA uint8 tensor for
        device inputs)."""
        keep = _Keep()
        cloud = make_cloud(x, y, z, (), keep)
        n = int(cloud.n)
        if cloud.on_device:
            import torch
            mask = torch.empty(max(n, 1), dtype=torch.uint8, device=torch.device("cuda", self.device))
            addr = mask.data_ptr()
        else:
            mask = np.empty(max(n, 1), np.uint8)
            addr = mask.ctypes.data
        prm = SrcuRansacParams(ctypes.c_float(distance_threshold), int(max_iterations),
                               int(min_inliers), int(seed))
        res = SrcuRansacResult()
        self._check(self._lib.srcu_ransac_plane_segment(self._h, ctypes.byref(cloud),
                                                        ctypes.byref(prm), ctypes.byref(res), addr))
        out = dict(normal=tuple(res.normal), d=float(res.d), inlier_count=int(res.inlier_count),
                   hypotheses=int(res.hypotheses), best_hypothesis=int(res.best_hypothesis),
                   hypothesis_normal=tuple(res.hypothesis_normal),
                   hypothesis_d=float(res.hypothesis_d))
        mask = mask[:n]
        return out, (mask if cloud.on_device else mask.astype(bool))

    def ransac_plane_scores(self, x, y, z, hypotheses, distance_threshold: float):
        """[(inlier_count, (nx, ny, nz), d)] per hypothesis (triples of point indices)."""
        keep = _Keep()
        cloud = make_cloud(x, y, z, (), keep)
        hyp = np.ascontiguousarray(hypotheses, np.uint32).reshape(-1, 3)
        scores = (SrcuPlaneScore * max(len(hyp), 1))()
        self._check(self._lib.srcu_ransac_plane_scores(self._h, ctypes.byref(cloud), hyp.ctypes.data,
                                                       len(hyp), ctypes.c_float(distance_threshold),
                                                       scores))
        return [(int(s.inlier_count), tuple(s.normal), float(s.d)) for s in scores[:len(hyp)]]

    def plane_covariances(self, x, y, z, radius: float, epsilon: float, with_stats: bool = False):
        """(n, 6) plane-regularised covariances [c00, c11, c22, c01, c02, c12]
        (numpy in and out, or CUDA tensors in and a CUDA tensor out)."""
        keep = _Keep()
        cloud = make_cloud(x, y, z, (), keep)
        n = int(cloud.n)
        if cloud.on_device:
            import torch
            cov = torch.empty((max(n, 1), 6), dtype=torch.float32,
                              device=torch.device("cuda", self.device))
            addr = cov.data_ptr()
        else:
            cov = np.empty((max(n, 1), 6), np.float32)
            addr = cov.ctypes.data
        stats = SrcuNormalStats()
        self._check(self._lib.srcu_plane_covariances(self._h, ctypes.byref(cloud),
                                                     ctypes.c_float(radius), ctypes.c_float(epsilon),
                                                     addr, ctypes.byref(stats)))
        return (cov[:n], _stats(stats)) if with_stats else cov[:n]

    def voxel_normals(self, x, y, z, attrs=(), leaf: float = 1.0, origin=None, radius: float = 0.5,
                      min_neighbors: int = 3, viewpoint=None, include_self: bool = False,
                      want_keys: bool = False, plain_xyz: bool = False):
        """Voxel centroids then radius normals on them (MvpPipeline chain), numpy outputs."""
        keep = _Keep()
        cloud = make_cloud(x, y, z, attrs, keep)
        n = int(cloud.n)
        ncol = 3 + int(cloud.n_attrs)
        vcols = [np.empty(max(n, 1), np.float32) for _ in range(ncol)]
        counts = np.empty(max(n, 1), np.uint32)
        keys = np.empty((max(n, 1), 3), np.int64) if want_keys else None
        attr_out = keep.add((ctypes.c_void_p * max(ncol - 3, 1))(*[o.ctypes.data for o in vcols[3:]]))
        vout = SrcuVoxelOut(vcols[0].ctypes.data, vcols[1].ctypes.data, vcols[2].ctypes.data,
                            ctypes.cast(attr_out, ctypes.c_void_p),
                            keys.ctypes.data if keys is not None else 0, counts.ctypes.data, 0)
        nouts = [np.empty(max(n, 1), np.float32) for _ in range(4)]
        ncounts = np.empty(max(n, 1), np.uint32)
        nout = SrcuNormalOut(*[o.ctypes.data for o in nouts], ncounts.ctypes.data, 0)
        vp = _voxel_params(leaf, origin, plain_xyz=plain_xyz)
        np_ = _normal_params(radius, min_neighbors, viewpoint, include_self)
        nv = ctypes.c_uint64(0)
        stats = SrcuNormalStats()
        self._check(self._lib.srcu_voxel_normals(self._h, ctypes.byref(cloud), ctypes.byref(vp),
                                                 ctypes.byref(np_), ctypes.byref(vout),
                                                 ctypes.byref(nout), ctypes.byref(nv),
                                                 ctypes.byref(stats)))
        v = int(nv.value)
        return dict(columns=[c[:v] for c in vcols], keys=keys[:v] if keys is not None else None,
                    counts=counts[:v], nx=nouts[0][:v], ny=nouts[1][:v], nz=nouts[2][:v],
                    curvature=nouts[3][:v], neighbor_counts=ncounts[:v], stats=_stats(stats))

    # ---- device-resident chain -------------------------------------------

    def voxel_normals_enqueue(self, cloud: SrcuCloud, leaf: float, origin, radius: float,
                              min_neighbors: int = 3, viewpoint=None, include_self: bool = False,
                              count_shell: bool = True):
        vp = _voxel_params(leaf, origin)
        np_ = _normal_params(radius, min_neighbors, viewpoint, include_self, count_shell)
        self._check(self._lib.srcu_voxel_normals_enqueue(self._h, ctypes.byref(cloud),
                                                         ctypes.byref(vp), ctypes.byref(np_)))

    def voxel_centroid_enqueue(self, cloud: SrcuCloud, leaf: float, origin=None,
                               approximate: bool = False, attribute_first: bool = False):
        """The voxel stage alone on a device-resident cloud, no host sync."""
        vp = _voxel_params(leaf, origin, approximate, attribute_first)
        self._check(self._lib.srcu_voxel_centroid_enqueue(self._h, ctypes.byref(cloud),
                                                          ctypes.byref(vp)))

    def batch_voxel_normals_enqueue(self, points: SrcuCloud, offsets, leaves, radii,
                                    min_neighbors: int = 3, viewpoints=None,
                                    include_self: bool = False, count_shell: bool = True,
                                    origins=None, modes=None):
        """Voxel -> normals for many clouds concatenated in `points` (device).
        modes: per cloud (approximate, attribute_first), default Centroid + Average."""
        count = len(offsets) - 1
        offs = (ctypes.c_uint64 * (count + 1))(*[int(o) for o in offsets])
        vps = (SrcuVoxelParams * count)(*[
            _voxel_params(leaves[b], None if origins is None else origins[b],
                          *((False, False) if modes is None else modes[b]))
            for b in range(count)])
        nps = (SrcuNormalParams * count)(*[
            _normal_params(radii[b], min_neighbors, None if viewpoints is None else viewpoints[b],
                           include_self, count_shell) for b in range(count)])
        self._check(self._lib.srcu_batch_voxel_normals_enqueue(self._h, ctypes.byref(points), offs,
                                                               count, vps, nps))
        self._last_batch = count

    def chain_graph(self, points: SrcuCloud, leaves, radii, offsets=None, min_neighbors=3,
                    viewpoints=None, count_shell=False) -> "ChainGraph":
        """Captures the chain (a batch when offsets is given) as a CUDA graph."""
        count = len(offsets) - 1 if offsets is not None else 1
        offs = (ctypes.c_uint64 * (count + 1))(*[int(o) for o in offsets]) if offsets is not None else None
        vps = (SrcuVoxelParams * count)(*[_voxel_params(leaves[b], None) for b in range(count)])
        nps = (SrcuNormalParams * count)(*[
            _normal_params(radii[b], min_neighbors, None if viewpoints is None else viewpoints[b],
                           False, count_shell) for b in range(count)])
        h = ctypes.c_void_p()
        self._check(self._lib.srcu_chain_graph_create(self._h, ctypes.byref(points), offs, count, vps,
                                                      nps, ctypes.byref(h)))
        self._last_batch = count
        return ChainGraph(self, h)

    def batch_voxel_offsets(self) -> np.ndarray:
        count = getattr(self, "_last_batch", 1)
        out = (ctypes.c_uint64 * (count + 1))()
        self._check(self._lib.srcu_batch_voxel_offsets(self._h, out))
        return np.frombuffer(out, dtype=np.uint64).astype(np.int64)

    def frame_view(self) -> SrcuFrameView:
        view = SrcuFrameView()
        self._check(self._lib.srcu_frame_view_get(self._h, ctypes.byref(view)))
        return view

    def frame_check(self):
        nv = ctypes.c_uint64(0)
        stats = SrcuNormalStats()
        self._check(self._lib.srcu_frame_check(self._h, ctypes.byref(nv), ctypes.byref(stats)))
        return int(nv.value), _stats(stats)

    def frame_fetch(self, capacity: int, n_attrs: int = 0):
        """Reads the last enqueued chain back to numpy (capacity >= V)."""
        keep = _Keep()
        vcols = [np.empty(max(capacity, 1), np.float32) for _ in range(3 + n_attrs)]
        counts = np.empty(max(capacity, 1), np.uint32)
        attr_out = keep.add((ctypes.c_void_p * max(n_attrs, 1))(*[o.ctypes.data for o in vcols[3:]]))
        vout = SrcuVoxelOut(vcols[0].ctypes.data, vcols[1].ctypes.data, vcols[2].ctypes.data,
                            ctypes.cast(attr_out, ctypes.c_void_p), 0, counts.ctypes.data, 0)
        nouts = [np.empty(max(capacity, 1), np.float32) for _ in range(4)]
        ncounts = np.empty(max(capacity, 1), np.uint32)
        nout = SrcuNormalOut(*[o.ctypes.data for o in nouts], ncounts.ctypes.data, 0)
        nv = ctypes.c_uint64(0)
        stats = SrcuNormalStats()
        self._check(self._lib.srcu_frame_fetch(self._h, ctypes.byref(vout), ctypes.byref(nout),
                                               ctypes.byref(nv), ctypes.byref(stats)))
        v = int(nv.value)
        return dict(columns=[c[:v] for c in vcols], counts=counts[:v], nx=nouts[0][:v],
                    ny=nouts[1][:v], nz=nouts[2][:v], curvature=nouts[3][:v],
                    neighbor_counts=ncounts[:v], stats=_stats(stats))


class StreamVoxel:
    """srcu_stream_voxel: global voxel centroids of a chunked stream, reduced
    run by run on the device (StreamingVoxelSource, streaming.rs:334-700).

    attr_f64: one flag per attribute column; True columns are pushed and
    averaged as FP64 (e.g. gps_time), the others as f32."""

    def __init__(self, ctx: "Context", leaf: float, attr_f64=(), run_points: int = 1 << 20,
                 max_runs: int = 1 << 40, spool_limit_bytes: int = 0, device_run_points: int = 0):
        self._ctx = ctx
        self._lib = ctx._lib
        self.attr_f64 = tuple(bool(f) for f in attr_f64)
        mask = sum(1 << i for i, f in enumerate(self.attr_f64) if f)
        prm = SrcuStreamVoxelParams(ctypes.c_float(leaf), len(self.attr_f64), mask,
                                    int(device_run_points), int(run_points), int(max_runs),
                                    int(spool_limit_bytes))
        h = ctypes.c_void_p()
        ctx._check(self._lib.srcu_stream_voxel_create(ctx._h, ctypes.byref(prm), ctypes.byref(h)))
        self._h = h
        self.info = None

    def close(self):
        if getattr(self, "_h", None):
            self._lib.srcu_stream_voxel_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def push(self, x, y, z, attrs=()):
        if len(attrs) != len(self.attr_f64):
            raise InvalidArgument(f"expected {len(self.attr_f64)} attribute columns, got {len(attrs)}")
        keep = _Keep()
        on_dev = _is_device(x)
        if on_dev:
            import torch
            cols = [x, y, z, *attrs]
            want = [torch.float32] * 3 + [torch.float64 if f else torch.float32 for f in self.attr_f64]
            for c, w in zip(cols, want):
                if not _is_device(c) or c.dtype != w or not c.is_contiguous():
                    raise InvalidArgument("device columns must be contiguous CUDA tensors of the "
                                          "stream's column types")
        else:
            cols = [keep.add(np.ascontiguousarray(c, np.float32)) for c in (x, y, z)]
            cols += [keep.add(np.ascontiguousarray(a, np.float64 if f else np.float32))
                     for a, f in zip(attrs, self.attr_f64)]
        n = int(cols[0].shape[0])
        for c in cols:
            if int(c.shape[0]) != n:
                raise BufferLengthMismatch(f"expected {n}, found {int(c.shape[0])}")
        arr = keep.add((ctypes.c_void_p * max(len(attrs), 1))(*[_addr(c) for c in cols[3:]]))
        cloud = SrcuCloud(_addr(cols[0]), _addr(cols[1]), _addr(cols[2]),
                          ctypes.cast(arr, ctypes.c_void_p), len(attrs), int(on_dev), n)
        self._ctx._check(self._lib.srcu_stream_voxel_push(self._h, ctypes.byref(cloud)))

    def finish(self) -> dict:
        info = SrcuStreamVoxelInfo()
        self._ctx._check(self._lib.srcu_stream_voxel_finish(self._h, ctypes.byref(info)))
        self.info = {k: int(getattr(info, k)) for k, _ in SrcuStreamVoxelInfo._fields_}
        return self.info

    def fetch(self, first: int = 0, count: int | None = None):
        """(x, y, z, attrs (count, n_attrs) FP64 means, keys (count, 3), counts)."""
        total = self.info["voxels"] if self.info else 0
        count = total - first if count is None else count
        m = max(count, 1)
        pos = [np.empty(m, np.float32) for _ in range(3)]
        attrs = [np.empty(m, np.float64) for _ in self.attr_f64]
        keys = np.empty((m, 3), np.int64)
        counts = np.empty(m, np.uint64)
        keep = _Keep()
        arr = keep.add((ctypes.c_void_p * max(len(attrs), 1))(*[a.ctypes.data for a in attrs]))
        out = SrcuStreamVoxelOut(pos[0].ctypes.data, pos[1].ctypes.data, pos[2].ctypes.data,
                                 ctypes.cast(arr, ctypes.c_void_p), keys.ctypes.data,
                                 counts.ctypes.data, 0)
        self._ctx._check(self._lib.srcu_stream_voxel_fetch(self._h, first, count, ctypes.byref(out)))
        a = np.stack([c[:count] for c in attrs], axis=1) if attrs else np.zeros((count, 0))
        return pos[0][:count], pos[1][:count], pos[2][:count], a, keys[:count], counts[:count]


class ChainGraph:
    """A captured voxel -> normals chain (srcu_chain_graph_create)."""

    def __init__(self, ctx: Context, handle: ctypes.c_void_p):
        self._ctx = ctx
        self._h = handle

    def launch(self):
        self._ctx._check(self._ctx._lib.srcu_graph_launch(self._ctx.handle, self._h))

    def close(self):
        if self._h:
            self._ctx._lib.srcu_graph_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class Server:
    """The continuous-batching request loop (srcu_server_*): frames and map
    chunks are submitted from host memory, run as voxel -> normals chains
    (small requests packed into batched chains, large ones on bulk slots) and
    polled back with their latency."""

    def __init__(self, device: int = 0, hbm_budget_bytes: int = 0, frame_slots: int = 0,
                 bulk_slots: int = 0, frame_batch_points: int = 0, bulk_threshold_points: int = 0,
                 bulk_max_points: int = 0, max_pending_points: int = 0, host_arena_bytes: int = 0):
        self._lib = load()
        cfg = SrcuServerConfig(device, hbm_budget_bytes, frame_slots, bulk_slots, frame_batch_points,
                               bulk_threshold_points, bulk_max_points, max_pending_points,
                               host_arena_bytes)
        h = ctypes.c_void_p()
        st = self._lib.srcu_server_create(ctypes.byref(cfg), ctypes.byref(h))
        if st != SRCU_OK:
            _raise(st, f"srcu_server_create(device={device}) failed")
        self._h = h

    def close(self):
        if getattr(self, "_h", None):
            self._lib.srcu_server_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def submit(self, req_id: int, x, y, z, intensity=None, *, leaf: float, radius: float,
               min_neighbors: int = 3, viewpoint=None, origin=None, include_self: bool = False,
               count_shell: bool = False) -> bool:
        """Queues one request; False when the pending queue is full (retry later)."""
        keep = _Keep()
        cloud = make_cloud(x, y, z, [] if intensity is None else [intensity], keep)
        vp = _voxel_params(leaf, origin)
        np_ = _normal_params(radius, min_neighbors, viewpoint, include_self, count_shell)
        st = self._lib.srcu_server_submit(self._h, int(req_id), ctypes.byref(cloud), ctypes.byref(vp),
                                          ctypes.byref(np_))
        if st == SRCU_ERR_BUSY:
            return False
        if st != SRCU_OK:
            _raise(st, f"srcu_server_submit(req_id={req_id}) failed")
        return True

    def poll(self, wait_us: int = 0, fetch: bool = True) -> dict | None:
        """One finished request (its columns copied out when fetch, then
        released), or None."""
        r = SrcuRequestResult()
        st = self._lib.srcu_server_poll(self._h, ctypes.byref(r), int(wait_us))
        if st == SRCU_ERR_BUSY:
            return None
        if st != SRCU_OK:
            _raise(st, "srcu_server_poll failed")
        v = int(r.voxels)
        if not fetch:
            self._lib.srcu_server_release(self._h, r.req_id)
            return dict(req_id=int(r.req_id), status=int(r.status), points=int(r.points), voxels=v,
                        latency_ms=float(r.latency_ms))

        def col(ptr, ctype, dtype):
            if not ptr or v == 0:
                return np.zeros(0, dtype=dtype)
            return np.ctypeslib.as_array(ctypes.cast(ptr, ctypes.POINTER(ctype)), (v,)).copy()

        out = dict(req_id=int(r.req_id), status=int(r.status), points=int(r.points), voxels=v,
                   latency_ms=float(r.latency_ms))
        for k in ("x", "y", "z", "nx", "ny", "nz", "curvature"):
            out[k] = col(getattr(r, k), ctypes.c_float, np.float32)
        out["intensity"] = col(r.intensity, ctypes.c_float, np.float32) if r.intensity else None
        out["counts"] = col(r.counts, ctypes.c_uint32, np.uint32)
        self._lib.srcu_server_release(self._h, r.req_id)
        return out

    def stats(self) -> dict:
        s = SrcuServerStats()
        st = self._lib.srcu_server_stats_get(self._h, ctypes.byref(s))
        if st != SRCU_OK:
            _raise(st, "srcu_server_stats_get failed")
        return {k: getattr(s, k) for k, _ in SrcuServerStats._fields_}

    def reset_stats(self):
        self._lib.srcu_server_stats_reset(self._h)


def _voxel_params(leaf, origin, approximate: bool = False,
                  attribute_first: bool = False, plain_xyz: bool = False) -> SrcuVoxelParams:
    mode = (SRCU_VOXEL_APPROXIMATE_FIRST if approximate
            else SRCU_VOXEL_CENTROID_XYZ if plain_xyz else SRCU_VOXEL_CENTROID)
    policy = SRCU_ATTRIBUTE_FIRST if attribute_first else SRCU_ATTRIBUTE_AVERAGE
    if origin is None:
        return SrcuVoxelParams(float(leaf), 0, c_float3(0, 0, 0), mode, policy)
    o = [float(v) for v in origin]
    return SrcuVoxelParams(float(leaf), 1, c_float3(*o), mode, policy)


def _normal_params(radius, min_neighbors, viewpoint, include_self,
                   count_shell=True) -> SrcuNormalParams:
    vp = c_float3(*(float(v) for v in viewpoint)) if viewpoint is not None else c_float3(0, 0, 0)
    return SrcuNormalParams(float(radius), int(min_neighbors), int(viewpoint is not None), vp,
                            int(bool(include_self)), int(bool(count_shell)))


def _stats(s: SrcuNormalStats) -> dict:
    return dict(valid_count=int(s.valid_count), invalid_count=int(s.invalid_count),
                shell_points=int(s.shell_points), fp64_eigensolves=int(s.fp64_eigensolves))


_default_ctx: dict[int, Context] = {}


def shared_context(device: int = 0) -> Context:
    """Process-wide context per device, the analogue of WgpuRuntime::shared()
    (crates/spatialrust-gpu/src/runtime.rs:72-95)."""
    ctx = _default_ctx.get(device)
    if ctx is None:
        ctx = Context(device)
        _default_ctx[device] = ctx
    return ctx
