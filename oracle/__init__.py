"""TEST INFRASTRUCTURE ONLY: CPU oracle for the uniform-grid hot path.

A C restatement of SpatialRust's CPU voxel-centroid and radius-normal paths
(``srcu_oracle.c`` cites the reference file:line of each function) plus an
FP64 normal oracle.  Only ``tests/``, ``__graft_entry__.smoke()`` and the
CPU-baseline legs of ``bench.py`` import this package; the product package
``spatialrust_b200`` never does.
"""
from __future__ import annotations

import ctypes
import os
import subprocess
from dataclasses import dataclass

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_SRC = os.path.join(_HERE, "srcu_oracle.c")
_LIB_PATH = os.path.join(_HERE, "liboracle.so")
# -ffp-contract=off keeps every f32 a*b+c rounded twice, as Rust does.
CFLAGS = ["-O3", "-ffp-contract=off", "-fno-fast-math", "-fPIC", "-shared", "-pthread", "-std=c11",
          "-D_GNU_SOURCE"]

_lib = None


def build(force: bool = False) -> str:
    """Compile srcu_oracle.c into oracle/liboracle.so with gcc."""
    if (not force and os.path.exists(_LIB_PATH)
            and os.path.getmtime(_LIB_PATH) >= os.path.getmtime(_SRC)):
        return _LIB_PATH
    tmp = _LIB_PATH + ".tmp"
    subprocess.check_call(["gcc", *CFLAGS, "-o", tmp, _SRC, "-lm"])
    os.replace(tmp, _LIB_PATH)
    return _LIB_PATH


def _load():
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(_LIB_PATH):
        build()
    lib = ctypes.CDLL(_LIB_PATH)
    P = ctypes.c_void_p
    lib.oracle_voxel_centroid.argtypes = [P, P, P, P, ctypes.c_int, ctypes.c_size_t, ctypes.c_float,
                                          ctypes.c_int, P, ctypes.c_int, P, P, P, P]
    lib.oracle_voxel_centroid.restype = ctypes.c_int
    lib.oracle_voxel_general.argtypes = [P, P, P, P, ctypes.c_int, ctypes.c_size_t, ctypes.c_float,
                                         ctypes.c_int, P, ctypes.c_int, ctypes.c_int, P, P, P, P]
    lib.oracle_voxel_general.restype = ctypes.c_int
    lib.oracle_euclidean_roots.argtypes = [P, P, P, ctypes.c_size_t, ctypes.c_float, P]
    lib.oracle_euclidean_roots.restype = ctypes.c_int
    lib.oracle_euclidean_roots_sparse.argtypes = [P, P, P, ctypes.c_size_t, ctypes.c_float, P]
    lib.oracle_euclidean_roots_sparse.restype = ctypes.c_int
    lib.oracle_radius_normals_ref.argtypes = [P, P, P, ctypes.c_size_t, ctypes.c_float,
                                              ctypes.c_uint32, ctypes.c_int, P, ctypes.c_int, P, P,
                                              P, P, P, P, P]
    lib.oracle_radius_normals_ref.restype = ctypes.c_int
    lib.oracle_radius_normals_fp64.argtypes = [P, P, P, ctypes.c_size_t, ctypes.c_float,
                                               ctypes.c_uint32, ctypes.c_int, P, ctypes.c_double,
                                               ctypes.c_int, P, P, P, P, P, P, P, ctypes.c_int]
    lib.oracle_radius_normals_fp64.restype = ctypes.c_int
    lib.oracle_grid_normals_wgsl.argtypes = [P, P, P, ctypes.c_size_t, ctypes.c_float, ctypes.c_int,
                                             P, ctypes.c_int, P, P, P, P, P]
    lib.oracle_grid_normals_wgsl.restype = ctypes.c_int
    lib.oracle_plane_covariances.argtypes = [P, P, P, ctypes.c_size_t, ctypes.c_float,
                                             ctypes.c_double, ctypes.c_int, P, P, P]
    lib.oracle_plane_covariances.restype = ctypes.c_int
    lib.oracle_stream_voxel.argtypes = [P, P, P, P, ctypes.c_int, ctypes.c_size_t, ctypes.c_float,
                                        P, P, P, P]
    lib.oracle_stream_voxel.restype = ctypes.c_longlong
    lib.oracle_las_decode.argtypes = [P, ctypes.c_size_t, ctypes.c_int, ctypes.c_int, P, P,
                                      ctypes.c_int, P, P, P, P, P, P, P, P]
    lib.oracle_las_decode.restype = ctypes.c_int
    lib.oracle_ransac_plane.argtypes = [P, P, P, ctypes.c_size_t, ctypes.c_float, ctypes.c_uint32,
                                        ctypes.c_uint64, ctypes.c_uint64, P, P, P, P]
    lib.oracle_ransac_plane.restype = ctypes.c_longlong
    lib.oracle_brute_radius_counts.argtypes = [P, P, P, ctypes.c_size_t, ctypes.c_float, P]
    lib.oracle_brute_radius_counts.restype = None
    lib.oracle_compute_bounds.argtypes = [P, P, P, ctypes.c_size_t, P, P]
    lib.oracle_compute_bounds.restype = None
    lib.oracle_smallest_eigenpair_f32.argtypes = [P, P, P]
    lib.oracle_smallest_eigenpair_f32.restype = None
    lib.oracle_parallel_worker_count.argtypes = [ctypes.c_size_t, ctypes.c_size_t]
    lib.oracle_parallel_worker_count.restype = ctypes.c_size_t
    _lib = lib
    return lib


def _f32(a) -> np.ndarray:
    return np.ascontiguousarray(a, dtype=np.float32)


def _ptr(a: np.ndarray) -> ctypes.c_void_p:
    return ctypes.c_void_p(a.ctypes.data)


class OracleError(RuntimeError):
    pass


@dataclass
class VoxelResult:
    fields: list  # x, y, z, attrs... (float32 arrays of length V)
    keys: np.ndarray  # (V, 3) int64
    counts: np.ndarray  # (V,) uint32

    @property
    def x(self):
        return self.fields[0]

    @property
    def y(self):
        return self.fields[1]

    @property
    def z(self):
        return self.fields[2]


def voxel_centroid(x, y, z, attrs=(), leaf=1.0, origin=None, plain_xyz=False) -> VoxelResult:
    """Reference CPU centroid downsample (voxel.rs:251-275, 464-636)."""
    lib = _load()
    x, y, z = _f32(x), _f32(y), _f32(z)
    attrs = [_f32(a) for a in attrs]
    n = x.shape[0]
    cap = max(n, 1)
    outs = [np.empty(cap, np.float32) for _ in range(3 + len(attrs))]
    keys = np.empty((cap, 3), np.int64)
    counts = np.empty(cap, np.uint32)
    attr_ptrs = (ctypes.c_void_p * max(len(attrs), 1))(*[a.ctypes.data for a in attrs])
    out_ptrs = (ctypes.c_void_p * len(outs))(*[o.ctypes.data for o in outs])
    org = np.asarray(origin if origin is not None else (0, 0, 0), np.float32)
    nv = ctypes.c_size_t(0)
    rc = lib.oracle_voxel_centroid(_ptr(x), _ptr(y), _ptr(z), ctypes.cast(attr_ptrs, ctypes.c_void_p),
                                   len(attrs), n, ctypes.c_float(leaf), int(origin is not None),
                                   _ptr(org), int(bool(plain_xyz)),
                                   ctypes.cast(out_ptrs, ctypes.c_void_p), _ptr(keys), _ptr(counts),
                                   ctypes.byref(nv))
    if rc != 0:
        raise OracleError(f"oracle_voxel_centroid failed: {rc}")
    v = nv.value
    return VoxelResult([o[:v].copy() for o in outs], keys[:v].copy(), counts[:v].copy())


def voxel_general(x, y, z, attrs=(), leaf=1.0, origin=None, approximate=False,
                  attribute_first=False) -> VoxelResult:
    """Reference CPU general voxel path (voxel.rs:703-716, 1123-1165): the
    modes other than Centroid + Average.  approximate: ApproximateFirst (every
    field from the voxel's first point); else Centroid with positions
    (sum / count) and attributes first (attribute_first) or (sum / count)."""
    lib = _load()
    x, y, z = _f32(x), _f32(y), _f32(z)
    attrs = [_f32(a) for a in attrs]
    n = x.shape[0]
    cap = max(n, 1)
    outs = [np.empty(cap, np.float32) for _ in range(3 + len(attrs))]
    keys = np.empty((cap, 3), np.int64)
    counts = np.empty(cap, np.uint32)
    attr_ptrs = (ctypes.c_void_p * max(len(attrs), 1))(*[a.ctypes.data for a in attrs])
    out_ptrs = (ctypes.c_void_p * len(outs))(*[o.ctypes.data for o in outs])
    org = np.asarray(origin if origin is not None else (0, 0, 0), np.float32)
    nv = ctypes.c_size_t(0)
    rc = lib.oracle_voxel_general(_ptr(x), _ptr(y), _ptr(z), ctypes.cast(attr_ptrs, ctypes.c_void_p),
                                  len(attrs), n, ctypes.c_float(leaf), int(origin is not None),
                                  _ptr(org), int(bool(approximate)), int(bool(attribute_first)),
                                  ctypes.cast(out_ptrs, ctypes.c_void_p), _ptr(keys), _ptr(counts),
                                  ctypes.byref(nv))
    if rc != 0:
        raise OracleError(f"oracle_voxel_general failed: {rc}")
    v = nv.value
    return VoxelResult([o[:v].copy() for o in outs], keys[:v].copy(), counts[:v].copy())


def euclidean_roots(x, y, z, tolerance, sparse=False) -> np.ndarray:
    """Reference grid union-find (uniform_grid.rs:90-139, 262-289, 389-425):
    the smallest point index of every point's connected component.  sparse:
    the reference's sparse-cell path (euclidean_cluster.rs:9-58 ->
    uniform_grid.rs:148-250), which has no dense cell cap."""
    lib = _load()
    x, y, z = _f32(x), _f32(y), _f32(z)
    n = x.shape[0]
    roots = np.empty(max(n, 1), np.uint32)
    fn = lib.oracle_euclidean_roots_sparse if sparse else lib.oracle_euclidean_roots
    rc = fn(_ptr(x), _ptr(y), _ptr(z), n, ctypes.c_float(tolerance), _ptr(roots))
    if rc == -1:
        raise OracleError("cluster_tolerance must be positive")
    if rc == -3:
        raise OracleError("grid would exceed the reference's dense cell cap")
    if rc != 0:
        raise OracleError(f"oracle_euclidean_roots failed: {rc}")
    return roots[:n].copy()


@dataclass
class NormalResult:
    nx: np.ndarray
    ny: np.ndarray
    nz: np.ndarray
    curvature: np.ndarray
    counts: np.ndarray
    valid_count: int = 0
    invalid_count: int = 0
    gap: np.ndarray | None = None
    shell: np.ndarray | None = None

    @property
    def normals(self) -> np.ndarray:
        return np.stack([self.nx, self.ny, self.nz], axis=1)


def radius_normals_ref(x, y, z, radius, min_neighbors=3, viewpoint=None, threads=0) -> NormalResult:
    """Reference CPU radius normals, f32 arithmetic (normal.rs:102-573)."""
    lib = _load()
    x, y, z = _f32(x), _f32(y), _f32(z)
    n = x.shape[0]
    outs = [np.empty(max(n, 1), np.float32) for _ in range(4)]
    counts = np.zeros(max(n, 1), np.uint32)
    vp = np.asarray(viewpoint if viewpoint is not None else (0, 0, 0), np.float32)
    valid = ctypes.c_size_t(0)
    invalid = ctypes.c_size_t(0)
    rc = lib.oracle_radius_normals_ref(_ptr(x), _ptr(y), _ptr(z), n, ctypes.c_float(radius),
                                       min_neighbors, int(viewpoint is not None), _ptr(vp), threads,
                                       *[_ptr(o) for o in outs], _ptr(counts), ctypes.byref(valid),
                                       ctypes.byref(invalid))
    if rc != 0:
        raise OracleError(f"oracle_radius_normals_ref failed: {rc}")
    return NormalResult(*[o[:n] for o in outs], counts[:n], valid.value, invalid.value)


def radius_normals_fp64(x, y, z, radius, min_neighbors=3, viewpoint=None, shell_rel=1e-6,
                        threads=0, include_self=False) -> NormalResult:
    """FP64 oracle: exact f32-predicate neighbour sets, FP64 covariance and Jacobi.

    include_self: the wgpu grid estimator's semantics (normals_grid.rs:86-197,
    normal_gpu.rs:33-83): the query is in its own neighbourhood (counts
    include it), fewer than 3 points give (0, 0, 1) turned toward the
    viewpoint with curvature 0, min_neighbors is ignored."""
    lib = _load()
    x, y, z = _f32(x), _f32(y), _f32(z)
    n = x.shape[0]
    outs = [np.empty(max(n, 1), np.float64) for _ in range(5)]
    counts = np.zeros(max(n, 1), np.uint32)
    shell = np.zeros(max(n, 1), np.uint8)
    vp = np.asarray(viewpoint if viewpoint is not None else (0, 0, 0), np.float32)
    rc = lib.oracle_radius_normals_fp64(_ptr(x), _ptr(y), _ptr(z), n, ctypes.c_float(radius),
                                        min_neighbors, int(viewpoint is not None), _ptr(vp),
                                        ctypes.c_double(shell_rel), threads,
                                        *[_ptr(o) for o in outs], _ptr(counts), _ptr(shell),
                                        int(bool(include_self)))
    if rc != 0:
        raise OracleError(f"oracle_radius_normals_fp64 failed: {rc}")
    nx, ny, nz, curv, gap = [o[:n] for o in outs]
    valid = int(np.count_nonzero(~np.isnan(nx)))
    return NormalResult(nx, ny, nz, curv, counts[:n], valid, n - valid, gap, shell[:n].astype(bool))


def grid_normals_wgsl(x, y, z, radius, viewpoint=None, threads=0) -> NormalResult:
    """The wgpu grid estimator's f32 arithmetic (NORMALS_GRID_WGSL,
    normals_grid.rs:86-197, 16-sweep Jacobi) and GpuNormalEstimator's
    orientation (normal_gpu.rs:63-70); sums in KD-tree order, so equal to the
    shader up to f32 rounding.  counts include the query."""
    lib = _load()
    x, y, z = _f32(x), _f32(y), _f32(z)
    n = x.shape[0]
    outs = [np.empty(max(n, 1), np.float32) for _ in range(4)]
    counts = np.zeros(max(n, 1), np.uint32)
    vp = np.asarray(viewpoint if viewpoint is not None else (0, 0, 0), np.float32)
    rc = lib.oracle_grid_normals_wgsl(_ptr(x), _ptr(y), _ptr(z), n, ctypes.c_float(radius),
                                      int(viewpoint is not None), _ptr(vp), threads,
                                      *[_ptr(o) for o in outs], _ptr(counts))
    if rc != 0:
        raise OracleError(f"oracle_grid_normals_wgsl failed: {rc}")
    nx, ny, nz, curv = [o[:n] for o in outs]
    valid = int(np.count_nonzero(counts[:n] >= 3))
    return NormalResult(nx, ny, nz, curv, counts[:n], valid, n - valid)


@dataclass
class PlaneCovResult:
    cov: np.ndarray     # (n, 6) float64: c00, c11, c22, c01, c02, c12
    gap: np.ndarray     # (l1 - l0) / l2 of the neighbourhood covariance (0 when invalid)
    counts: np.ndarray  # points within radius, the query included


def plane_covariances(x, y, z, radius, epsilon, threads=0) -> PlaneCovResult:
    """GICP plane-regularised covariances on radius neighbourhoods
    (covariances_grid.rs:87-206), FP64 covariance and Jacobi."""
    lib = _load()
    x, y, z = _f32(x), _f32(y), _f32(z)
    n = x.shape[0]
    cov = np.empty((max(n, 1), 6), np.float64)
    gap = np.zeros(max(n, 1), np.float64)
    counts = np.zeros(max(n, 1), np.uint32)
    rc = lib.oracle_plane_covariances(_ptr(x), _ptr(y), _ptr(z), n, ctypes.c_float(radius),
                                      ctypes.c_double(epsilon), threads, _ptr(cov), _ptr(gap),
                                      _ptr(counts))
    if rc == -1:
        raise OracleError("grid radius must be positive")
    if rc != 0:
        raise OracleError(f"oracle_plane_covariances failed: {rc}")
    return PlaneCovResult(cov[:n], gap[:n], counts[:n])


@dataclass
class StreamVoxelResult:
    keys: np.ndarray    # (V, 3) int64
    counts: np.ndarray  # (V,) uint64
    pos: np.ndarray     # (V, 3) float32
    attrs: np.ndarray   # (V, n_attrs) float64 means


def stream_voxel(x, y, z, attrs=(), leaf=1.0) -> StreamVoxelResult:
    """StreamingVoxelSource's global voxel centroids (streaming.rs:334-700)
    over the whole stream; attributes are FP64 columns."""
    lib = _load()
    x, y, z = _f32(x), _f32(y), _f32(z)
    n = x.shape[0]
    cols = [np.ascontiguousarray(a, np.float64) for a in attrs]
    arr = (ctypes.c_void_p * max(len(cols), 1))(*[c.ctypes.data for c in cols])
    m = max(n, 1)
    keys = np.empty((m, 3), np.int64)
    counts = np.empty(m, np.uint64)
    pos = np.empty((m, 3), np.float32)
    out_attrs = np.empty((m, max(len(cols), 1)), np.float64)
    v = lib.oracle_stream_voxel(_ptr(x), _ptr(y), _ptr(z), ctypes.cast(arr, ctypes.c_void_p),
                                len(cols), n, ctypes.c_float(leaf), _ptr(keys), _ptr(counts),
                                _ptr(pos), _ptr(out_attrs))
    if v == -4:
        raise OracleError("voxel coordinate exceeds signed 64-bit range")
    if v < 0:
        raise OracleError(f"oracle_stream_voxel failed: {v}")
    return StreamVoxelResult(keys[:v], counts[:v], pos[:v], out_attrs[:v, :len(cols)])


def las_decode(records, point_format, record_length, scale, offset, origin=None) -> dict:
    """The point-record fields read_las keeps (reader.rs:242-279), decoded on
    the CPU: x, y, z (f32 of scale * X + offset [- origin] in f64), intensity,
    classification, gps_time, red, green, blue."""
    lib = _load()
    rec = np.ascontiguousarray(np.frombuffer(bytes(records), np.uint8) if not isinstance(
        records, np.ndarray) else records, np.uint8)
    n = rec.nbytes // record_length
    m = max(n, 1)
    out = {k: np.zeros(m, np.float32) for k in ("x", "y", "z", "intensity")}
    out["classification"] = np.zeros(m, np.uint8)
    out["gps_time"] = np.zeros(m, np.float64)
    rgb = np.zeros(3 * m, np.uint16)
    sc = np.asarray(scale, np.float64)
    of = np.asarray(offset, np.float64)
    org = np.asarray(origin if origin is not None else (0, 0, 0), np.float64)
    rc = lib.oracle_las_decode(_ptr(rec), n, point_format, record_length, _ptr(sc), _ptr(of),
                               int(origin is not None), _ptr(org), _ptr(out["x"]), _ptr(out["y"]),
                               _ptr(out["z"]), _ptr(out["intensity"]), _ptr(out["classification"]),
                               _ptr(out["gps_time"]), _ptr(rgb))
    if rc != 0:
        raise OracleError(f"oracle_las_decode failed: {rc}")
    out = {k: v[:n] for k, v in out.items()}
    out["red"], out["green"], out["blue"] = rgb[:n], rgb[n:2 * n], rgb[2 * n:3 * n]
    return out


def ransac_plane(x, y, z, distance_threshold=0.01, max_iterations=1000, min_inliers=3,
                 seed=42) -> dict:
    """RansacPlaneSegmenter::segment_cpu + finalize_plane_segmentation
    (plane.rs:266-345): model (refined), hypothesis model, best hypothesis
    index, inlier count and mask."""
    lib = _load()
    x, y, z = _f32(x), _f32(y), _f32(z)
    n = x.shape[0]
    model = np.zeros(4, np.float32)
    hyp = np.zeros(4, np.float32)
    best = np.zeros(1, np.uint32)
    mask = np.zeros(max(n, 1), np.uint8)
    rc = lib.oracle_ransac_plane(_ptr(x), _ptr(y), _ptr(z), n, ctypes.c_float(distance_threshold),
                                 int(max_iterations), int(min_inliers), int(seed), _ptr(model),
                                 _ptr(hyp), _ptr(best), _ptr(mask))
    if rc == -1:
        raise OracleError("cannot segment plane from empty point cloud")
    if rc == -2:
        raise OracleError("plane segmentation requires at least three points")
    if rc == -5:
        raise OracleError("RANSAC found fewer inliers than min_inliers")
    if rc == -6:
        raise OracleError("failed to refine plane model")
    return dict(model=model, hypothesis=hyp, best_index=int(best[0]), inlier_count=int(rc),
                mask=mask[:n].astype(bool))


def brute_radius_counts(x, y, z, radius) -> np.ndarray:
    lib = _load()
    x, y, z = _f32(x), _f32(y), _f32(z)
    counts = np.zeros(max(x.shape[0], 1), np.uint32)
    lib.oracle_brute_radius_counts(_ptr(x), _ptr(y), _ptr(z), x.shape[0], ctypes.c_float(radius),
                                   _ptr(counts))
    return counts[:x.shape[0]]


def compute_bounds(x, y, z):
    lib = _load()
    x, y, z = _f32(x), _f32(y), _f32(z)
    mn = np.zeros(3, np.float32)
    mx = np.zeros(3, np.float32)
    lib.oracle_compute_bounds(_ptr(x), _ptr(y), _ptr(z), x.shape[0], _ptr(mn), _ptr(mx))
    return mn, mx


def smallest_eigenpair_f32(c00, c11, c22, c01, c02, c12):
    lib = _load()
    c = np.asarray([c00, c11, c22, c01, c02, c12], np.float32)
    normal = np.zeros(3, np.float32)
    curv = ctypes.c_float(0)
    lib.oracle_smallest_eigenpair_f32(_ptr(c), _ptr(normal), ctypes.byref(curv))
    return normal, curv.value


def parallel_worker_count(n: int, available: int) -> int:
    return int(_load().oracle_parallel_worker_count(n, available))
