/*
 * srcuda.h -- C ABI of the B200 (sm_100a) uniform-grid hot path of SpatialRust:
 * VoxelGrid centroid downsample and radius-mode normal estimation.
 *
 * Plain C: pointers, sizes and POD structs only.  Every entry point returns an
 * srcu_status; a message for the last failure on a context is available from
 * srcu_last_error().  Nothing here aborts the process or traps the GPU: device
 * side failures (a bounded wait that gave up, a key that does not fit) are
 * written to a device status word and surfaced as a status code.
 *
 * Threading: a context is NOT thread-safe.  Use one context per host thread,
 * or let one thread own it (the serving loop in this library does so).
 *
 * Reference interfaces replaced (SpatialRust, Rust):
 *   - ExecutionPolicy::Gpu(DeviceKind::Cuda) arm of
 *     VoxelGridDownsample::filter_internal
 *     (crates/spatialrust-filtering/src/voxel.rs:278-308, today rejected at
 *     voxel.rs:336-339),
 *   - ExecutionPolicy::Gpu(DeviceKind::Cuda) arm of
 *     NormalEstimator::estimate_policy_output / resolve_policy
 *     (crates/spatialrust-features/src/normal.rs:208-230, 276-297, today
 *     rejected at normal.rs:292-294),
 *   - GpuNormalEstimator::estimate radius mode
 *     (crates/spatialrust-features/src/normal_gpu.rs:33-83 ->
 *     crates/spatialrust-gpu/src/kernels/normals_grid.rs:208-350),
 *   - the device-resident voxel -> radius-grid -> normals frame chain
 *     (crates/spatialrust-gpu/src/gpu_frame.rs:344-365).
 */
#ifndef SRCUDA_H
#define SRCUDA_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define SRCU_ABI_VERSION 1

/* Status codes.  The first four map 1:1 onto SpatialError
 * (crates/spatialrust-core/src/error.rs:8-37); the rest surface as
 * SpatialError::InvalidArgument(text) on the Rust side. */
typedef enum srcu_status {
  SRCU_OK = 0,
  SRCU_ERR_INVALID_ARGUMENT = 1, /* SpatialError::InvalidArgument */
  SRCU_ERR_LENGTH_MISMATCH = 2,  /* SpatialError::BufferLengthMismatch */
  SRCU_ERR_UNSUPPORTED_DTYPE = 3,/* SpatialError::UnsupportedDType */
  SRCU_ERR_MISSING_FIELD = 4,    /* SpatialError::MissingField */
  SRCU_ERR_OUT_OF_BUDGET = 5,    /* device memory would exceed the context's HBM budget */
  SRCU_ERR_CUDA = 6,             /* CUDA runtime error; text in srcu_last_error() */
  SRCU_ERR_TIMEOUT = 7,          /* a bounded device-side wait gave up */
  SRCU_ERR_KEY_OVERFLOW = 8,     /* packed voxel/cell key would need more than 64 bits */
  SRCU_ERR_NO_DEVICE = 9,        /* no CUDA device of compute capability 10.x */
  SRCU_ERR_BUSY = 10             /* serving loop: request not admitted yet (retry) */
} srcu_status;

typedef struct srcu_ctx srcu_ctx;

/* One point cloud as SoA f32 columns (PointCloud::positions3 plus the F32
 * attribute columns, crates/spatialrust-core/src/capabilities.rs:22-29).
 * Non-F32 attribute columns are widened to f32 by the caller, as the
 * reference's read_buffer_f32 does (voxel.rs:692-701).
 * When on_device != 0 every pointer is a device pointer on the context's
 * device; otherwise host memory (pageable or pinned). */
typedef struct srcu_cloud {
  const float *x;
  const float *y;
  const float *z;
  const float *const *attrs; /* n_attrs columns, e.g. { intensity }; may be NULL if n_attrs == 0 */
  uint32_t n_attrs;
  int32_t on_device;
  uint64_t n;
  /* f32 elements between consecutive points of every column: 0 or 1 for
   * packed columns; larger for interleaved records such as the reference's
   * AoSoA chunks (crates/spatialrust-core/src/tensor_aoso.rs:10-66: [x, y, z,
   * intensity] stride 4, [x, y, z, nx, ny, nz] stride 6, ...), where x, y, z
   * and attrs point at the first record's fields.  At most 64. */
  uint32_t stride;
  uint32_t reserved;
} srcu_cloud;

/* VoxelAggregationMode (voxel.rs:68-76) and AttributeAggregation (voxel.rs:78-86). */
#define SRCU_VOXEL_CENTROID 0          /* mean of every point of the voxel */
#define SRCU_VOXEL_APPROXIMATE_FIRST 1 /* the voxel's first point (input order) */
/* Centroid + Average on a cloud whose only fields are x, y, z: the reference's
 * plain-xyz fast path (filter_cpu_xyz_centroid_fast, voxel.rs:550-636) --
 * f32 sums in input order, (sum * (1 / count)) in f32, voxels in the order of
 * their first point.  srcu_voxel_centroid and srcu_voxel_normals only, with
 * n_attrs == 0 and SRCU_ATTRIBUTE_AVERAGE. */
#define SRCU_VOXEL_CENTROID_XYZ 2
#define SRCU_ATTRIBUTE_AVERAGE 0
#define SRCU_ATTRIBUTE_FIRST 1

/* VoxelGridDownsampleConfig (crates/spatialrust-filtering/src/voxel.rs:112-183).
 * Centroid + Average is the reference's fast path (voxel.rs:464-540:
 * (sum * (1/count)) as f32 for every field).  The other combinations follow
 * its general path (voxel.rs:1123-1165): Centroid + First averages the
 * positions as (sum / count) as f32 and takes the other fields from the
 * voxel's first point; ApproximateFirst takes every field from the first
 * point, whatever the attribute policy.  Zero-initialised = Centroid + Average. */
typedef struct srcu_voxel_params {
  float leaf_size;  /* must be > 0 (NaN passes, as in voxel.rs:260) */
  int32_t has_origin;
  float origin[3];  /* used when has_origin != 0: floor keys; else origin = min corner, truncated keys */
  int32_t mode;             /* SRCU_VOXEL_CENTROID or SRCU_VOXEL_APPROXIMATE_FIRST */
  int32_t attribute_policy; /* SRCU_ATTRIBUTE_AVERAGE or SRCU_ATTRIBUTE_FIRST */
} srcu_voxel_params;

/* Voxel output.  Each column needs capacity >= input n (the voxel count is
 * never larger).  Voxels are emitted in ascending (ix, iy, iz) order, the
 * reference's output order for point_xyzi (voxel.rs:522-536), or in
 * first-seen order under SRCU_VOXEL_CENTROID_XYZ. */
typedef struct srcu_voxel_out {
  float *x;
  float *y;
  float *z;
  float *const *attrs; /* n_attrs columns (same count as the input cloud) */
  int64_t *keys;       /* nullable: 3 int64 per voxel, the reference's (ix, iy, iz) */
  uint32_t *counts;    /* nullable: points per voxel */
  int32_t on_device;
} srcu_voxel_out;

/* NormalEstimationConfig in radius mode
 * (crates/spatialrust-features/src/normal.rs:17-71). */
typedef struct srcu_normal_params {
  float radius;            /* search_radius; must be >= 0 (normal.rs:109-111) */
  uint32_t min_neighbors;  /* default 3 */
  int32_t has_viewpoint;
  float viewpoint[3];
  int32_t include_self;    /* 0: NormalEstimator CPU semantics (self excluded, NaN when invalid).
                              1: GpuNormalEstimator grid semantics (self included, fewer than
                                 3 points -> (0,0,1), curvature 0; normals_grid.rs:86-197). */
  int32_t count_shell;     /* 1: count shell points into srcu_normal_stats (a few extra
                              instructions per candidate); 0: shell_points stays 0 */
} srcu_normal_params;

typedef struct srcu_normal_out {
  float *nx;
  float *ny;
  float *nz;
  float *curvature;
  uint32_t *neighbor_counts; /* nullable: neighbours found per point (self excluded unless include_self) */
  int32_t on_device;
} srcu_normal_out;

/* NormalEstimationResult (normal.rs:74-80) plus diagnostics. */
typedef struct srcu_normal_stats {
  uint64_t valid_count;
  uint64_t invalid_count;
  uint64_t shell_points;  /* points with some other point at |d^2 - r^2| <= 1e-6 r^2 */
  uint64_t fp64_eigensolves; /* near-degenerate covariances recomputed with FP64 moments */
} srcu_normal_stats;

/* ---- context ------------------------------------------------------------ */

int srcu_abi_version(void);

/* Creates a context on CUDA device `device`.  hbm_budget_bytes caps the device
 * memory this context may hold (0 = no cap); allocations beyond it fail with
 * SRCU_ERR_OUT_OF_BUDGET.  Replaces WgpuRuntime::shared()
 * (crates/spatialrust-gpu/src/runtime.rs:72-95). */
srcu_status srcu_create(int device, uint64_t hbm_budget_bytes, srcu_ctx **out);
void srcu_destroy(srcu_ctx *ctx);
const char *srcu_last_error(const srcu_ctx *ctx);
/* The element counts behind the last SRCU_ERR_LENGTH_MISMATCH on this context
 * (SpatialError::BufferLengthMismatch { expected, found }, error.rs:27-32);
 * both 0 when the last failure was of another kind. */
srcu_status srcu_last_length_mismatch(const srcu_ctx *ctx, uint64_t *expected, uint64_t *found);

/* Runs subsequent work on a caller stream (a cudaStream_t); NULL restores the
 * context's own stream. */
srcu_status srcu_set_stream(srcu_ctx *ctx, void *cuda_stream);
srcu_status srcu_synchronize(srcu_ctx *ctx);
/* Device bytes currently held by the context. */
uint64_t srcu_device_bytes(const srcu_ctx *ctx);

/* ---- one cloud ------------------------------------------------------------ */

/* VoxelGridDownsample::filter_with_policy(cloud, Gpu(Cuda)) for
 * Centroid + Average (voxel.rs:213-237, 251-368, 464-540): per-voxel means of
 * x, y, z and every attribute, accumulated in FP64, emitted in key order.
 * Synchronous: returns after the outputs are written; *out_voxels = V. */
srcu_status srcu_voxel_centroid(srcu_ctx *ctx, const srcu_cloud *cloud,
                                const srcu_voxel_params *params, const srcu_voxel_out *out,
                                uint64_t *out_voxels);

/* NormalEstimator::estimate_with_policy(cloud, Gpu(Cuda)) with
 * search_radius = Some(r) (normal.rs:102-164, 321-573), or, with
 * include_self = 1, GpuNormalEstimator::estimate (normal_gpu.rs:33-83).
 * Outputs are in input point order.  Synchronous.  stats is nullable. */
srcu_status srcu_radius_normals(srcu_ctx *ctx, const srcu_cloud *cloud,
                                const srcu_normal_params *params, const srcu_normal_out *out,
                                srcu_normal_stats *stats);

/* MvpPipeline voxel -> normals chain (crates/spatialrust-pipeline/src/mvp.rs:193-226):
 * centroid downsample, then radius normals on the centroids, all on the
 * device.  vout gets the centroids, nout the normals of each centroid (both
 * V long, capacity n).  Synchronous. */
srcu_status srcu_voxel_normals(srcu_ctx *ctx, const srcu_cloud *cloud,
                               const srcu_voxel_params *vparams, const srcu_normal_params *nparams,
                               const srcu_voxel_out *vout, const srcu_normal_out *nout,
                               uint64_t *out_voxels, srcu_normal_stats *stats);

/* ---- Euclidean clustering on the same grid -------------------------------- */

/* Connected-component roots of the graph "dx*dx + dy*dy + dz*dz <= tol*tol"
 * (f32): roots[i] is the smallest point index of point i's component, the
 * result of spatialrust_search::euclidean_cluster_roots
 * (crates/spatialrust-search/src/uniform_grid.rs:90-139), which
 * GpuEuclideanClusterExtractor::extract (crates/spatialrust-segmentation/src/
 * cluster_gpu.rs:31-63) and the Gpu(Cuda) arm of
 * EuclideanClusterExtractor::extract_with_policy (cluster.rs:156-235, rejected
 * today at cluster.rs:233-235) turn into labels.  The whole union-find runs on
 * the device (the reference runs it on the host).  roots: n entries, host or
 * device memory as cloud->on_device.  cluster_tolerance must be > 0 and
 * finite.  Synchronous. */
srcu_status srcu_euclidean_cluster_roots(srcu_ctx *ctx, const srcu_cloud *cloud,
                                         float cluster_tolerance, uint32_t *roots);

/* ---- GICP plane covariances on the same grid ------------------------------ */

/* Replaces spatialrust_gpu::estimate_plane_covariances_grid_gpu
 * (crates/spatialrust-gpu/src/kernels/covariances_grid.rs:216-364), which
 * GicpRegistration::point_covariances calls when covariance_radius is set
 * (crates/spatialrust-registration/src/gicp.rs:89-101, 237-256).  For every
 * point: the covariance of the points within radius of it (itself included,
 * f32 predicate), its eigenvalues replaced by (epsilon, 1, 1) -- the
 * plane-to-plane model -- as 6 floats [c00, c11, c22, c01, c02, c12]
 * (GpuCovariance) at cov[6 i .. 6 i + 5]; fewer than 3 points in the
 * neighbourhood give (epsilon, epsilon, epsilon, 0, 0, 0).  cov: 6 n floats,
 * host or device memory as cloud->on_device.  radius must be > 0 and finite.
 * stats (nullable) counts the valid and the fallback points.  Synchronous. */
srcu_status srcu_plane_covariances(srcu_ctx *ctx, const srcu_cloud *cloud, float radius,
                                   float epsilon, float *cov, srcu_normal_stats *stats);

/* ---- sort launch shapes and their tuning ------------------------------------ */

/* The onesweep radix sort is built in several launch shapes -- keys per thread,
 * the blocks per SM its registers are capped for, threads per block (256 or
 * 512) and digit width: 8 bits, or 9 bits in the 512-thread shapes built for
 * them, which take 9-bit digits only where that saves a pass over the key
 * width at hand (and 8-bit digits otherwise).
 * A context picks one per sort from a table of input sizes, one table per sort
 * kind: the voxel-key sort over the input points and the cell-key sort of the
 * radius grid, each for one cloud and for a batch of clouds (whose keys carry
 * the cloud id above the per-cloud key, so they are wider).  The built-in
 * tables were measured by spatialrust_b200.autotune on a B200;
 * srcu_set_sort_tuning installs others (the autotuner does so while it
 * measures).  No counterpart in the reference (its wgpu bitonic sort has fixed
 * workgroups). */
#define SRCU_SORT_TUNING_MAX 32
#define SRCU_SORT_VOXEL_KEYS 0
#define SRCU_SORT_CELL_KEYS 1
#define SRCU_SORT_BATCH_VOXEL_KEYS 2
#define SRCU_SORT_BATCH_CELL_KEYS 3
#define SRCU_SORT_KINDS 4

typedef struct srcu_sort_config {
  uint32_t items_per_thread;
  uint32_t blocks_per_sm;
  uint32_t digit_bits;
  uint32_t threads_per_block;
} srcu_sort_config;

/* Fills up to max_entries shapes; returns how many the library has. */
int srcu_sort_configs(srcu_sort_config *out, int max_entries);
/* Entry k of the `kind` table: sorts of at most max_points[k] keys use shape
 * config[k] (ascending sizes; the last entry also covers every larger sort).
 * count 0 restores the built-in table. */
srcu_status srcu_set_sort_tuning(srcu_ctx *ctx, int32_t kind, const uint64_t *max_points,
                                 const int32_t *config, uint32_t count);
/* *count: capacity in, entries out. */
srcu_status srcu_get_sort_tuning(srcu_ctx *ctx, int32_t kind, uint64_t *max_points,
                                 int32_t *config, uint32_t *count);

/* The normals kernel's neighbour walk.  0: range by range through L1.  1: range
 * by range, each warp's candidate records (the x-strips of its 3x3 column
 * block) first staged in shared memory by non-multicast cp.async.bulk copies.
 * 2: walk 0 with the predicate and the moments in packed f32x2 arithmetic.
 * Every walk gives the same neighbour sets and counts, and walks 0 and 2 give
 * bit-identical outputs.  -1 restores the built-in choice (measured by the
 * autotuner).  Plane covariances take walk 2 when it is chosen, else 0. */
srcu_status srcu_set_neighbor_staging(srcu_ctx *ctx, int32_t mode);
int32_t srcu_get_neighbor_staging(srcu_ctx *ctx);

/* ---- failure path self-test ------------------------------------------------ */

/* No counterpart in the reference.  Runs one device-side wait on a flag that
 * nothing sets, bounded at max_polls polls about a microsecond apart (at most
 * 2^21), so that the wait gives up the way every wait in this library does:
 * the call returns SRCU_ERR_TIMEOUT and the context stays usable.  For
 * health checks and tests of the error path; it never faults the GPU. */
srcu_status srcu_selftest_bounded_wait(srcu_ctx *ctx, uint32_t max_polls);

/* ---- epoch of the look-back tags (tests) ------------------------------------ */

/* No counterpart in the reference.  Every chain tags the look-back words and
 * hash slots it publishes with a 32-bit epoch that advances by 64 per chain
 * (or graph replay).  Before the epoch would wrap, the context clears every
 * tagged array and restarts the epoch at 0, so a tag never repeats while an
 * old word may carry it.  These two calls exist for tests of that restart:
 * set_epoch (a multiple of 64) places a context just below the wrap;
 * get_epoch synchronises and returns the epoch and how many restarts ran. */
srcu_status srcu_debug_set_epoch(srcu_ctx *ctx, uint32_t epoch);
srcu_status srcu_debug_get_epoch(srcu_ctx *ctx, uint32_t *epoch, uint64_t *restarts);

/* ---- RANSAC plane segmentation ------------------------------------------- */

/* GpuPlaneScore (crates/spatialrust-gpu/src/kernels/ransac_plane.rs:27-37). */
typedef struct srcu_plane_score {
  uint32_t inlier_count;
  float normal[3];
  float d;
} srcu_plane_score;

/* RansacPlaneConfig (crates/spatialrust-segmentation/src/plane.rs:55-93). */
typedef struct srcu_ransac_params {
  float distance_threshold; /* default 0.01 */
  uint32_t max_iterations;  /* default 1000 (at most 2^26) */
  uint64_t min_inliers;     /* default 3 */
  uint64_t seed;            /* default 42 */
} srcu_ransac_params;

typedef struct srcu_ransac_result {
  float normal[3];            /* the model: refined from the inliers (>= 3), else the hypothesis */
  float d;
  uint64_t inlier_count;
  uint32_t hypotheses;        /* hypotheses scored */
  uint32_t best_hypothesis;   /* index of the winning hypothesis (UINT32_MAX: none) */
  float hypothesis_normal[3]; /* its plane, before refinement */
  float hypothesis_d;
} srcu_ransac_result;

/* Replaces score_ransac_plane_hypotheses_gpu (ransac_plane.rs:104-263): the
 * plane of each hypothesis (3 point indices, host memory) and its inlier count
 * with the CPU path's f32 arithmetic (plane_ransac.rs:54-94, plane.rs:39-41);
 * a degenerate triple scores all zeros.  scores: count entries, host memory.
 * Synchronous. */
srcu_status srcu_ransac_plane_scores(srcu_ctx *ctx, const srcu_cloud *cloud,
                                     const uint32_t *hypotheses, uint32_t count,
                                     float distance_threshold, srcu_plane_score *scores);

/* The Gpu(Cuda) arm of RansacPlaneSegmenter::segment_with_policy (plane.rs:
 * 151-264, rejected today at plane.rs:259-261) with the CPU segmenter's
 * results (plane.rs:266-345): the reference's seeded hypotheses, all scored on
 * the device, the first hypothesis with the most inliers, its inlier mask
 * (inlier_mask: n bytes, nullable, host or device memory as cloud->on_device)
 * and the model refined from the inliers in FP64.  Fails as the reference does
 * for empty clouds, fewer than 3 points and fewer than min_inliers inliers.
 * Synchronous. */
srcu_status srcu_ransac_plane_segment(srcu_ctx *ctx, const srcu_cloud *cloud,
                                      const srcu_ransac_params *params, srcu_ransac_result *result,
                                      uint8_t *inlier_mask);

/* ---- bounded streaming voxel centroids ------------------------------------ */

/* Replaces StreamingVoxelSource (crates/spatialrust-pipeline/src/streaming.rs:
 * 334-700): global voxel centroids of a chunked stream.  The voxel of a point
 * is floor(f64(v) / f64(leaf)) per axis (no origin, :986-994); points with a
 * non-finite coordinate are skipped (:464-466); every column is averaged in
 * FP64 over the whole stream; voxels come out in ascending (ix, iy, iz) order.
 * Chunks are reduced on the device run by run; only the reduced runs stay
 * resident (device memory under the context's HBM budget plays the part of
 * the reference's disk spool).  push and finish use the context's sort
 * buffers and stream; like the context, a stream belongs to one thread. */
typedef struct srcu_stream_voxel srcu_stream_voxel;

typedef struct srcu_stream_voxel_params {
  float leaf_size;          /* > 0 and finite (StreamingVoxelConfig::new, streaming.rs:345-363) */
  uint32_t n_attrs;         /* attribute columns in every chunk */
  uint32_t attr_f64_mask;   /* bit a: attrs[a] of every chunk points at f64 data, not f32 */
  uint32_t device_run_points; /* points sorted per device run; 0: max(run_points, 2^22) */
  uint64_t run_points;      /* > 0: finite points per run of the reference's run limit */
  uint64_t max_runs;        /* > 0: more runs than this fail, as flush_run does (:742-746) */
  uint64_t spool_limit_bytes; /* 0: none; else the reference's spool extent rule: runs * 8 +
                                 finite points * (32 + 8 * (3 + n_attrs)) bytes at most */
} srcu_stream_voxel_params;

typedef struct srcu_stream_voxel_info {
  uint64_t points;          /* points pushed */
  uint64_t finite_points;   /* points kept */
  uint64_t runs;            /* the reference's run count: ceil(finite / run_points) */
  uint64_t spool_bytes;     /* the reference's spool bytes for those runs */
  uint64_t device_runs;     /* runs reduced on the device */
  uint64_t partial_records; /* reduced records held before the final merge */
  uint64_t voxels;          /* output voxels */
} srcu_stream_voxel_info;

typedef struct srcu_stream_voxel_out {
  float *x;
  float *y;
  float *z;
  double *const *attrs; /* n_attrs columns of FP64 means (nullable entries skip a column) */
  int64_t *keys;        /* nullable: 3 int64 per voxel */
  uint64_t *counts;     /* nullable: points per voxel */
  int32_t on_device;
} srcu_stream_voxel_out;

srcu_status srcu_stream_voxel_create(srcu_ctx *ctx, const srcu_stream_voxel_params *params,
                                     srcu_stream_voxel **out);
/* Appends one chunk (packed columns, host or device; stride must be 0 or 1). */
srcu_status srcu_stream_voxel_push(srcu_stream_voxel *sv, const srcu_cloud *chunk);
/* Reduces the last run and merges every run; info is nullable. */
srcu_status srcu_stream_voxel_finish(srcu_stream_voxel *sv, srcu_stream_voxel_info *info);
/* Copies voxels [first, first + count) of the finished stream. */
srcu_status srcu_stream_voxel_fetch(srcu_stream_voxel *sv, uint64_t first, uint64_t count,
                                    const srcu_stream_voxel_out *out);
/* Ends a stream.  Its device buffers stay with the context for the context's next
 * stream (srcu_destroy frees them); destroy every stream before its context. */
void srcu_stream_voxel_destroy(srcu_stream_voxel *sv);

/* ---- LAS point records ---------------------------------------------------- */

/* One LAS file's point data layout (public header fields, ASPRS LAS 1.4 R15
 * table 3) and an optional FP64 origin. */
typedef struct srcu_las_format {
  uint32_t point_format;   /* point data record format 0-10 (header byte 104, compression bits clear) */
  uint32_t record_length;  /* point data record length (header bytes 105-106), extra bytes included */
  double scale[3];         /* x, y, z scale factors (header bytes 131-154) */
  double offset[3];        /* x, y, z offsets (header bytes 155-178) */
  int32_t has_origin;      /* 1: subtract origin from scale * X + offset in FP64 before the f32 */
  int32_t reserved;
  double origin[3];
} srcu_las_format;

/* Decoded columns (n entries each; every pointer but x, y, z is nullable). */
typedef struct srcu_las_out {
  float *x;
  float *y;
  float *z;
  float *intensity;        /* F32, as schema_for_las_header's point_xyzi */
  uint8_t *classification; /* class number: low 5 bits for formats 0-5, the byte for 6-10 */
  double *gps_time;        /* formats 1, 3-10 */
  uint16_t *red;           /* formats 2, 3, 5, 7, 8, 10 */
  uint16_t *green;
  uint16_t *blue;
  int32_t on_device;
} srcu_las_out;

/* Decodes n uncompressed LAS point records (records: n * record_length
 * bytes, host or device memory as records_on_device) into columns, the
 * fields read_las keeps (crates/spatialrust-io/src/las/reader.rs:242-279):
 * each coordinate is scale * X + offset in FP64 (minus origin when
 * has_origin), stored as f32.  Synchronous. */
srcu_status srcu_las_decode(srcu_ctx *ctx, const void *records, uint64_t n,
                            int32_t records_on_device, const srcu_las_format *fmt,
                            const srcu_las_out *out);

/* ---- many clouds in one chain ---------------------------------------------- */

/* Enqueues voxel -> normals for `count` clouds in one chain: the clouds'
 * points are concatenated in `points` (device-resident), cloud b owning
 * points [offsets[b], offsets[b+1]) (host array, count + 1 entries, offsets[0]
 * = 0, offsets[count] = points->n).  Each cloud has its own voxel and normal
 * parameters (host arrays of count entries).  The cloud id rides above the
 * per-cloud key bits, so one sort, one segment pass and one radius grid serve
 * every cloud; neighbours never cross clouds.  Results stay on the device in
 * cloud order (srcu_frame_view_get / srcu_frame_fetch); the voxel range of
 * each cloud comes from srcu_batch_voxel_offsets.  Replaces a per-cloud loop
 * of MvpPipeline::run (crates/spatialrust-pipeline/src/mvp.rs:193-226). */
srcu_status srcu_batch_voxel_normals_enqueue(srcu_ctx *ctx, const srcu_cloud *points,
                                             const uint64_t *offsets, uint32_t count,
                                             const srcu_voxel_params *vparams,
                                             const srcu_normal_params *nparams);
/* Synchronises and copies the count + 1 voxel offsets of the last batch. */
srcu_status srcu_batch_voxel_offsets(srcu_ctx *ctx, uint64_t *voxel_offsets);

/* ---- CUDA graphs ---------------------------------------------------------- */

typedef struct srcu_graph srcu_graph;

/* Captures the voxel -> normals chain for these exact inputs (a batch when
 * offsets is non-NULL, else one cloud) as a CUDA graph on the context
 * stream.  Runs the chain once uncaptured first (sizing buffers and staging
 * parameters), then captures only the kernels.  Replays read the same input
 * pointers and write the context's result buffers; the context must not run
 * other chains while the graph is in use. */
srcu_status srcu_chain_graph_create(srcu_ctx *ctx, const srcu_cloud *points,
                                    const uint64_t *offsets, uint32_t count,
                                    const srcu_voxel_params *vparams,
                                    const srcu_normal_params *nparams, srcu_graph **out);
srcu_status srcu_graph_launch(srcu_ctx *ctx, srcu_graph *graph);
void srcu_graph_destroy(srcu_graph *graph);

/* ---- device-resident chain (GpuSpatialFrame, gpu_frame.rs:71-365) --------- */

/* Enqueues the voxel -> normals chain on the context stream for a cloud
 * already on the device, without any host synchronisation; results stay in
 * context-owned device buffers (valid until the next enqueue).  Safe to
 * capture in a CUDA graph after one uncaptured warm-up call of the same size. */
srcu_status srcu_voxel_normals_enqueue(srcu_ctx *ctx, const srcu_cloud *cloud,
                                       const srcu_voxel_params *vparams,
                                       const srcu_normal_params *nparams);

/* The voxel stage alone (VoxelGridDownsample on a device-resident cloud):
 * bounds, key plan, sort and the fused segment reduction, enqueued on the
 * context stream without host synchronisation.  The centroids stay in the
 * context's buffers (srcu_frame_view_get: x, y, z, attrs, counts,
 * voxel_count; the normal pointers are not written); srcu_frame_check reads
 * the status and V.  Same conditions as srcu_voxel_normals_enqueue. */
srcu_status srcu_voxel_centroid_enqueue(srcu_ctx *ctx, const srcu_cloud *cloud,
                                        const srcu_voxel_params *vparams);

typedef struct srcu_frame_view {
  const float *x, *y, *z;        /* device: centroids (capacity n) */
  const float *const *attrs;     /* host array of device column pointers */
  const float *nx, *ny, *nz, *curvature; /* device */
  const uint32_t *counts;        /* device: points per voxel */
  const uint64_t *voxel_count;   /* device: V */
  uint32_t n_attrs;
} srcu_frame_view;

/* Device pointers of the last enqueued chain's results. */
srcu_status srcu_frame_view_get(srcu_ctx *ctx, srcu_frame_view *view);
/* Synchronises and checks the device status word of the last enqueue. */
srcu_status srcu_frame_check(srcu_ctx *ctx, uint64_t *out_voxels, srcu_normal_stats *stats);

/* Facts about the last chain (after srcu_frame_check or a synchronous call). */
typedef struct srcu_chain_info {
  uint64_t points;
  uint64_t voxels;
  uint64_t cells;             /* occupied radius-grid cells */
  uint32_t voxel_key_bits;
  uint32_t cell_key_bits;
  uint32_t voxel_sort_passes; /* onesweep digit passes that ran */
  uint32_t cell_sort_passes;
  double cell_size;           /* radius-grid cell edge (>= radius) */
} srcu_chain_info;

srcu_status srcu_chain_info_get(srcu_ctx *ctx, srcu_chain_info *info);

/* Explicit read-back of the last enqueued chain (GpuSpatialFrame readback,
 * gpu_frame.rs:292-328): synchronises, then copies the V centroids and their
 * normals into caller buffers (capacity >= V; either out may be NULL). */
srcu_status srcu_frame_fetch(srcu_ctx *ctx, const srcu_voxel_out *vout, const srcu_normal_out *nout,
                             uint64_t *out_voxels, srcu_normal_stats *stats);

/* ---- serving loop ------------------------------------------------------------ */

/* A request loop that admits frames and map chunks of different sizes as they
 * arrive and runs voxel -> normals on them with continuous batching: small
 * requests waiting when a batch slot frees up are packed into one batched
 * chain (srcu_batch_voxel_normals_enqueue) on that slot's stream, large
 * requests run on their own slots so they never hold small ones back, and
 * several slots overlap on the device.  Admission is gated by the pending
 * queue (max_pending_points) and by the HBM budget that sizes the slots.
 * One worker thread owns all device work; submit / poll / release may be
 * called from any threads. */
typedef struct srcu_server srcu_server;

typedef struct srcu_server_config {
  int device;
  uint64_t hbm_budget_bytes;      /* device memory for all slots (0: 40 GB) */
  uint32_t frame_slots;           /* concurrent batches of small requests (0: 3) */
  uint32_t bulk_slots;            /* concurrent large requests (0: 1) */
  uint64_t frame_batch_points;    /* most points packed into one small-request batch (0: 1M) */
  uint64_t bulk_threshold_points; /* requests with at least this many points use bulk slots (0: 500k) */
  uint64_t bulk_max_points;       /* largest admissible request (0: 4.5M) */
  uint64_t max_pending_points;    /* beyond this queued total, submit returns SRCU_ERR_BUSY (0: 64M) */
  uint64_t host_arena_bytes;      /* pinned host memory for queued inputs and unreleased
                                     results; submit returns SRCU_ERR_BUSY when full (0: 2 GB) */
} srcu_server_config;

typedef struct srcu_request_result {
  uint64_t req_id;
  srcu_status status;
  uint64_t points;
  uint64_t voxels;
  const float *x, *y, *z, *intensity;      /* centroids (intensity NULL without it) */
  const float *nx, *ny, *nz, *curvature;  /* normals of each centroid */
  const uint32_t *counts;                 /* points per voxel */
  double latency_ms;                      /* submit -> results ready */
} srcu_request_result;

typedef struct srcu_server_stats {
  uint64_t submitted, rejected, completed, failed, batches, points;
  double frame_p50_ms, frame_p99_ms;      /* requests below bulk_threshold_points */
  double bulk_p50_ms, bulk_p99_ms;        /* the others */
  double all_p50_ms, all_p99_ms;
  double elapsed_s;                       /* since the first submit */
} srcu_server_stats;

srcu_status srcu_server_create(const srcu_server_config *config, srcu_server **out);
void srcu_server_destroy(srcu_server *server);
/* Copies the request (host columns: x, y, z and at most one attribute) into
 * pinned memory and queues it.  SRCU_ERR_BUSY: the queue or the pinned arena
 * is full -- retry later. */
srcu_status srcu_server_submit(srcu_server *server, uint64_t req_id, const srcu_cloud *cloud,
                               const srcu_voxel_params *vparams,
                               const srcu_normal_params *nparams);
/* Returns one finished request, waiting up to wait_us; SRCU_ERR_BUSY if
 * none.  Its result columns live in the pinned arena until
 * srcu_server_release(req_id); unreleased results hold arena space. */
srcu_status srcu_server_poll(srcu_server *server, srcu_request_result *out, uint32_t wait_us);
srcu_status srcu_server_release(srcu_server *server, uint64_t req_id);
srcu_status srcu_server_stats_get(srcu_server *server, srcu_server_stats *stats);
/* Discards the latency history (e.g. after a warm-up phase). */
srcu_status srcu_server_stats_reset(srcu_server *server);

/* ---- launch accounting and kernel timing ---------------------------------- */

/* Kernel groups of the chain, in launch order. */
typedef enum srcu_kernel_id {
  SRCU_K_BEGIN = 0,      /* control-block reset */
  SRCU_K_BOUNDS,         /* per-axis min/max */
  SRCU_K_VOXEL_PLAN,     /* voxel-key packing plan */
  SRCU_K_VOXEL_HIST,     /* reserved: the histograms run inside SRCU_K_VOXEL_SORT */
  SRCU_K_VOXEL_SORT,     /* persistent onesweep sort of the voxel keys (histograms + passes) */
  SRCU_K_VOXEL_SEGMENTS, /* fused voxel segmentation + FP64 centroid reduction */
  SRCU_K_UNPACK_KEYS,    /* packed key -> (ix, iy, iz) */
  SRCU_K_CELL_PLAN,      /* radius-grid plan */
  SRCU_K_CELL_HIST,      /* reserved: the histograms run inside SRCU_K_CELL_SORT */
  SRCU_K_CELL_SORT,      /* persistent onesweep sort of the cell keys (histograms + passes) */
  SRCU_K_CELLS,          /* cell table + cell-sorted point records */
  SRCU_K_HASH,           /* cell hash table */
  SRCU_K_RANGES,         /* 3x3 neighbour column ranges */
  SRCU_K_NORMALS,        /* radius neighbours + covariance + eigensolve */
  SRCU_K_CLUSTER,        /* Euclidean clustering: union-find over the radius grid */
  SRCU_K_LAS_DECODE,     /* LAS point records -> columns */
  SRCU_K_RANSAC,         /* RANSAC plane hypotheses, scores, inlier mask and moments */
  SRCU_K_COUNT
} srcu_kernel_id;

typedef struct srcu_kernel_stat {
  char name[32];
  uint64_t launches;      /* kernel launches since the last reset */
  uint64_t timed_regions; /* launch groups timed with CUDA events (see srcu_profile_enable) */
  double total_ms;        /* summed event time of the timed groups */
} srcu_kernel_stat;

/* Times every launch group whose bit (1 << srcu_kernel_id) is set with a pair
 * of CUDA events on the context stream; 0 turns timing off.  Launch counting
 * is always on. */
srcu_status srcu_profile_enable(srcu_ctx *ctx, uint64_t timed_kernel_mask);
/* Synchronises, then fills up to max_entries stats (one per srcu_kernel_id)
 * and returns how many were written (negative on error).  reset != 0 clears
 * the counters afterwards. */
int srcu_profile_read(srcu_ctx *ctx, srcu_kernel_stat *out, int max_entries, int reset);

/* ---- allocation-free entry point ------------------------------------------ */

/* No counterpart in the reference.  For callers that cannot allocate device
 * memory once they are running: a real-time loop (a ROS 2 executor thread
 * handling each LiDAR frame) that must not allocate after start-up, or a host
 * application whose device memory belongs to another allocator that forbids
 * raw cudaMalloc.  It runs the centroid downsample of srcu_voxel_centroid
 * without a context and calls no cudaMalloc / cudaFree: its scratch (about
 * 4.6 MB) is one file-scope __device__ array that every GPU which loads this
 * library holds until the process exits.
 *  - At most SRCU_NOALLOC_MAX_POINTS points; larger clouds are rejected with
 *    SRCU_ERR_INVALID_ARGUMENT.
 *  - cloud and out must be device pointers (on_device = 1) on the current
 *    device; cuda_stream (NULL = legacy default stream) must belong to it.
 *  - The first call on each device performs one-time set-up (the scratch's
 *    device address and launch attributes); make that first call before any
 *    stream capture.
 *  - Every call uses the same scratch array and leaves its contents behind;
 *    calls that overlap on the GPU (different streams or host threads) race.
 *  - Synchronous: returns after the outputs are written.  Status codes only;
 *    no message is recorded. */
#define SRCU_NOALLOC_MAX_POINTS 131072
srcu_status srcu_voxel_centroid_noalloc(const srcu_cloud *cloud, const srcu_voxel_params *params,
                                        const srcu_voxel_out *out, uint64_t *out_voxels,
                                        void *cuda_stream);
/* Test hooks for the epoch restart of that scratch on the current device
 * (the same rule as srcu_debug_set_epoch / srcu_debug_get_epoch). */
srcu_status srcu_noalloc_debug_set_epoch(uint32_t epoch);
srcu_status srcu_noalloc_debug_get_epoch(uint32_t *epoch, uint64_t *restarts);

#ifdef __cplusplus
}
#endif

#endif /* SRCUDA_H */
