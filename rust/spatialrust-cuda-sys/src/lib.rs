//! Raw bindings to libsrcuda (`include/srcuda.h`): the C ABI of the B200 (sm_100a)
//! uniform-grid path -- VoxelGrid centroid downsample and radius-mode normals.
//!
//! Every declaration mirrors the header one for one (same names, field order and
//! widths); the repository's `tests/test_rust_binding_cpu.py` checks that.  The
//! safe wrapper and the `ExecutionPolicy::Gpu(DeviceKind::Cuda)` arms live in
//! `spatialrust-gpu-cuda`.  Status codes are plain `c_int`s: an out-of-range value
//! from a newer library must not become an invalid Rust enum.
#![allow(non_camel_case_types)]
#![no_std]

use core::ffi::{c_char, c_int, c_void};

pub type srcu_status = c_int;
pub type srcu_kernel_id = c_int;

// ---- constants (#define) ----
pub const SRCU_ABI_VERSION: c_int = 1;
pub const SRCU_VOXEL_CENTROID: c_int = 0;
pub const SRCU_VOXEL_APPROXIMATE_FIRST: c_int = 1;
pub const SRCU_VOXEL_CENTROID_XYZ: c_int = 2;
pub const SRCU_ATTRIBUTE_AVERAGE: c_int = 0;
pub const SRCU_ATTRIBUTE_FIRST: c_int = 1;
pub const SRCU_SORT_TUNING_MAX: c_int = 32;
pub const SRCU_SORT_VOXEL_KEYS: c_int = 0;
pub const SRCU_SORT_CELL_KEYS: c_int = 1;
pub const SRCU_SORT_BATCH_VOXEL_KEYS: c_int = 2;
pub const SRCU_SORT_BATCH_CELL_KEYS: c_int = 3;
pub const SRCU_SORT_KINDS: c_int = 4;
pub const SRCU_NOALLOC_MAX_POINTS: c_int = 131072;

// ---- srcu_status and srcu_kernel_id values ----
pub const SRCU_OK: c_int = 0;
pub const SRCU_ERR_INVALID_ARGUMENT: c_int = 1;
pub const SRCU_ERR_LENGTH_MISMATCH: c_int = 2;
pub const SRCU_ERR_UNSUPPORTED_DTYPE: c_int = 3;
pub const SRCU_ERR_MISSING_FIELD: c_int = 4;
pub const SRCU_ERR_OUT_OF_BUDGET: c_int = 5;
pub const SRCU_ERR_CUDA: c_int = 6;
pub const SRCU_ERR_TIMEOUT: c_int = 7;
pub const SRCU_ERR_KEY_OVERFLOW: c_int = 8;
pub const SRCU_ERR_NO_DEVICE: c_int = 9;
pub const SRCU_ERR_BUSY: c_int = 10;
pub const SRCU_K_BEGIN: c_int = 0;
pub const SRCU_K_BOUNDS: c_int = 1;
pub const SRCU_K_VOXEL_PLAN: c_int = 2;
pub const SRCU_K_VOXEL_HIST: c_int = 3;
pub const SRCU_K_VOXEL_SORT: c_int = 4;
pub const SRCU_K_VOXEL_SEGMENTS: c_int = 5;
pub const SRCU_K_UNPACK_KEYS: c_int = 6;
pub const SRCU_K_CELL_PLAN: c_int = 7;
pub const SRCU_K_CELL_HIST: c_int = 8;
pub const SRCU_K_CELL_SORT: c_int = 9;
pub const SRCU_K_CELLS: c_int = 10;
pub const SRCU_K_HASH: c_int = 11;
pub const SRCU_K_RANGES: c_int = 12;
pub const SRCU_K_NORMALS: c_int = 13;
pub const SRCU_K_CLUSTER: c_int = 14;
pub const SRCU_K_LAS_DECODE: c_int = 15;
pub const SRCU_K_RANSAC: c_int = 16;
pub const SRCU_K_COUNT: c_int = 17;

// ---- types ----
/// Opaque handle (`typedef struct srcu_ctx srcu_ctx;`).
#[repr(C)]
pub struct srcu_ctx {
    _p: [u8; 0],
}

#[repr(C)]
#[derive(Clone, Copy, Debug)]
pub struct srcu_cloud {
    pub x: *const f32,
    pub y: *const f32,
    pub z: *const f32,
    pub attrs: *const *const f32,
    pub n_attrs: u32,
    pub on_device: i32,
    pub n: u64,
    pub stride: u32,
    pub reserved: u32,
}

#[repr(C)]
#[derive(Clone, Copy, Debug)]
pub struct srcu_voxel_params {
    pub leaf_size: f32,
    pub has_origin: i32,
    pub origin: [f32; 3],
    pub mode: i32,
    pub attribute_policy: i32,
}

#[repr(C)]
#[derive(Clone, Copy, Debug)]
pub struct srcu_voxel_out {
    pub x: *mut f32,
    pub y: *mut f32,
    pub z: *mut f32,
    pub attrs: *const *mut f32,
    pub keys: *mut i64,
    pub counts: *mut u32,
    pub on_device: i32,
}

#[repr(C)]
#[derive(Clone, Copy, Debug)]
pub struct srcu_normal_params {
    pub radius: f32,
    pub min_neighbors: u32,
    pub has_viewpoint: i32,
    pub viewpoint: [f32; 3],
    pub include_self: i32,
    pub count_shell: i32,
}

#[repr(C)]
#[derive(Clone, Copy, Debug)]
pub struct srcu_normal_out {
    pub nx: *mut f32,
    pub ny: *mut f32,
    pub nz: *mut f32,
    pub curvature: *mut f32,
    pub neighbor_counts: *mut u32,
    pub on_device: i32,
}

#[repr(C)]
#[derive(Clone, Copy, Debug)]
pub struct srcu_normal_stats {
    pub valid_count: u64,
    pub invalid_count: u64,
    pub shell_points: u64,
    pub fp64_eigensolves: u64,
}

#[repr(C)]
#[derive(Clone, Copy, Debug)]
pub struct srcu_sort_config {
    pub items_per_thread: u32,
    pub blocks_per_sm: u32,
    pub digit_bits: u32,
    pub threads_per_block: u32,
}

#[repr(C)]
#[derive(Clone, Copy, Debug)]
pub struct srcu_plane_score {
    pub inlier_count: u32,
    pub normal: [f32; 3],
    pub d: f32,
}

#[repr(C)]
#[derive(Clone, Copy, Debug)]
pub struct srcu_ransac_params {
    pub distance_threshold: f32,
    pub max_iterations: u32,
    pub min_inliers: u64,
    pub seed: u64,
}

#[repr(C)]
#[derive(Clone, Copy, Debug)]
pub struct srcu_ransac_result {
    pub normal: [f32; 3],
    pub d: f32,
    pub inlier_count: u64,
    pub hypotheses: u32,
    pub best_hypothesis: u32,
    pub hypothesis_normal: [f32; 3],
    pub hypothesis_d: f32,
}

/// Opaque handle (`typedef struct srcu_stream_voxel srcu_stream_voxel;`).
#[repr(C)]
pub struct srcu_stream_voxel {
    _p: [u8; 0],
}

#[repr(C)]
#[derive(Clone, Copy, Debug)]
pub struct srcu_stream_voxel_params {
    pub leaf_size: f32,
    pub n_attrs: u32,
    pub attr_f64_mask: u32,
    pub device_run_points: u32,
    pub run_points: u64,
    pub max_runs: u64,
    pub spool_limit_bytes: u64,
}

#[repr(C)]
#[derive(Clone, Copy, Debug)]
pub struct srcu_stream_voxel_info {
    pub points: u64,
    pub finite_points: u64,
    pub runs: u64,
    pub spool_bytes: u64,
    pub device_runs: u64,
    pub partial_records: u64,
    pub voxels: u64,
}

#[repr(C)]
#[derive(Clone, Copy, Debug)]
pub struct srcu_stream_voxel_out {
    pub x: *mut f32,
    pub y: *mut f32,
    pub z: *mut f32,
    pub attrs: *const *mut f64,
    pub keys: *mut i64,
    pub counts: *mut u64,
    pub on_device: i32,
}

#[repr(C)]
#[derive(Clone, Copy, Debug)]
pub struct srcu_las_format {
    pub point_format: u32,
    pub record_length: u32,
    pub scale: [f64; 3],
    pub offset: [f64; 3],
    pub has_origin: i32,
    pub reserved: i32,
    pub origin: [f64; 3],
}

#[repr(C)]
#[derive(Clone, Copy, Debug)]
pub struct srcu_las_out {
    pub x: *mut f32,
    pub y: *mut f32,
    pub z: *mut f32,
    pub intensity: *mut f32,
    pub classification: *mut u8,
    pub gps_time: *mut f64,
    pub red: *mut u16,
    pub green: *mut u16,
    pub blue: *mut u16,
    pub on_device: i32,
}

/// Opaque handle (`typedef struct srcu_graph srcu_graph;`).
#[repr(C)]
pub struct srcu_graph {
    _p: [u8; 0],
}

#[repr(C)]
#[derive(Clone, Copy, Debug)]
pub struct srcu_frame_view {
    pub x: *const f32,
    pub y: *const f32,
    pub z: *const f32,
    pub attrs: *const *const f32,
    pub nx: *const f32,
    pub ny: *const f32,
    pub nz: *const f32,
    pub curvature: *const f32,
    pub counts: *const u32,
    pub voxel_count: *const u64,
    pub n_attrs: u32,
}

#[repr(C)]
#[derive(Clone, Copy, Debug)]
pub struct srcu_chain_info {
    pub points: u64,
    pub voxels: u64,
    pub cells: u64,
    pub voxel_key_bits: u32,
    pub cell_key_bits: u32,
    pub voxel_sort_passes: u32,
    pub cell_sort_passes: u32,
    pub cell_size: f64,
}

/// Opaque handle (`typedef struct srcu_server srcu_server;`).
#[repr(C)]
pub struct srcu_server {
    _p: [u8; 0],
}

#[repr(C)]
#[derive(Clone, Copy, Debug)]
pub struct srcu_server_config {
    pub device: i32,
    pub hbm_budget_bytes: u64,
    pub frame_slots: u32,
    pub bulk_slots: u32,
    pub frame_batch_points: u64,
    pub bulk_threshold_points: u64,
    pub bulk_max_points: u64,
    pub max_pending_points: u64,
    pub host_arena_bytes: u64,
}

#[repr(C)]
#[derive(Clone, Copy, Debug)]
pub struct srcu_request_result {
    pub req_id: u64,
    pub status: srcu_status,
    pub points: u64,
    pub voxels: u64,
    pub x: *const f32,
    pub y: *const f32,
    pub z: *const f32,
    pub intensity: *const f32,
    pub nx: *const f32,
    pub ny: *const f32,
    pub nz: *const f32,
    pub curvature: *const f32,
    pub counts: *const u32,
    pub latency_ms: f64,
}

#[repr(C)]
#[derive(Clone, Copy, Debug)]
pub struct srcu_server_stats {
    pub submitted: u64,
    pub rejected: u64,
    pub completed: u64,
    pub failed: u64,
    pub batches: u64,
    pub points: u64,
    pub frame_p50_ms: f64,
    pub frame_p99_ms: f64,
    pub bulk_p50_ms: f64,
    pub bulk_p99_ms: f64,
    pub all_p50_ms: f64,
    pub all_p99_ms: f64,
    pub elapsed_s: f64,
}

#[repr(C)]
#[derive(Clone, Copy, Debug)]
pub struct srcu_kernel_stat {
    pub name: [c_char; 32],
    pub launches: u64,
    pub timed_regions: u64,
    pub total_ms: f64,
}

extern "C" {
    pub fn srcu_abi_version() -> c_int;
    /// Creates a context on CUDA device `device`.
    pub fn srcu_create(device: i32, hbm_budget_bytes: u64, out: *mut *mut srcu_ctx) -> srcu_status;
    pub fn srcu_destroy(ctx: *mut srcu_ctx);
    pub fn srcu_last_error(ctx: *const srcu_ctx) -> *const c_char;
    /// The element counts behind the last SRCU_ERR_LENGTH_MISMATCH on this context (SpatialError::BufferLengthMismatch { expected, found }, ...
    pub fn srcu_last_length_mismatch(ctx: *const srcu_ctx, expected: *mut u64, found: *mut u64) -> srcu_status;
    /// Runs subsequent work on a caller stream (a cudaStream_t); NULL restores the context's own stream.
    pub fn srcu_set_stream(ctx: *mut srcu_ctx, cuda_stream: *mut c_void) -> srcu_status;
    pub fn srcu_synchronize(ctx: *mut srcu_ctx) -> srcu_status;
    /// Device bytes currently held by the context.
    pub fn srcu_device_bytes(ctx: *const srcu_ctx) -> u64;
    /// VoxelGridDownsample::filter_with_policy(cloud, Gpu(Cuda)) for Centroid + Average (voxel.rs:213-237, 251-368, 464-540):
    pub fn srcu_voxel_centroid(ctx: *mut srcu_ctx, cloud: *const srcu_cloud, params: *const srcu_voxel_params, out: *const srcu_voxel_out, out_voxels: *mut u64) -> srcu_status;
    /// NormalEstimator::estimate_with_policy(cloud, Gpu(Cuda)) with search_radius = Some(r) (normal.rs:102-164, 321-573), or, with include_self = 1, ...
    pub fn srcu_radius_normals(ctx: *mut srcu_ctx, cloud: *const srcu_cloud, params: *const srcu_normal_params, out: *const srcu_normal_out, stats: *mut srcu_normal_stats) -> srcu_status;
    /// MvpPipeline voxel -> normals chain (crates/spatialrust-pipeline/src/mvp.rs:193-226):
    pub fn srcu_voxel_normals(ctx: *mut srcu_ctx, cloud: *const srcu_cloud, vparams: *const srcu_voxel_params, nparams: *const srcu_normal_params, vout: *const srcu_voxel_out, nout: *const srcu_normal_out, out_voxels: *mut u64, stats: *mut srcu_normal_stats) -> srcu_status;
    /// Connected-component roots of the graph "dx dx + dy dy + dz dz <= tol tol" (f32):
    pub fn srcu_euclidean_cluster_roots(ctx: *mut srcu_ctx, cloud: *const srcu_cloud, cluster_tolerance: f32, roots: *mut u32) -> srcu_status;
    /// Replaces spatialrust_gpu::estimate_plane_covariances_grid_gpu (crates/spatialrust-gpu/src/kernels/covariances_grid.rs:216-364), which ...
    pub fn srcu_plane_covariances(ctx: *mut srcu_ctx, cloud: *const srcu_cloud, radius: f32, epsilon: f32, cov: *mut f32, stats: *mut srcu_normal_stats) -> srcu_status;
    /// Fills up to max_entries shapes; returns how many the library has.
    pub fn srcu_sort_configs(out: *mut srcu_sort_config, max_entries: i32) -> i32;
    /// Entry k of the `kind` table:
    pub fn srcu_set_sort_tuning(ctx: *mut srcu_ctx, kind: i32, max_points: *const u64, config: *const i32, count: u32) -> srcu_status;
    /// count:
    pub fn srcu_get_sort_tuning(ctx: *mut srcu_ctx, kind: i32, max_points: *mut u64, config: *mut i32, count: *mut u32) -> srcu_status;
    /// The normals kernel's neighbour gather:
    pub fn srcu_set_neighbor_staging(ctx: *mut srcu_ctx, mode: i32) -> srcu_status;
    pub fn srcu_get_neighbor_staging(ctx: *mut srcu_ctx) -> i32;
    /// No counterpart in the reference.
    pub fn srcu_selftest_bounded_wait(ctx: *mut srcu_ctx, max_polls: u32) -> srcu_status;
    /// No counterpart in the reference.
    pub fn srcu_debug_set_epoch(ctx: *mut srcu_ctx, epoch: u32) -> srcu_status;
    pub fn srcu_debug_get_epoch(ctx: *mut srcu_ctx, epoch: *mut u32, restarts: *mut u64) -> srcu_status;
    /// Replaces score_ransac_plane_hypotheses_gpu (ransac_plane.rs:104-263):
    pub fn srcu_ransac_plane_scores(ctx: *mut srcu_ctx, cloud: *const srcu_cloud, hypotheses: *const u32, count: u32, distance_threshold: f32, scores: *mut srcu_plane_score) -> srcu_status;
    /// The Gpu(Cuda) arm of RansacPlaneSegmenter::segment_with_policy (plane.rs:
    pub fn srcu_ransac_plane_segment(ctx: *mut srcu_ctx, cloud: *const srcu_cloud, params: *const srcu_ransac_params, result: *mut srcu_ransac_result, inlier_mask: *mut u8) -> srcu_status;
    pub fn srcu_stream_voxel_create(ctx: *mut srcu_ctx, params: *const srcu_stream_voxel_params, out: *mut *mut srcu_stream_voxel) -> srcu_status;
    /// Appends one chunk (packed columns, host or device; stride must be 0 or 1).
    pub fn srcu_stream_voxel_push(sv: *mut srcu_stream_voxel, chunk: *const srcu_cloud) -> srcu_status;
    /// Reduces the last run and merges every run; info is nullable.
    pub fn srcu_stream_voxel_finish(sv: *mut srcu_stream_voxel, info: *mut srcu_stream_voxel_info) -> srcu_status;
    /// Copies voxels [first, first + count) of the finished stream.
    pub fn srcu_stream_voxel_fetch(sv: *mut srcu_stream_voxel, first: u64, count: u64, out: *const srcu_stream_voxel_out) -> srcu_status;
    /// Ends a stream.
    pub fn srcu_stream_voxel_destroy(sv: *mut srcu_stream_voxel);
    /// Decodes n uncompressed LAS point records (records:
    pub fn srcu_las_decode(ctx: *mut srcu_ctx, records: *const c_void, n: u64, records_on_device: i32, fmt: *const srcu_las_format, out: *const srcu_las_out) -> srcu_status;
    /// Enqueues voxel -> normals for `count` clouds in one chain:
    pub fn srcu_batch_voxel_normals_enqueue(ctx: *mut srcu_ctx, points: *const srcu_cloud, offsets: *const u64, count: u32, vparams: *const srcu_voxel_params, nparams: *const srcu_normal_params) -> srcu_status;
    /// Synchronises and copies the count + 1 voxel offsets of the last batch.
    pub fn srcu_batch_voxel_offsets(ctx: *mut srcu_ctx, voxel_offsets: *mut u64) -> srcu_status;
    /// Captures the voxel -> normals chain for these exact inputs (a batch when offsets is non-NULL, else one cloud) as a CUDA graph on the context stream.
    pub fn srcu_chain_graph_create(ctx: *mut srcu_ctx, points: *const srcu_cloud, offsets: *const u64, count: u32, vparams: *const srcu_voxel_params, nparams: *const srcu_normal_params, out: *mut *mut srcu_graph) -> srcu_status;
    pub fn srcu_graph_launch(ctx: *mut srcu_ctx, graph: *mut srcu_graph) -> srcu_status;
    pub fn srcu_graph_destroy(graph: *mut srcu_graph);
    /// Enqueues the voxel -> normals chain on the context stream for a cloud already on the device, without any host synchronisation; results stay in ...
    pub fn srcu_voxel_normals_enqueue(ctx: *mut srcu_ctx, cloud: *const srcu_cloud, vparams: *const srcu_voxel_params, nparams: *const srcu_normal_params) -> srcu_status;
    /// The voxel stage alone (VoxelGridDownsample on a device-resident cloud): bounds, key plan,
    /// sort and the fused segment reduction, enqueued without host synchronisation.
    pub fn srcu_voxel_centroid_enqueue(ctx: *mut srcu_ctx, cloud: *const srcu_cloud, vparams: *const srcu_voxel_params) -> srcu_status;
    /// Device pointers of the last enqueued chain's results.
    pub fn srcu_frame_view_get(ctx: *mut srcu_ctx, view: *mut srcu_frame_view) -> srcu_status;
    /// Synchronises and checks the device status word of the last enqueue.
    pub fn srcu_frame_check(ctx: *mut srcu_ctx, out_voxels: *mut u64, stats: *mut srcu_normal_stats) -> srcu_status;
    pub fn srcu_chain_info_get(ctx: *mut srcu_ctx, info: *mut srcu_chain_info) -> srcu_status;
    /// Explicit read-back of the last enqueued chain (GpuSpatialFrame readback, gpu_frame.rs:292-328):
    pub fn srcu_frame_fetch(ctx: *mut srcu_ctx, vout: *const srcu_voxel_out, nout: *const srcu_normal_out, out_voxels: *mut u64, stats: *mut srcu_normal_stats) -> srcu_status;
    pub fn srcu_server_create(config: *const srcu_server_config, out: *mut *mut srcu_server) -> srcu_status;
    pub fn srcu_server_destroy(server: *mut srcu_server);
    /// Copies the request (host columns:
    pub fn srcu_server_submit(server: *mut srcu_server, req_id: u64, cloud: *const srcu_cloud, vparams: *const srcu_voxel_params, nparams: *const srcu_normal_params) -> srcu_status;
    /// Returns one finished request, waiting up to wait_us; SRCU_ERR_BUSY if none.
    pub fn srcu_server_poll(server: *mut srcu_server, out: *mut srcu_request_result, wait_us: u32) -> srcu_status;
    pub fn srcu_server_release(server: *mut srcu_server, req_id: u64) -> srcu_status;
    pub fn srcu_server_stats_get(server: *mut srcu_server, stats: *mut srcu_server_stats) -> srcu_status;
    /// Discards the latency history (e.g.
    pub fn srcu_server_stats_reset(server: *mut srcu_server) -> srcu_status;
    /// Times every launch group whose bit (1 << srcu_kernel_id) is set with a pair of CUDA events on the context stream; 0 turns timing off.
    pub fn srcu_profile_enable(ctx: *mut srcu_ctx, timed_kernel_mask: u64) -> srcu_status;
    /// Synchronises, then fills up to max_entries stats (one per srcu_kernel_id) and returns how many were written (negative on error).
    pub fn srcu_profile_read(ctx: *mut srcu_ctx, out: *mut srcu_kernel_stat, max_entries: i32, reset: i32) -> i32;
    /// No counterpart in the reference.
    pub fn srcu_voxel_centroid_noalloc(cloud: *const srcu_cloud, params: *const srcu_voxel_params, out: *const srcu_voxel_out, out_voxels: *mut u64, cuda_stream: *mut c_void) -> srcu_status;
    /// Test hooks for the epoch restart of that scratch on the current device (the same rule as srcu_debug_set_epoch / srcu_debug_get_epoch).
    pub fn srcu_noalloc_debug_set_epoch(epoch: u32) -> srcu_status;
    pub fn srcu_noalloc_debug_get_epoch(epoch: *mut u32, restarts: *mut u64) -> srcu_status;
}
