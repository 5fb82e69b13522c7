// srcuda.cu -- host layer and C ABI (include/srcuda.h) of the sm_100a
// uniform-grid path: context, HBM-budgeted buffer pool, chain launches.
#include <cuda_runtime.h>

#include <algorithm>
#include <cstdarg>
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>

#include "../../include/srcuda.h"
#include "cluster.cuh"
#include "host_copy.h"
#include "normals.cuh"
#include "sort_tuning.h"
#include "voxel.cuh"

using namespace srcu;

namespace {

struct DevBuf {
  void *p = nullptr;
  size_t bytes = 0;
};

}  // namespace

struct srcu_ctx {
  int device = 0;
  int num_sms = 148;
  cudaStream_t own_stream = nullptr;
  cudaStream_t stream = nullptr;
  uint64_t budget = 0;  // 0 = unlimited
  uint64_t used = 0;
  std::string err;
  Control *ctl = nullptr;       // device
  Control *ctl_host = nullptr;  // pinned mirror for read-back
  // Host mirror of ctl->epoch (epoch_guard), restarts of it, and whether a
  // chain is being captured into a graph (its epoch advances at launch).
  uint32_t epoch_host = 0;
  uint64_t epoch_restarts = 0;
  bool capturing = false;
  // the counts behind the last SRCU_ERR_LENGTH_MISMATCH (srcu_last_length_mismatch)
  uint64_t mismatch_expected = 0, mismatch_found = 0;
  // pinned staging ring for copies from and to pageable host memory (host_copy.h)
  unsigned char *ring[3] = {nullptr, nullptr, nullptr};
  cudaEvent_t ring_ev[3] = {nullptr, nullptr, nullptr};
  int ring_next = 0;
  // Side stream for read-backs that overlap later kernels of the same chain,
  // the event that releases them, and a pinned copy of the control-block head
  // (epoch, status, point and voxel counts) read once the voxel stage is done.
  cudaStream_t side_stream = nullptr;
  cudaEvent_t ev_voxel = nullptr;
  unsigned char *head_host = nullptr;
  int occ_normals = 1, occ_normals_staged = 1, occ_normals_packed = 1, occ_seg = 1, occ_cells = 1;
  int neighbor_staging = 0;  // k_normals' neighbour walk: WALK_L1, WALK_STAGED or WALK_PACKED
  // co-resident blocks per SM of each sort launch shape, voxel-key and cell-key sorts
  int occ_sort_v[SORT_CONFIGS] = {}, occ_sort_c[SORT_CONFIGS] = {};
  // sort launch shape by input size, per sort kind (SRCU_SORT_VOXEL_KEYS ..
  // SRCU_SORT_BATCH_CELL_KEYS; sort_tuning.h, srcu_set_sort_tuning)
  uint64_t tune_max_points[SRCU_SORT_KINDS][SRCU_SORT_TUNING_MAX] = {};
  int32_t tune_config[SRCU_SORT_KINDS][SRCU_SORT_TUNING_MAX] = {};
  uint32_t tune_count[SRCU_SORT_KINDS] = {};
  // input staging (host inputs are copied here)
  DevBuf in[MAX_COLS];
  // sort
  DevBuf keys[2], vals[2], lb_sort, lb_seg, lb_cells;
  // voxel outputs: x, y, z, attrs..., packed keys, counts, unpacked keys
  DevBuf vout[MAX_COLS], vkeys, vcounts, vkeys3, vaos;
  // plain-xyz path: gathered voxels (x, y, z, counts, keys) and first points
  DevBuf xyz_tmp;
  bool xyz_order = false;  // this chain emits voxels in first-seen order (plain xyz)
  int occ_sort_order = 1;
  DevBuf in_aos;  // AoS (x, y, z, first attribute) copy of the chain's input
  // radius grid
  DevBuf pts, pt_cell, cell_key, cell_start, table, ranges;
  uint32_t table_log2 = 0;
  // normals outputs
  DevBuf nout[4], ncounts;
  DevBuf parent;  // union-find parents (Euclidean clustering)
  DevBuf cov6;    // plane-regularised covariances, 6 floats per point
  DevBuf stage_block;  // host interleaved records, copied once before deinterleaving
  // the buffers of the last destroyed streaming voxel, kept for the next one
  srcu_stream_voxel *parked_stream = nullptr;
  // RANSAC plane scoring: hypotheses, planes, validity, counts, block partials, mask
  DevBuf rs_hyp, rs_planes, rs_valid, rs_counts, rs_partials, rs_mask;
  uint32_t last_attrs = 0;  // attribute count of the last enqueued chain
  const float *frame_attr_ptrs[MAX_COLS] = {};
  // batch arrays (clouds of the last chain) and pinned staging for their parameters
  DevBuf b_offsets, b_bounds, b_vplans, b_cplans, b_vparams, b_nparams, b_voff;
  uint32_t batch_cap = 0;
  uint32_t last_clouds = 1;
  int32_t agg_all = AGG_FAST;  // the chain's voxel aggregation when every cloud shares it, else -1
  bool count_shell = true;     // some cloud of the chain reports shell points
  unsigned char *h_stage[2] = {nullptr, nullptr};
  size_t h_stage_bytes[2] = {0, 0};
  cudaEvent_t h_stage_ev[2] = {nullptr, nullptr};
  int h_stage_next = 0;
  // launch accounting / CUDA-event timing per kernel group (srcu_profile_*)
  uint64_t prof_mask = 0;
  uint64_t launches[SRCU_K_COUNT] = {};
  uint64_t timed[SRCU_K_COUNT] = {};
  double timed_ms[SRCU_K_COUNT] = {};
  std::vector<cudaEvent_t> ev_pool;     // 2 per pending region
  std::vector<int> ev_pending;          // kernel id per pending region
};

// Frees a streaming voxel and its buffers (stream.cu).
void stream_voxel_free(srcu_stream_voxel *sv);

namespace {

srcu_status fail(srcu_ctx *c, srcu_status st, const char *fmt, ...) {
  if (c) c->mismatch_expected = c->mismatch_found = 0;
  char buf[512];
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(buf, sizeof(buf), fmt, ap);
  va_end(ap);
  if (c) c->err = buf;
  return st;
}

#define CU_TRY(expr)                                                                     \
  do {                                                                                   \
    cudaError_t e_ = (expr);                                                             \
    if (e_ != cudaSuccess)                                                               \
      return fail(ctx, SRCU_ERR_CUDA, "%s failed: %s", #expr, cudaGetErrorString(e_));   \
  } while (0)

#define ST_TRY(expr)                 \
  do {                               \
    srcu_status s_ = (expr);         \
    if (s_ != SRCU_OK) return s_;    \
  } while (0)

// Grows a device buffer to at least `bytes` (contents are not preserved).
srcu_status ensure(srcu_ctx *ctx, DevBuf &b, size_t bytes, bool zero = false) {
  if (bytes == 0) bytes = 16;
  if (b.bytes >= bytes) return SRCU_OK;
  size_t want = std::max(bytes, b.bytes + b.bytes / 4);  // amortise growth
  want = (want + 255) & ~size_t(255);
  if (ctx->budget && ctx->used - b.bytes + want > ctx->budget) {
    want = (bytes + 255) & ~size_t(255);
    if (ctx->used - b.bytes + want > ctx->budget)
      return fail(ctx, SRCU_ERR_OUT_OF_BUDGET,
                  "device allocation of %zu bytes exceeds the HBM budget (%llu of %llu bytes in use)",
                  want, (unsigned long long)ctx->used, (unsigned long long)ctx->budget);
  }
  if (b.p) {
    CU_TRY(cudaStreamSynchronize(ctx->stream));
    CU_TRY(cudaFree(b.p));
    ctx->used -= b.bytes;
    b.p = nullptr;
    b.bytes = 0;
  }
  void *p = nullptr;
  cudaError_t e = cudaMalloc(&p, want);
  if (e != cudaSuccess) {
    cudaGetLastError();
    return fail(ctx, SRCU_ERR_OUT_OF_BUDGET, "cudaMalloc(%zu) failed: %s", want, cudaGetErrorString(e));
  }
  if (zero) CU_TRY(cudaMemsetAsync(p, 0, want, ctx->stream));
  b.p = p;
  b.bytes = want;
  ctx->used += want;
  return SRCU_OK;
}

// ---- host <-> device copies of pageable host memory ---------------------------
// Chunks of kRingChunk bytes through the context's ring of pinned buffers: the
// host-side copy of a chunk (split over HostCopyPool's threads) overlaps the
// DMA of the previous chunk.  Pinned memory and small copies go straight to
// cudaMemcpyAsync.
constexpr size_t kRingChunk = size_t(4) << 20;
constexpr int kRingSlots = 3;
constexpr size_t kRingMin = size_t(1) << 20;

srcu_status ring_ready(srcu_ctx *ctx) {
  if (ctx->ring[0]) return SRCU_OK;
  for (int k = 0; k < kRingSlots; ++k) {
    CU_TRY(cudaMallocHost(reinterpret_cast<void **>(&ctx->ring[k]), kRingChunk));
    CU_TRY(cudaEventCreateWithFlags(&ctx->ring_ev[k], cudaEventDisableTiming));
  }
  return SRCU_OK;
}

// Host -> device, ordered on `stream`; returns once the source has been read.
srcu_status host_to_device(srcu_ctx *ctx, void *dst, const void *src, size_t bytes,
                           cudaStream_t stream) {
  if (bytes < kRingMin || !is_pageable(src)) {
    CU_TRY(cudaMemcpyAsync(dst, src, bytes, cudaMemcpyHostToDevice, stream));
    return SRCU_OK;
  }
  ST_TRY(ring_ready(ctx));
  for (size_t off = 0; off < bytes; off += kRingChunk) {
    const size_t len = std::min(kRingChunk, bytes - off);
    const int slot = ctx->ring_next;
    ctx->ring_next = (slot + 1) % kRingSlots;
    CU_TRY(cudaEventSynchronize(ctx->ring_ev[slot]));  // the slot's last DMA is done
    HostCopyPool::get().copy(ctx->ring[slot], static_cast<const char *>(src) + off, len);
    CU_TRY(cudaMemcpyAsync(static_cast<char *>(dst) + off, ctx->ring[slot], len,
                           cudaMemcpyHostToDevice, stream));
    CU_TRY(cudaEventRecord(ctx->ring_ev[slot], stream));
  }
  return SRCU_OK;
}

// Device -> host, ordered on `stream`.  Pageable destinations are complete on
// return (as a driver-staged copy would be); pinned ones when the stream is.
srcu_status device_to_host(srcu_ctx *ctx, void *dst, const void *src, size_t bytes,
                           cudaStream_t stream) {
  if (bytes < kRingMin || !is_pageable(dst)) {
    CU_TRY(cudaMemcpyAsync(dst, src, bytes, cudaMemcpyDeviceToHost, stream));
    return SRCU_OK;
  }
  ST_TRY(ring_ready(ctx));
  int pend = -1;
  size_t pend_off = 0, pend_len = 0;
  for (size_t off = 0;; off += kRingChunk) {
    const bool more = off < bytes;
    int slot = -1;
    size_t len = 0;
    if (more) {
      len = std::min(kRingChunk, bytes - off);
      slot = ctx->ring_next;
      ctx->ring_next = (slot + 1) % kRingSlots;
      CU_TRY(cudaEventSynchronize(ctx->ring_ev[slot]));
      CU_TRY(cudaMemcpyAsync(ctx->ring[slot], static_cast<const char *>(src) + off, len,
                             cudaMemcpyDeviceToHost, stream));
      CU_TRY(cudaEventRecord(ctx->ring_ev[slot], stream));
    }
    if (pend >= 0) {  // the previous chunk, while this one's DMA runs
      CU_TRY(cudaEventSynchronize(ctx->ring_ev[pend]));
      HostCopyPool::get().copy(static_cast<char *>(dst) + pend_off, ctx->ring[pend], pend_len);
    }
    if (!more) break;
    pend = slot;
    pend_off = off;
    pend_len = len;
  }
  return SRCU_OK;
}

void release(srcu_ctx *ctx, DevBuf &b) {
  if (b.p) {
    cudaFree(b.p);
    ctx->used -= b.bytes;
  }
  b.p = nullptr;
  b.bytes = 0;
}

template <class T>
T *ptr(DevBuf &b) {
  return static_cast<T *>(b.p);
}

uint32_t ceil_div(uint64_t a, uint64_t b) { return uint32_t((a + b - 1) / b); }

const char *const kKernelNames[SRCU_K_COUNT] = {
    "k_begin",          "k_bounds",        "k_voxel_plan",  "(in k_sort<voxel>)",
    "k_sort<voxel>",    "k_voxel_segments", "k_unpack_voxel_keys", "k_cell_plan",
    "(in k_sort<cell>)", "k_sort<cell>",    "k_cells",       "k_column_insert",
    "k_ranges",         "k_normals",       "k_cluster_union", "k_las_decode",
    "k_ransac_score"};

// Counts the launches of one kernel group and, when its bit is set in
// prof_mask, brackets them with CUDA events on the context stream.
struct Launch {
  srcu_ctx *ctx;
  int id;
  bool timed;
  cudaEvent_t stop = nullptr;
  Launch(srcu_ctx *c, int kid, uint64_t count = 1) : ctx(c), id(kid) {
    ctx->launches[id] += count;
    timed = (ctx->prof_mask >> id) & 1u;
    if (!timed) return;
    const size_t need = 2 * (ctx->ev_pending.size() + 1);
    while (ctx->ev_pool.size() < need) {
      cudaEvent_t e;
      if (cudaEventCreate(&e) != cudaSuccess) {
        timed = false;
        return;
      }
      ctx->ev_pool.push_back(e);
    }
    const size_t slot = ctx->ev_pending.size();
    ctx->ev_pending.push_back(id);
    cudaEventRecord(ctx->ev_pool[2 * slot], ctx->stream);
    stop = ctx->ev_pool[2 * slot + 1];
  }
  ~Launch() {
    if (timed) cudaEventRecord(stop, ctx->stream);
  }
};

uint32_t log2_ceil(uint64_t v) {
  uint32_t l = 0;
  while ((1ull << l) < v) ++l;
  return l;
}

srcu_status check_cloud(srcu_ctx *ctx, const srcu_cloud *cloud) {
  if (!cloud) return fail(ctx, SRCU_ERR_INVALID_ARGUMENT, "cloud is NULL");
  if (cloud->n > LB_MAX_COUNT)
    return fail(ctx, SRCU_ERR_INVALID_ARGUMENT, "cloud has %llu points; the limit is %llu",
                (unsigned long long)cloud->n, (unsigned long long)LB_MAX_COUNT);
  if (cloud->n_attrs > MAX_COLS - 3)
    return fail(ctx, SRCU_ERR_INVALID_ARGUMENT, "at most %d attribute columns are supported",
                MAX_COLS - 3);
  if (cloud->n > 0 && (!cloud->x || !cloud->y || !cloud->z))
    return fail(ctx, SRCU_ERR_MISSING_FIELD, "position column is NULL");
  for (uint32_t a = 0; a < cloud->n_attrs; ++a)
    if (cloud->n > 0 && (!cloud->attrs || !cloud->attrs[a]))
      return fail(ctx, SRCU_ERR_MISSING_FIELD, "attribute column %u is NULL", a);
  if (cloud->stride > 64)
    return fail(ctx, SRCU_ERR_INVALID_ARGUMENT, "stride %u exceeds 64 f32 elements", cloud->stride);
  return SRCU_OK;
}

bool strided(const srcu_cloud *cloud) { return cloud->stride > 1; }

// Host input, or interleaved records: the columns are staged in ctx->in[].
bool needs_staging(const srcu_cloud *cloud) { return !cloud->on_device || strided(cloud); }

// Buffers for a chain over n points with `cols` columns.
srcu_status reserve(srcu_ctx *ctx, uint64_t n, uint32_t cols, bool host_input, bool voxel,
                    bool normals) {
  const uint64_t m = std::max<uint64_t>(n, 1);
  if (host_input)
    for (uint32_t c = 0; c < cols; ++c) ST_TRY(ensure(ctx, ctx->in[c], m * 4));
  ST_TRY(ensure(ctx, ctx->keys[0], m * 8));
  ST_TRY(ensure(ctx, ctx->keys[1], m * 8));
  ST_TRY(ensure(ctx, ctx->vals[0], m * 4));
  ST_TRY(ensure(ctx, ctx->vals[1], m * 4));
  // Sort look-back words: a launch shape with tiles of T keys and B digit bins
  // writes ceil(m / T) * B words, and B / T <= RADIX_BINS / SORT_MIN_TILE
  // (lookback_fits), so this covers every shape up to one tile's rounding.
  ST_TRY(ensure(ctx, ctx->lb_sort,
                (size_t(ceil_div(m, SORT_MIN_TILE)) * RADIX_BINS + MAX_RADIX_BINS) * 8, true));
  ST_TRY(ensure(ctx, ctx->in_aos, m * 16));
  if (voxel) {
    ST_TRY(ensure(ctx, ctx->vaos, m * 16));
    ST_TRY(ensure(ctx, ctx->lb_seg, size_t(ceil_div(m, SEG_TILE)) * 8, true));
    for (uint32_t c = 0; c < cols; ++c) ST_TRY(ensure(ctx, ctx->vout[c], m * 4));
    ST_TRY(ensure(ctx, ctx->vkeys, m * 8));
    ST_TRY(ensure(ctx, ctx->vcounts, m * 4));
  }
  if (normals) {
    ST_TRY(ensure(ctx, ctx->lb_cells, size_t(ceil_div(m, CELL_TILE)) * 8, true));
    ST_TRY(ensure(ctx, ctx->pts, m * 16));
    ST_TRY(ensure(ctx, ctx->pt_cell, m * 4));
    ST_TRY(ensure(ctx, ctx->cell_key, m * 8));
    ST_TRY(ensure(ctx, ctx->cell_start, (m + 1) * 4));
    ST_TRY(ensure(ctx, ctx->ranges, m * 9 * sizeof(uint2)));
    const uint32_t l2 = std::max<uint32_t>(log2_ceil(2 * m), 4);
    const size_t tbytes = (size_t(1) << l2) * 8;
    if (ctx->table.bytes < tbytes || ctx->table_log2 == 0) {
      ST_TRY(ensure(ctx, ctx->table, tbytes, true));
    }
    // use the whole allocation (a power of two no smaller than 2m)
    uint32_t have = 4;
    while ((size_t(1) << (have + 1)) * 8 <= ctx->table.bytes) ++have;
    ctx->table_log2 = have;
    for (int c = 0; c < 4; ++c) ST_TRY(ensure(ctx, ctx->nout[c], m * 4));
    ST_TRY(ensure(ctx, ctx->ncounts, m * 4));
  }
  return SRCU_OK;
}

srcu_status stage_input(srcu_ctx *ctx, const srcu_cloud *cloud, const float **cols) {
  const uint32_t nc = 3 + cloud->n_attrs;
  const float *src[MAX_COLS] = {cloud->x, cloud->y, cloud->z};
  for (uint32_t a = 0; a < cloud->n_attrs; ++a) src[3 + a] = cloud->attrs[a];
  if (strided(cloud)) {
    // Interleaved records: deinterleave into the staged columns on the device
    // (from a copy of the record block when it lives in host memory).
    Interleaved iv{};
    iv.nc = nc;
    iv.stride = cloud->stride;
    if (cloud->on_device) {
      for (uint32_t c = 0; c < nc; ++c) iv.src[c] = src[c];
    } else if (cloud->n) {
      uintptr_t base = reinterpret_cast<uintptr_t>(src[0]), top = base;
      for (uint32_t c = 1; c < nc; ++c) {
        base = std::min(base, reinterpret_cast<uintptr_t>(src[c]));
        top = std::max(top, reinterpret_cast<uintptr_t>(src[c]));
      }
      for (uint32_t c = 0; c < nc; ++c) {
        const uintptr_t off = reinterpret_cast<uintptr_t>(src[c]) - base;
        if (off % 4 != 0 || off / 4 >= cloud->stride)
          return fail(ctx, SRCU_ERR_INVALID_ARGUMENT,
                      "interleaved host columns must be fields of one record array");
      }
      const size_t floats = size_t(cloud->n - 1) * cloud->stride + (top - base) / 4 + 1;
      ST_TRY(ensure(ctx, ctx->stage_block, floats * 4));
      ST_TRY(host_to_device(ctx, ctx->stage_block.p, reinterpret_cast<const void *>(base),
                            floats * 4, ctx->stream));
      for (uint32_t c = 0; c < nc; ++c)
        iv.src[c] = ptr<const float>(ctx->stage_block) +
                    (reinterpret_cast<uintptr_t>(src[c]) - base) / 4;
    }
    for (uint32_t c = 0; c < nc; ++c) {
      iv.dst[c] = ptr<float>(ctx->in[c]);
      cols[c] = ptr<const float>(ctx->in[c]);
    }
    if (cloud->n) {
      const uint32_t grid = std::max<uint32_t>(
          1, std::min<uint32_t>(ceil_div(cloud->n, 256), uint32_t(ctx->num_sms) * 8));
      k_deinterleave<<<grid, 256, 0, ctx->stream>>>(iv, cloud->n);
      CU_TRY(cudaGetLastError());
    }
    return SRCU_OK;
  }
  for (uint32_t c = 0; c < nc; ++c) {
    if (cloud->on_device) {
      cols[c] = src[c];
    } else {
      if (cloud->n) ST_TRY(host_to_device(ctx, ctx->in[c].p, src[c], cloud->n * 4, ctx->stream));
      cols[c] = ptr<const float>(ctx->in[c]);
    }
  }
  return SRCU_OK;
}

SortBuffers sort_buffers(srcu_ctx *ctx) {
  SortBuffers sb;
  sb.keys[0] = ptr<uint64_t>(ctx->keys[0]);
  sb.keys[1] = ptr<uint64_t>(ctx->keys[1]);
  sb.vals[0] = ptr<uint32_t>(ctx->vals[0]);
  sb.vals[1] = ptr<uint32_t>(ctx->vals[1]);
  sb.lookback = ptr<uint64_t>(ctx->lb_sort);
  return sb;
}

// Launches the persistent cooperative sort (histogram + every needed digit
// pass in one kernel).  The grid never exceeds the co-resident block count.
srcu_status reserve_batch(srcu_ctx *ctx, uint32_t clouds) {
  const uint64_t b = std::max<uint32_t>(clouds, 1);
  ST_TRY(ensure(ctx, ctx->b_offsets, (b + 1) * 4));
  ST_TRY(ensure(ctx, ctx->b_bounds, b * sizeof(Bounds)));
  ST_TRY(ensure(ctx, ctx->b_vplans, b * sizeof(VoxelPlan)));
  ST_TRY(ensure(ctx, ctx->b_cplans, b * sizeof(CellPlan)));
  ST_TRY(ensure(ctx, ctx->b_vparams, b * sizeof(VoxelParamsDev)));
  ST_TRY(ensure(ctx, ctx->b_nparams, b * sizeof(NormalParamsDev)));
  ST_TRY(ensure(ctx, ctx->b_voff, (b + 1) * 4));
  ctx->batch_cap = std::max<uint32_t>(ctx->batch_cap, uint32_t(b));
  return SRCU_OK;
}

Batch make_batch(srcu_ctx *ctx, uint32_t clouds) {
  Batch bt;
  bt.clouds = clouds;
  bt.offsets = ptr<const uint32_t>(ctx->b_offsets);
  bt.bounds = ptr<Bounds>(ctx->b_bounds);
  bt.vplans = ptr<VoxelPlan>(ctx->b_vplans);
  bt.cplans = ptr<CellPlan>(ctx->b_cplans);
  bt.vparams = ptr<const VoxelParamsDev>(ctx->b_vparams);
  bt.nparams = ptr<const NormalParamsDev>(ctx->b_nparams);
  bt.voxel_offsets = ptr<uint32_t>(ctx->b_voff);
  return bt;
}

VoxelParamsDev to_dev(const srcu_voxel_params *vp) {
  VoxelParamsDev d{};
  if (!vp) return d;
  d.leaf = vp->leaf_size;
  d.has_origin = vp->has_origin;
  for (int a = 0; a < 3; ++a) d.origin[a] = vp->origin[a];
  d.agg = vp->mode == SRCU_VOXEL_APPROXIMATE_FIRST ? AGG_FIRST
          : vp->attribute_policy == SRCU_ATTRIBUTE_FIRST ? AGG_CENTROID_FIRST
                                                         : AGG_FAST;
  return d;
}

NormalParamsDev to_dev(const srcu_normal_params *np) {
  NormalParamsDev d{};
  if (!np) return d;
  d.radius = np->radius;
  d.min_neighbors = np->min_neighbors;
  d.include_self = np->include_self;
  d.has_viewpoint = np->has_viewpoint;
  d.count_shell = np->count_shell;
  for (int a = 0; a < 3; ++a) d.vp[a] = np->viewpoint[a];
  return d;
}

uint32_t cloud_bits_for(uint32_t clouds) { return clouds > 1 ? bit_width_u64(clouds - 1) : 0; }

// Copies the offsets and per-cloud parameters of a batch to the device
// through a pinned staging slot (two slots alternate; a slot is reused only
// after its previous copy has completed).
srcu_status stage_batch(srcu_ctx *ctx, uint32_t clouds, const uint64_t *offsets,
                        const srcu_voxel_params *vp, const srcu_normal_params *np) {
  const size_t off_bytes = (size_t(clouds) + 1) * 4;
  const size_t vp_bytes = size_t(clouds) * sizeof(VoxelParamsDev);
  const size_t np_bytes = size_t(clouds) * sizeof(NormalParamsDev);
  const size_t need = off_bytes + vp_bytes + np_bytes;
  const int slot = ctx->h_stage_next;
  ctx->h_stage_next ^= 1;
  if (ctx->h_stage_ev[slot]) CU_TRY(cudaEventSynchronize(ctx->h_stage_ev[slot]));
  if (ctx->h_stage_bytes[slot] < need) {
    if (ctx->h_stage[slot]) CU_TRY(cudaFreeHost(ctx->h_stage[slot]));
    ctx->h_stage[slot] = nullptr;
    CU_TRY(cudaMallocHost(reinterpret_cast<void **>(&ctx->h_stage[slot]), need));
    ctx->h_stage_bytes[slot] = need;
  }
  if (!ctx->h_stage_ev[slot])
    CU_TRY(cudaEventCreateWithFlags(&ctx->h_stage_ev[slot], cudaEventDisableTiming));
  unsigned char *h = ctx->h_stage[slot];
  uint32_t *ho = reinterpret_cast<uint32_t *>(h);
  for (uint32_t b = 0; b <= clouds; ++b) ho[b] = uint32_t(offsets[b]);
  VoxelParamsDev *hv = reinterpret_cast<VoxelParamsDev *>(h + off_bytes);
  NormalParamsDev *hn = reinterpret_cast<NormalParamsDev *>(h + off_bytes + vp_bytes);
  for (uint32_t b = 0; b < clouds; ++b) {
    hv[b] = to_dev(vp ? &vp[b] : nullptr);
    hn[b] = to_dev(np ? &np[b] : nullptr);
  }
  CU_TRY(cudaMemcpyAsync(ctx->b_offsets.p, ho, off_bytes, cudaMemcpyHostToDevice, ctx->stream));
  CU_TRY(cudaMemcpyAsync(ctx->b_vparams.p, hv, vp_bytes, cudaMemcpyHostToDevice, ctx->stream));
  CU_TRY(cudaMemcpyAsync(ctx->b_nparams.p, hn, np_bytes, cudaMemcpyHostToDevice, ctx->stream));
  CU_TRY(cudaEventRecord(ctx->h_stage_ev[slot], ctx->stream));
  return SRCU_OK;
}

template <class Src>
cudaError_t launch_sort_kernel(cudaStream_t stream, int num_sms, int occ, const Src &src,
                               Control *ctl, uint32_t *hist, const SortBuffers &sb,
                               uint32_t epoch_off, int work_slot, SortState *st, uint64_t n_max) {
  const uint32_t tiles = std::max<uint32_t>(1, ceil_div(n_max, OS_TILE));
  const uint32_t grid = std::max<uint32_t>(1, std::min<uint32_t>(tiles, uint32_t(num_sms) * uint32_t(occ)));
  Src s = src;
  Control *c = ctl;
  uint32_t *h = hist;
  SortBuffers b = sb;
  uint32_t e = epoch_off;
  int w = work_slot;
  SortState *ss = st;
  void *args[] = {&s, &c, &h, &b, &e, &w, &ss};
  return cudaLaunchCooperativeKernel(reinterpret_cast<const void *>(&k_sort<Src>), dim3(grid),
                                     dim3(OS_THREADS), args, sizeof(OnesweepSmem), stream);
}

template <class Src>
srcu_status launch_sort(srcu_ctx *ctx, const Src &src, uint64_t n_max, uint32_t *hist,
                        uint32_t epoch_off, int work_slot, SortState *st, int occ, int sort_id) {
  Launch l(ctx, sort_id);
  CU_TRY(launch_sort_kernel(ctx->stream, ctx->num_sms, occ, src, ctx->ctl, hist, sort_buffers(ctx),
                            epoch_off, work_slot, st, n_max));
  return SRCU_OK;
}

// One launch shape of the sort: C indexes kSortItems / kSortMinBlocks.
template <class Src, int C>
cudaError_t launch_sort_config(cudaStream_t stream, uint32_t grid_cap, const Src &src,
                               Control *ctl, uint32_t *hist, const SortBuffers &sb,
                               uint32_t epoch_off, int work_slot, SortState *st, uint64_t n_max) {
  constexpr int THREADS = kSortThreads[C];
  constexpr int TILE = THREADS * kSortItems[C];
  constexpr int DBITS = kSortDigitBits[C];
  static_assert(lookback_fits(TILE, 1 << DBITS), "the look-back buffer's words per key");
  const uint32_t tiles = std::max<uint32_t>(1, ceil_div(n_max, TILE));
  const uint32_t grid = std::max<uint32_t>(1, std::min<uint32_t>(tiles, grid_cap));
  Src s = src;
  Control *c = ctl;
  uint32_t *h = hist;
  SortBuffers b = sb;
  uint32_t e = epoch_off;
  int w = work_slot;
  SortState *ss = st;
  void *args[] = {&s, &c, &h, &b, &e, &w, &ss};
  return cudaLaunchCooperativeKernel(
      reinterpret_cast<const void *>(&k_sort<Src, kSortItems[C], kSortMinBlocks[C], THREADS, DBITS>),
      dim3(grid), dim3(THREADS), args, sizeof(OnesweepSmemT<TILE, THREADS / 32, DBITS>), stream);
}

template <class Src, int C>
cudaError_t sort_config_setup(int *occ) {
  constexpr int THREADS = kSortThreads[C];
  constexpr int TILE = THREADS * kSortItems[C];
  constexpr int DBITS = kSortDigitBits[C];
  using Smem = OnesweepSmemT<TILE, THREADS / 32, DBITS>;
  const void *kern = reinterpret_cast<const void *>(
      &k_sort<Src, kSortItems[C], kSortMinBlocks[C], THREADS, DBITS>);
  cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                       int(sizeof(Smem)));
  if (e != cudaSuccess) return e;
  e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(occ, kern, THREADS, sizeof(Smem));
  *occ = std::max(1, *occ);
  return e;
}

template <class Src>
cudaError_t sort_setup(int (&occ)[SORT_CONFIGS]) {
  static_assert(SORT_CONFIGS == 8, "one setup per launch shape");
  cudaError_t e = sort_config_setup<Src, 0>(&occ[0]);
  if (e == cudaSuccess) e = sort_config_setup<Src, 1>(&occ[1]);
  if (e == cudaSuccess) e = sort_config_setup<Src, 2>(&occ[2]);
  if (e == cudaSuccess) e = sort_config_setup<Src, 3>(&occ[3]);
  if (e == cudaSuccess) e = sort_config_setup<Src, 4>(&occ[4]);
  if (e == cudaSuccess) e = sort_config_setup<Src, 5>(&occ[5]);
  if (e == cudaSuccess) e = sort_config_setup<Src, 6>(&occ[6]);
  if (e == cudaSuccess) e = sort_config_setup<Src, 7>(&occ[7]);
  return e;
}

int sort_config_for(const srcu_ctx *ctx, int kind, uint64_t n) {
  const uint32_t cnt = ctx->tune_count[kind];
  for (uint32_t k = 0; k < cnt; ++k)
    if (n <= ctx->tune_max_points[kind][k]) return ctx->tune_config[kind][k];
  return cnt ? ctx->tune_config[kind][cnt - 1] : 0;
}

void builtin_sort_tuning(srcu_ctx *ctx, int kind) {
  uint32_t cnt;
  const uint64_t *mp;
  const int32_t *cf;
  switch (kind) {
    case SRCU_SORT_VOXEL_KEYS:
      cnt = kVoxelSortTuneCount, mp = kVoxelSortTuneMaxPoints, cf = kVoxelSortTuneConfig;
      break;
    case SRCU_SORT_CELL_KEYS:
      cnt = kCellSortTuneCount, mp = kCellSortTuneMaxPoints, cf = kCellSortTuneConfig;
      break;
    case SRCU_SORT_BATCH_VOXEL_KEYS:
      cnt = kBatchVoxelSortTuneCount, mp = kBatchVoxelSortTuneMaxPoints, cf = kBatchVoxelSortTuneConfig;
      break;
    default:
      cnt = kBatchCellSortTuneCount, mp = kBatchCellSortTuneMaxPoints, cf = kBatchCellSortTuneConfig;
  }
  ctx->tune_count[kind] = cnt;
  for (uint32_t k = 0; k < cnt; ++k) {
    ctx->tune_max_points[kind][k] = mp[k];
    ctx->tune_config[kind][k] = cf[k];
  }
}

// The voxel-key and cell-key sorts, in the launch shape the context's tuning
// table of that sort kind gives for n_max keys.
template <class Src>
srcu_status launch_sort_tuned(srcu_ctx *ctx, int kind, const Src &src, uint64_t n_max,
                              uint32_t *hist, uint32_t epoch_off, int work_slot, SortState *st,
                              const int (&occ)[SORT_CONFIGS], int sort_id) {
  Launch l(ctx, sort_id);
  const int c = sort_config_for(ctx, kind, n_max);
  const uint32_t cap = uint32_t(ctx->num_sms) * uint32_t(occ[c]);
  const SortBuffers sb = sort_buffers(ctx);
  cudaError_t e;
  switch (c) {
    case 1:
      e = launch_sort_config<Src, 1>(ctx->stream, cap, src, ctx->ctl, hist, sb, epoch_off, work_slot, st, n_max);
      break;
    case 2:
      e = launch_sort_config<Src, 2>(ctx->stream, cap, src, ctx->ctl, hist, sb, epoch_off, work_slot, st, n_max);
      break;
    case 3:
      e = launch_sort_config<Src, 3>(ctx->stream, cap, src, ctx->ctl, hist, sb, epoch_off, work_slot, st, n_max);
      break;
    case 4:
      e = launch_sort_config<Src, 4>(ctx->stream, cap, src, ctx->ctl, hist, sb, epoch_off, work_slot, st, n_max);
      break;
    case 5:
      e = launch_sort_config<Src, 5>(ctx->stream, cap, src, ctx->ctl, hist, sb, epoch_off, work_slot, st, n_max);
      break;
    case 6:
      e = launch_sort_config<Src, 6>(ctx->stream, cap, src, ctx->ctl, hist, sb, epoch_off, work_slot, st, n_max);
      break;
    case 7:
      e = launch_sort_config<Src, 7>(ctx->stream, cap, src, ctx->ctl, hist, sb, epoch_off, work_slot, st, n_max);
      break;
    default:
      e = launch_sort_config<Src, 0>(ctx->stream, cap, src, ctx->ctl, hist, sb, epoch_off, work_slot, st, n_max);
  }
  CU_TRY(e);
  return SRCU_OK;
}

template <int NC>
void launch_segments_nc(srcu_ctx *ctx, const float **in, uint32_t grid, const Batch &bt) {
  Columns<NC> cols;
  for (int c = 0; c < NC; ++c) {
    cols.in[c] = in[c];
    cols.out[c] = ptr<float>(ctx->vout[c]);
  }
  k_voxel_segments<NC><<<grid, SEG_THREADS, segment_smem_bytes(NC), ctx->stream>>>(
      ctx->ctl, sort_buffers(ctx), &ctx->ctl->vsort, cols, ptr<uint64_t>(ctx->vkeys),
      ptr<uint32_t>(ctx->vcounts), ptr<uint64_t>(ctx->lb_seg), ptr<const float4>(ctx->in_aos),
      ptr<float4>(ctx->vaos), bt, ctx->agg_all);
}

// The plain-xyz path after the segment kernel: f32 centroids in input order,
// then the voxels (columns, counts, keys, AoS copy) in first-seen order.
srcu_status enqueue_first_seen(srcu_ctx *ctx, const float **in, uint64_t n) {
  ST_TRY(ensure(ctx, ctx->xyz_tmp, std::max<uint64_t>(n, 1) * 28));
  float *tx = ptr<float>(ctx->xyz_tmp);
  float *ty = tx + n;
  float *tz = ty + n;
  uint32_t *tc = reinterpret_cast<uint32_t *>(tz + n);
  uint64_t *tk = reinterpret_cast<uint64_t *>(tc + n);  // byte offset 16 n: 8-aligned
  uint32_t *first = reinterpret_cast<uint32_t *>(tk + n);
  const uint32_t grid = std::max<uint32_t>(1, std::min<uint32_t>(ceil_div(n, 256), ctx->num_sms * 8));
  {
    Launch l(ctx, SRCU_K_VOXEL_SEGMENTS);
    k_voxel_xyz_f32<<<grid, 256, 0, ctx->stream>>>(
        ctx->ctl, sort_buffers(ctx), &ctx->ctl->vsort, in[0], in[1], in[2],
        ptr<uint64_t>(ctx->vkeys), ptr<uint32_t>(ctx->vcounts), ptr<float>(ctx->vout[0]),
        ptr<float>(ctx->vout[1]), ptr<float>(ctx->vout[2]), first);
    CU_TRY(cudaGetLastError());
  }
  // The voxel sort is consumed: its histogram is reused, zeroed, by the order
  // sort, whose state is the cell sort's (the cell sort, if any, comes after).
  CU_TRY(cudaMemsetAsync(ctx->ctl->hist_v, 0, sizeof(ctx->ctl->hist_v), ctx->stream));
  FirstSeenSrc src;
  src.first = first;
  src.bits = n > 1 ? bit_width_u64(n - 1) : 0u;
  ST_TRY(launch_sort(ctx, src, n, ctx->ctl->hist_v, EP_ORDER, WK_ORDER, &ctx->ctl->csort,
                     ctx->occ_sort_order, SRCU_K_VOXEL_SORT));
  Launch l(ctx, SRCU_K_VOXEL_SEGMENTS);
  k_voxel_first_seen_gather<<<grid, 256, 0, ctx->stream>>>(
      ctx->ctl, sort_buffers(ctx), &ctx->ctl->csort, ptr<float>(ctx->vout[0]),
      ptr<float>(ctx->vout[1]), ptr<float>(ctx->vout[2]), ptr<uint32_t>(ctx->vcounts),
      ptr<uint64_t>(ctx->vkeys), tx, ty, tz, tc, tk);
  k_voxel_copy_back<<<grid, 256, 0, ctx->stream>>>(
      ctx->ctl, tx, ty, tz, tc, tk, ptr<float>(ctx->vout[0]), ptr<float>(ctx->vout[1]),
      ptr<float>(ctx->vout[2]), ptr<uint32_t>(ctx->vcounts), ptr<uint64_t>(ctx->vkeys),
      ptr<float4>(ctx->vaos));
  CU_TRY(cudaGetLastError());
  return SRCU_OK;
}

// Voxel stage: bounds -> plan -> sort -> fused segment/centroid reduction.
srcu_status enqueue_voxel(srcu_ctx *ctx, const float **in, uint32_t nc, uint64_t n,
                          const Batch &bt) {
  const uint32_t grid_b = std::max<uint32_t>(1, std::min<uint32_t>(ceil_div(n, BND_THREADS * 4),
                                                                    uint32_t(ctx->num_sms) * 16));
  {
    Launch l(ctx, SRCU_K_BOUNDS);
    k_bounds<<<grid_b, BND_THREADS, 0, ctx->stream>>>(in[0], in[1], in[2], ctx->ctl, nullptr,
                                                       nc > 3 ? in[3] : nullptr,
                                                       ptr<float4>(ctx->in_aos), bt);
  }
  {
    Launch l(ctx, SRCU_K_VOXEL_PLAN);
    k_voxel_plans<<<ceil_div(bt.clouds, 128), 128, 0, ctx->stream>>>(ctx->ctl, bt);
  }
  VoxelKeySrc src;
  src.x = in[0];
  src.y = in[1];
  src.z = in[2];
  src.bt = bt;
  // a batch's keys carry the cloud id above the per-cloud key: tuned apart
  ST_TRY(launch_sort_tuned(ctx, bt.clouds > 1 ? SRCU_SORT_BATCH_VOXEL_KEYS : SRCU_SORT_VOXEL_KEYS,
                           src, n, ctx->ctl->hist_v, EP_VSORT, WK_VSORT, &ctx->ctl->vsort,
                           ctx->occ_sort_v, SRCU_K_VOXEL_SORT));
  const uint32_t tiles = std::max<uint32_t>(1, ceil_div(n, SEG_TILE));
  const uint32_t grid = std::min<uint32_t>(tiles, uint32_t(ctx->num_sms) * uint32_t(ctx->occ_seg));
  Launch l(ctx, SRCU_K_VOXEL_SEGMENTS);
  switch (nc) {
    case 3: launch_segments_nc<3>(ctx, in, grid, bt); break;
    case 4: launch_segments_nc<4>(ctx, in, grid, bt); break;
    case 5: launch_segments_nc<5>(ctx, in, grid, bt); break;
    case 6: launch_segments_nc<6>(ctx, in, grid, bt); break;
    case 7: launch_segments_nc<7>(ctx, in, grid, bt); break;
    case 8: launch_segments_nc<8>(ctx, in, grid, bt); break;
    case 9: launch_segments_nc<9>(ctx, in, grid, bt); break;
    case 10: launch_segments_nc<10>(ctx, in, grid, bt); break;
    case 11: launch_segments_nc<11>(ctx, in, grid, bt); break;
    case 12: launch_segments_nc<12>(ctx, in, grid, bt); break;
    default: return fail(ctx, SRCU_ERR_INVALID_ARGUMENT, "unsupported column count %u", nc);
  }
  if (bt.clouds > 1)  // one cloud's range is [0, V), read from the control block
    k_voxel_offsets<<<ceil_div(bt.clouds + 1, 128), 128, 0, ctx->stream>>>(
        ctx->ctl, ptr<uint64_t>(ctx->vkeys), bt);
  CU_TRY(cudaGetLastError());
  if (ctx->xyz_order && bt.clouds == 1) ST_TRY(enqueue_first_seen(ctx, in, n));
  return SRCU_OK;
}

// Normals stage over (x, y, z) with the point count in *count_dev (device)
// or ctl->n_points when count_dev is null; n_max bounds the grid sizes.
// Radius grid: cell plans, cell sort, cell table, column hash, column ranges.
srcu_status enqueue_grid(srcu_ctx *ctx, const float *x, const float *y, const float *z,
                         const float4 *aos, const unsigned long long *count_dev, uint64_t n_max,
                         const Batch &bt, const uint64_t *voxel_keys) {
  {
    Launch l(ctx, SRCU_K_CELL_PLAN);
    k_cell_plans<<<ceil_div(bt.clouds, 128), 128, 0, ctx->stream>>>(ctx->ctl, bt);
    k_column_base<<<1, 256, 0, ctx->stream>>>(ctx->ctl, bt, uint64_t(1) << ctx->table_log2);
  }
  CellKeySrc src;
  src.x = x;
  src.y = y;
  src.z = z;
  src.count_dev = count_dev;
  src.voxel_keys = voxel_keys;
  src.bt = bt;
  ST_TRY(launch_sort_tuned(ctx, bt.clouds > 1 ? SRCU_SORT_BATCH_CELL_KEYS : SRCU_SORT_CELL_KEYS,
                           src, n_max, ctx->ctl->hist_c, EP_CSORT, WK_CSORT, &ctx->ctl->csort,
                           ctx->occ_sort_c, SRCU_K_CELL_SORT));
  const uint32_t tiles = std::max<uint32_t>(1, ceil_div(n_max, CELL_TILE));
  const uint32_t grid_c = std::min<uint32_t>(tiles, uint32_t(ctx->num_sms) * uint32_t(ctx->occ_cells));
  {
    Launch l(ctx, SRCU_K_CELLS);
    k_cells<<<grid_c, CELL_THREADS, 0, ctx->stream>>>(
        ctx->ctl, sort_buffers(ctx), &ctx->ctl->csort, count_dev, aos,
        ptr<float4>(ctx->pts), ptr<uint32_t>(ctx->pt_cell), ptr<uint64_t>(ctx->cell_key),
        ptr<uint32_t>(ctx->cell_start), ptr<uint64_t>(ctx->lb_cells));
  }
  const uint32_t grid_g = std::max<uint32_t>(1, std::min<uint32_t>(ceil_div(n_max, 256),
                                                                    uint32_t(ctx->num_sms) * 8));
  {
    Launch l(ctx, SRCU_K_HASH);
    k_column_insert<<<grid_g, 256, 0, ctx->stream>>>(ctx->ctl, ptr<uint64_t>(ctx->cell_key),
                                                     ptr<uint64_t>(ctx->table), ctx->table_log2, bt);
  }
  const uint32_t grid_r = std::max<uint32_t>(1, std::min<uint32_t>(ceil_div(n_max, 256),
                                                                    uint32_t(ctx->num_sms) * 8));
  {
    Launch l(ctx, SRCU_K_RANGES);
    k_ranges<<<grid_r, 256, 0, ctx->stream>>>(ctx->ctl, ptr<uint64_t>(ctx->cell_key),
                                              ptr<uint32_t>(ctx->cell_start),
                                              ptr<uint64_t>(ctx->table), ctx->table_log2,
                                              ptr<uint2>(ctx->ranges), bt);
  }
  CU_TRY(cudaGetLastError());
  return SRCU_OK;
}

srcu_status enqueue_normals(srcu_ctx *ctx, const float *x, const float *y, const float *z,
                            const float4 *aos, const unsigned long long *count_dev, uint64_t n_max,
                            const Batch &bt, const uint64_t *voxel_keys) {
  ST_TRY(enqueue_grid(ctx, x, y, z, aos, count_dev, n_max, bt, voxel_keys));
  const uint32_t grid_n = uint32_t(ctx->num_sms) * uint32_t(ctx->occ_normals);
  Launch l(ctx, SRCU_K_NORMALS);
  const int walk = ctx->neighbor_staging;
  auto kernel = walk == WALK_STAGED
                    ? (ctx->count_shell ? k_normals<true, false, WALK_STAGED>
                                        : k_normals<false, false, WALK_STAGED>)
                : walk == WALK_PACKED
                    ? (ctx->count_shell ? k_normals<true, false, WALK_PACKED>
                                        : k_normals<false, false, WALK_PACKED>)
                    : (ctx->count_shell ? k_normals<true> : k_normals<false>);
  const uint32_t grid = walk == WALK_STAGED ? uint32_t(ctx->num_sms) * uint32_t(ctx->occ_normals_staged)
                        : walk == WALK_PACKED ? uint32_t(ctx->num_sms) * uint32_t(ctx->occ_normals_packed)
                                            : grid_n;
  kernel<<<grid, NM_THREADS, 0, ctx->stream>>>(
      ctx->ctl, ptr<float4>(ctx->pts), ptr<uint32_t>(ctx->pt_cell), ptr<uint2>(ctx->ranges),
      ptr<uint64_t>(ctx->cell_key), bt, count_dev, ptr<float>(ctx->nout[0]),
      ptr<float>(ctx->nout[1]), ptr<float>(ctx->nout[2]), ptr<float>(ctx->nout[3]),
      ptr<uint32_t>(ctx->ncounts), nullptr, 0.0f);
  CU_TRY(cudaGetLastError());
  return SRCU_OK;
}

// Keeps look-back and hash tags unique.  Every chain's k_begin advances the
// device epoch by EPOCHS_PER_RUN and tags the words it publishes with
// epoch + offset (offset < EPOCHS_PER_RUN); a word counts as published only
// when its tag equals the reader's.  If the 32-bit epoch wrapped, a word left
// behind 2^26 chains earlier (on a tile index no chain has written since)
// would carry the current tag and be read as a published prefix.  So before
// the chain whose tags would pass 2^32 - 1, every epoch-tagged array is
// cleared and the epoch restarts at 0 (tag 0, the tag of a cleared word, is
// never used: the first chain after a restart runs at EPOCHS_PER_RUN).  The
// host mirrors the device epoch exactly -- k_begin is its only writer and
// each chain or graph replay runs one k_begin -- so the restart is issued on
// the host, in stream order, before that chain.
constexpr uint32_t kEpochLast = 0xffffffffu - 2 * EPOCHS_PER_RUN + 1;  // last epoch a chain may start from

srcu_status epoch_guard(srcu_ctx *ctx) {
  if (ctx->epoch_host > kEpochLast) {
    DevBuf *tagged[] = {&ctx->lb_sort, &ctx->lb_seg, &ctx->lb_cells, &ctx->table};
    for (DevBuf *b : tagged)
      if (b->p) CU_TRY(cudaMemsetAsync(b->p, 0, b->bytes, ctx->stream));
    CU_TRY(cudaMemsetAsync(&ctx->ctl->epoch, 0, sizeof(uint32_t), ctx->stream));
    ctx->epoch_host = 0;
    ++ctx->epoch_restarts;
  }
  ctx->epoch_host += EPOCHS_PER_RUN;
  return SRCU_OK;
}

// Starts a chain over one cloud (parameters written by k_begin itself) or
// a staged batch (single == 0).
srcu_status begin_chain(srcu_ctx *ctx, uint64_t n, const Batch &bt, int single,
                        const srcu_voxel_params *vp, const srcu_normal_params *np) {
  // a captured chain advances the epoch when its graph is launched
  if (!ctx->capturing) ST_TRY(epoch_guard(ctx));
  Launch l(ctx, SRCU_K_BEGIN);
  k_begin<<<1, 256, 0, ctx->stream>>>(ctx->ctl, n, bt, cloud_bits_for(bt.clouds), single,
                                      to_dev(vp), to_dev(np));
  ctx->last_clouds = bt.clouds;
  if (single) {
    ctx->agg_all = to_dev(vp).agg;
    ctx->count_shell = np && np->count_shell;
  }
  ctx->xyz_order = single && vp && vp->mode == SRCU_VOXEL_CENTROID_XYZ;
  return SRCU_OK;
}

srcu_status read_control(srcu_ctx *ctx) {
  CU_TRY(cudaMemcpyAsync(ctx->ctl_host, ctx->ctl, sizeof(Control), cudaMemcpyDeviceToHost,
                         ctx->stream));
  CU_TRY(cudaStreamSynchronize(ctx->stream));
  const uint32_t st = ctx->ctl_host->status;
  if (st == 0) return SRCU_OK;
  if (st & ST_TIMEOUT)
    return fail(ctx, SRCU_ERR_TIMEOUT, "a bounded device-side wait gave up (status 0x%x)", st);
  if (st & ST_TOO_MANY_POINTS)
    return fail(ctx, SRCU_ERR_INVALID_ARGUMENT, "too many points for one chain (status 0x%x)", st);
  if (st & ST_KEY_OVERFLOW)
    return fail(ctx, SRCU_ERR_KEY_OVERFLOW,
                "voxel keys of this cloud need more than 64 bits or a coordinate is infinite "
                "(status 0x%x)", st);
  if (st & ST_BAD_PARAMS)
    return fail(ctx, SRCU_ERR_INVALID_ARGUMENT, "search_radius must be a finite, non-negative number");
  if (st & ST_INTERNAL)
    return fail(ctx, SRCU_ERR_CUDA, "internal consistency check failed on the device (status 0x%x)", st);
  return fail(ctx, SRCU_ERR_CUDA, "device status 0x%x", st);
}

srcu_status copy_out(srcu_ctx *ctx, void *dst, const void *src, size_t bytes, int on_device,
                     cudaStream_t stream = nullptr) {
  if (!dst || bytes == 0) return SRCU_OK;
  if (!on_device) return device_to_host(ctx, dst, src, bytes, stream ? stream : ctx->stream);
  CU_TRY(cudaMemcpyAsync(dst, src, bytes, cudaMemcpyDeviceToDevice, stream ? stream : ctx->stream));
  return SRCU_OK;
}

// plain_cloud: the one cloud of a srcu_voxel_centroid / srcu_voxel_normals
// call, the only calls that take SRCU_VOXEL_CENTROID_XYZ.
srcu_status check_voxel_params(srcu_ctx *ctx, const srcu_voxel_params *vp,
                               const srcu_cloud *plain_cloud = nullptr) {
  if (!vp) return fail(ctx, SRCU_ERR_INVALID_ARGUMENT, "voxel params are NULL");
  if (vp->leaf_size <= 0.0f)  // voxel.rs:260-264 (a NaN leaf is not rejected there either)
    return fail(ctx, SRCU_ERR_INVALID_ARGUMENT, "leaf_size must be greater than zero");
  if (vp->mode == SRCU_VOXEL_CENTROID_XYZ) {
    if (!plain_cloud)
      return fail(ctx, SRCU_ERR_INVALID_ARGUMENT,
                  "the plain-xyz voxel mode runs through srcu_voxel_centroid and "
                  "srcu_voxel_normals only");
    if (plain_cloud->n_attrs != 0 || vp->attribute_policy != SRCU_ATTRIBUTE_AVERAGE)
      return fail(ctx, SRCU_ERR_INVALID_ARGUMENT,
                  "the plain-xyz voxel mode takes clouds of x, y, z only, Average policy");
    return SRCU_OK;
  }
  if ((vp->mode != SRCU_VOXEL_CENTROID && vp->mode != SRCU_VOXEL_APPROXIMATE_FIRST) ||
      (vp->attribute_policy != SRCU_ATTRIBUTE_AVERAGE && vp->attribute_policy != SRCU_ATTRIBUTE_FIRST))
    return fail(ctx, SRCU_ERR_INVALID_ARGUMENT, "unknown voxel aggregation mode %d / policy %d",
                vp->mode, vp->attribute_policy);
  return SRCU_OK;
}

srcu_status check_normal_params(srcu_ctx *ctx, const srcu_normal_params *np) {
  if (!np) return fail(ctx, SRCU_ERR_INVALID_ARGUMENT, "normal params are NULL");
  if (np->radius < 0.0f)  // normal.rs:109-111
    return fail(ctx, SRCU_ERR_INVALID_ARGUMENT, "search_radius must be non-negative");
  if (!(np->radius >= 0.0f) || np->radius == INFINITY)
    return fail(ctx, SRCU_ERR_INVALID_ARGUMENT, "search_radius must be finite");
  return SRCU_OK;
}

srcu_status fetch_voxels(srcu_ctx *ctx, uint32_t nc, const srcu_voxel_out *out, uint64_t v,
                         cudaStream_t stream = nullptr, bool keys = true) {
  if (!out) return SRCU_OK;
  float *dst[MAX_COLS] = {out->x, out->y, out->z};
  for (uint32_t a = 3; a < nc; ++a) dst[a] = out->attrs ? out->attrs[a - 3] : nullptr;
  for (uint32_t c = 0; c < nc; ++c)
    ST_TRY(copy_out(ctx, dst[c], ctx->vout[c].p, v * 4, out->on_device, stream));
  ST_TRY(copy_out(ctx, out->counts, ctx->vcounts.p, v * 4, out->on_device, stream));
  if (keys && out->keys)
    ST_TRY(copy_out(ctx, out->keys, ctx->vkeys3.p, v * 24, out->on_device, stream));
  return SRCU_OK;
}

srcu_status fetch_normals(srcu_ctx *ctx, const srcu_normal_out *out, uint64_t m,
                          srcu_normal_stats *stats) {
  if (out) {
    float *dst[4] = {out->nx, out->ny, out->nz, out->curvature};
    for (int c = 0; c < 4; ++c) ST_TRY(copy_out(ctx, dst[c], ctx->nout[c].p, m * 4, out->on_device));
    ST_TRY(copy_out(ctx, out->neighbor_counts, ctx->ncounts.p, m * 4, out->on_device));
  }
  if (stats) {
    stats->valid_count = ctx->ctl_host->ncount.valid;
    stats->invalid_count = ctx->ctl_host->ncount.invalid;
    stats->shell_points = ctx->ctl_host->ncount.shell;
    stats->fp64_eigensolves = ctx->ctl_host->ncount.fp64;
  }
  return SRCU_OK;
}

srcu_status unpack_keys(srcu_ctx *ctx, uint64_t n) {
  ST_TRY(ensure(ctx, ctx->vkeys3, std::max<uint64_t>(n, 1) * 24));
  const uint32_t grid = std::max<uint32_t>(1, std::min<uint32_t>(ceil_div(n, 256), ctx->num_sms * 8));
  Launch l(ctx, SRCU_K_UNPACK_KEYS);
  k_unpack_voxel_keys<<<grid, 256, 0, ctx->stream>>>(ctx->ctl, ptr<uint64_t>(ctx->vkeys),
                                                     ptr<int64_t>(ctx->vkeys3),
                                                     make_batch(ctx, ctx->last_clouds));
  CU_TRY(cudaGetLastError());
  return SRCU_OK;
}

}  // namespace

extern "C" {

int srcu_abi_version(void) { return SRCU_ABI_VERSION; }

srcu_status srcu_create(int device, uint64_t hbm_budget_bytes, srcu_ctx **out) {
  if (!out) return SRCU_ERR_INVALID_ARGUMENT;
  *out = nullptr;
  int count = 0;
  if (cudaGetDeviceCount(&count) != cudaSuccess || count <= device || device < 0) {
    cudaGetLastError();
    return SRCU_ERR_NO_DEVICE;
  }
  cudaDeviceProp prop;
  if (cudaGetDeviceProperties(&prop, device) != cudaSuccess || prop.major != 10) {
    cudaGetLastError();
    return SRCU_ERR_NO_DEVICE;
  }
  srcu_ctx *ctx = new srcu_ctx();
  ctx->device = device;
  ctx->budget = hbm_budget_bytes;
  ctx->num_sms = prop.multiProcessorCount;
  auto bail = [&](srcu_status st) {
    srcu_destroy(ctx);
    return st;
  };
  if (cudaSetDevice(device) != cudaSuccess) return bail(SRCU_ERR_CUDA);
  if (cudaStreamCreateWithFlags(&ctx->own_stream, cudaStreamNonBlocking) != cudaSuccess)
    return bail(SRCU_ERR_CUDA);
  ctx->stream = ctx->own_stream;
  if (cudaMalloc(&ctx->ctl, sizeof(Control)) != cudaSuccess) return bail(SRCU_ERR_OUT_OF_BUDGET);
  ctx->used += sizeof(Control);
  if (cudaMemset(ctx->ctl, 0, sizeof(Control)) != cudaSuccess) return bail(SRCU_ERR_CUDA);
  if (cudaMallocHost(&ctx->ctl_host, sizeof(Control)) != cudaSuccess) return bail(SRCU_ERR_CUDA);
  if (cudaStreamCreateWithFlags(&ctx->side_stream, cudaStreamNonBlocking) != cudaSuccess ||
      cudaEventCreateWithFlags(&ctx->ev_voxel, cudaEventDisableTiming) != cudaSuccess ||
      cudaMallocHost(reinterpret_cast<void **>(&ctx->head_host), offsetof(Control, n_cells)) !=
          cudaSuccess)
    return bail(SRCU_ERR_CUDA);
  // Kernels with more than 48 KB of dynamic shared memory opt in once; every
  // sort launch shape, with its co-resident block count.
  if (sort_setup<VoxelKeySrc>(ctx->occ_sort_v) != cudaSuccess ||
      sort_setup<CellKeySrc>(ctx->occ_sort_c) != cudaSuccess ||
      sort_config_setup<FirstSeenSrc, 0>(&ctx->occ_sort_order) != cudaSuccess)
    return bail(SRCU_ERR_CUDA);
  for (int kind = 0; kind < SRCU_SORT_KINDS; ++kind) builtin_sort_tuning(ctx, kind);
  cudaOccupancyMaxActiveBlocksPerMultiprocessor(&ctx->occ_normals, k_normals<true>, NM_THREADS, 0);
  cudaOccupancyMaxActiveBlocksPerMultiprocessor(&ctx->occ_normals_staged,
                                                k_normals<true, false, WALK_STAGED>, NM_THREADS, 0);
  cudaOccupancyMaxActiveBlocksPerMultiprocessor(&ctx->occ_normals_packed,
                                                k_normals<true, false, WALK_PACKED>, NM_THREADS, 0);
  ctx->neighbor_staging = kNeighborStaging;
  if (configure_segment_kernels() != cudaSuccess) return bail(SRCU_ERR_CUDA);
  cudaOccupancyMaxActiveBlocksPerMultiprocessor(&ctx->occ_seg, k_voxel_segments<4>, SEG_THREADS,
                                                segment_smem_bytes(4));
  cudaOccupancyMaxActiveBlocksPerMultiprocessor(&ctx->occ_cells, k_cells, CELL_THREADS, 0);
  ctx->occ_normals = std::max(1, ctx->occ_normals);
  ctx->occ_normals_staged = std::max(1, ctx->occ_normals_staged);
  ctx->occ_normals_packed = std::max(1, ctx->occ_normals_packed);
  ctx->occ_seg = std::max(1, ctx->occ_seg);
  ctx->occ_cells = std::max(1, ctx->occ_cells);
  if (cudaGetLastError() != cudaSuccess) return bail(SRCU_ERR_CUDA);
  *out = ctx;
  return SRCU_OK;
}

void srcu_destroy(srcu_ctx *ctx) {
  if (!ctx) return;
  cudaSetDevice(ctx->device);
  if (ctx->stream) cudaStreamSynchronize(ctx->stream);
  stream_voxel_free(ctx->parked_stream);
  ctx->parked_stream = nullptr;
  DevBuf *all[] = {&ctx->in_aos, &ctx->vaos, &ctx->keys[0], &ctx->keys[1], &ctx->vals[0], &ctx->vals[1], &ctx->lb_sort,
                   &ctx->lb_seg, &ctx->lb_cells, &ctx->vkeys, &ctx->vcounts, &ctx->vkeys3,
                   &ctx->pts, &ctx->pt_cell, &ctx->cell_key, &ctx->cell_start, &ctx->table, &ctx->ranges,
                   &ctx->ncounts, &ctx->parent, &ctx->cov6, &ctx->stage_block,
                   &ctx->rs_hyp, &ctx->rs_planes, &ctx->rs_valid, &ctx->rs_counts,
                   &ctx->rs_partials, &ctx->rs_mask, &ctx->xyz_tmp};
  for (DevBuf *b : all) release(ctx, *b);
  for (auto &b : ctx->in) release(ctx, b);
  for (auto &b : ctx->vout) release(ctx, b);
  for (auto &b : ctx->nout) release(ctx, b);
  DevBuf *batch[] = {&ctx->b_offsets, &ctx->b_bounds, &ctx->b_vplans, &ctx->b_cplans,
                     &ctx->b_vparams, &ctx->b_nparams, &ctx->b_voff};
  for (DevBuf *b : batch) release(ctx, *b);
  for (int slot = 0; slot < 2; ++slot) {
    if (ctx->h_stage_ev[slot]) cudaEventDestroy(ctx->h_stage_ev[slot]);
    if (ctx->h_stage[slot]) cudaFreeHost(ctx->h_stage[slot]);
  }
  for (cudaEvent_t e : ctx->ev_pool) cudaEventDestroy(e);
  for (int k = 0; k < 3; ++k) {
    if (ctx->ring_ev[k]) cudaEventSynchronize(ctx->ring_ev[k]), cudaEventDestroy(ctx->ring_ev[k]);
    if (ctx->ring[k]) cudaFreeHost(ctx->ring[k]);
  }
  if (ctx->ctl) cudaFree(ctx->ctl);
  if (ctx->ctl_host) cudaFreeHost(ctx->ctl_host);
  if (ctx->head_host) cudaFreeHost(ctx->head_host);
  if (ctx->ev_voxel) cudaEventDestroy(ctx->ev_voxel);
  if (ctx->side_stream) cudaStreamDestroy(ctx->side_stream);
  if (ctx->own_stream) cudaStreamDestroy(ctx->own_stream);
  delete ctx;
}

const char *srcu_last_error(const srcu_ctx *ctx) { return ctx ? ctx->err.c_str() : "no context"; }

srcu_status srcu_last_length_mismatch(const srcu_ctx *ctx, uint64_t *expected, uint64_t *found) {
  if (!ctx || !expected || !found) return SRCU_ERR_INVALID_ARGUMENT;
  *expected = ctx->mismatch_expected;
  *found = ctx->mismatch_found;
  return SRCU_OK;
}

srcu_status srcu_set_stream(srcu_ctx *ctx, void *cuda_stream) {
  if (!ctx) return SRCU_ERR_INVALID_ARGUMENT;
  ctx->stream = cuda_stream ? static_cast<cudaStream_t>(cuda_stream) : ctx->own_stream;
  return SRCU_OK;
}

int srcu_sort_configs(srcu_sort_config *out, int max_entries) {
  for (int c = 0; c < SORT_CONFIGS && c < max_entries && out; ++c) {
    out[c].items_per_thread = uint32_t(kSortItems[c]);
    out[c].blocks_per_sm = uint32_t(kSortMinBlocks[c]);
    out[c].digit_bits = uint32_t(kSortDigitBits[c]);
    out[c].threads_per_block = uint32_t(kSortThreads[c]);
  }
  return SORT_CONFIGS;
}

srcu_status srcu_set_sort_tuning(srcu_ctx *ctx, int32_t kind, const uint64_t *max_points,
                                 const int32_t *config, uint32_t count) {
  if (!ctx) return SRCU_ERR_INVALID_ARGUMENT;
  if (kind < 0 || kind >= SRCU_SORT_KINDS)
    return fail(ctx, SRCU_ERR_INVALID_ARGUMENT,
                "sort kind %d is not voxel keys (0), cell keys (1), batch voxel keys (2) or "
                "batch cell keys (3)", kind);
  if (count == 0) {
    builtin_sort_tuning(ctx, kind);
    return SRCU_OK;
  }
  if (count > SRCU_SORT_TUNING_MAX || !max_points || !config)
    return fail(ctx, SRCU_ERR_INVALID_ARGUMENT, "a sort tuning table has 1 to %d entries",
                SRCU_SORT_TUNING_MAX);
  for (uint32_t k = 0; k < count; ++k) {
    if (config[k] < 0 || config[k] >= SORT_CONFIGS)
      return fail(ctx, SRCU_ERR_INVALID_ARGUMENT, "sort launch shape %d is not 0-%d", config[k],
                  SORT_CONFIGS - 1);
    if (k > 0 && max_points[k] <= max_points[k - 1])
      return fail(ctx, SRCU_ERR_INVALID_ARGUMENT, "sort tuning sizes must ascend");
  }
  ctx->tune_count[kind] = count;
  for (uint32_t k = 0; k < count; ++k) {
    ctx->tune_max_points[kind][k] = max_points[k];
    ctx->tune_config[kind][k] = config[k];
  }
  return SRCU_OK;
}

srcu_status srcu_get_sort_tuning(srcu_ctx *ctx, int32_t kind, uint64_t *max_points,
                                 int32_t *config, uint32_t *count) {
  if (!ctx || !count || kind < 0 || kind >= SRCU_SORT_KINDS) return SRCU_ERR_INVALID_ARGUMENT;
  const uint32_t cap = *count;
  *count = ctx->tune_count[kind];
  for (uint32_t k = 0; k < ctx->tune_count[kind] && k < cap; ++k) {
    if (max_points) max_points[k] = ctx->tune_max_points[kind][k];
    if (config) config[k] = ctx->tune_config[kind][k];
  }
  return SRCU_OK;
}

srcu_status srcu_set_neighbor_staging(srcu_ctx *ctx, int32_t mode) {
  if (!ctx) return SRCU_ERR_INVALID_ARGUMENT;
  if (mode < -1 || mode > WALK_PACKED)
    return fail(ctx, SRCU_ERR_INVALID_ARGUMENT, "the neighbour walk is -1 (built-in), 0, 1 or 2");
  ctx->neighbor_staging = mode < 0 ? kNeighborStaging : mode;
  return SRCU_OK;
}

int32_t srcu_get_neighbor_staging(srcu_ctx *ctx) {
  return ctx ? ctx->neighbor_staging : -1;
}

srcu_status srcu_selftest_bounded_wait(srcu_ctx *ctx, uint32_t max_polls) {
  if (!ctx) return SRCU_ERR_INVALID_ARGUMENT;
  if (max_polls == 0 || max_polls > SPIN_LIMIT)
    return fail(ctx, SRCU_ERR_INVALID_ARGUMENT, "max_polls must be in [1, %u]", SPIN_LIMIT);
  CU_TRY(cudaSetDevice(ctx->device));
  // the flag is a word of the control block that this call zeroes and nothing sets
  uint32_t *flag = &ctx->ctl->work[63];
  CU_TRY(cudaMemsetAsync(flag, 0, sizeof(uint32_t), ctx->stream));
  CU_TRY(cudaMemsetAsync(&ctx->ctl->status, 0, sizeof(uint32_t), ctx->stream));
  k_selftest_wait<<<1, 32, 0, ctx->stream>>>(ctx->ctl, flag, max_polls);
  CU_TRY(cudaGetLastError());
  return read_control(ctx);
}

srcu_status srcu_synchronize(srcu_ctx *ctx) {
  if (!ctx) return SRCU_ERR_INVALID_ARGUMENT;
  CU_TRY(cudaStreamSynchronize(ctx->stream));
  return SRCU_OK;
}

uint64_t srcu_device_bytes(const srcu_ctx *ctx) { return ctx ? ctx->used : 0; }

srcu_status srcu_voxel_centroid(srcu_ctx *ctx, const srcu_cloud *cloud,
                                const srcu_voxel_params *params, const srcu_voxel_out *out,
                                uint64_t *out_voxels) {
  if (!ctx) return SRCU_ERR_INVALID_ARGUMENT;
  if (out_voxels) *out_voxels = 0;
  ST_TRY(check_cloud(ctx, cloud));
  ST_TRY(check_voxel_params(ctx, params, cloud));
  CU_TRY(cudaSetDevice(ctx->device));
  const uint64_t n = cloud->n;
  if (n == 0) return SRCU_OK;  // voxel.rs:257-259: empty input is returned unchanged
  const uint32_t nc = 3 + cloud->n_attrs;
  ST_TRY(reserve(ctx, n, nc, needs_staging(cloud), true, false));
  ST_TRY(reserve_batch(ctx, 1));
  if (out && out->keys) ST_TRY(ensure(ctx, ctx->vkeys3, n * 24));
  const float *cols[MAX_COLS];
  ST_TRY(stage_input(ctx, cloud, cols));
  const Batch bt = make_batch(ctx, 1);
  ST_TRY(begin_chain(ctx, n, bt, 1, params, nullptr));
  ST_TRY(enqueue_voxel(ctx, cols, nc, n, bt));
  if (out && out->keys) ST_TRY(unpack_keys(ctx, n));
  ST_TRY(read_control(ctx));
  const uint64_t v = ctx->ctl_host->n_voxels;
  ST_TRY(fetch_voxels(ctx, nc, out, v));
  CU_TRY(cudaStreamSynchronize(ctx->stream));
  if (out_voxels) *out_voxels = v;
  return SRCU_OK;
}

srcu_status srcu_radius_normals(srcu_ctx *ctx, const srcu_cloud *cloud,
                                const srcu_normal_params *params, const srcu_normal_out *out,
                                srcu_normal_stats *stats) {
  if (!ctx) return SRCU_ERR_INVALID_ARGUMENT;
  if (stats) memset(stats, 0, sizeof(*stats));
  ST_TRY(check_cloud(ctx, cloud));
  ST_TRY(check_normal_params(ctx, params));
  CU_TRY(cudaSetDevice(ctx->device));
  const uint64_t n = cloud->n;
  if (n == 0) return SRCU_OK;  // normal.rs:106-108
  ST_TRY(reserve(ctx, n, 3, needs_staging(cloud), false, true));
  ST_TRY(reserve_batch(ctx, 1));
  srcu_cloud xyz = *cloud;
  xyz.n_attrs = 0;
  const float *cols[MAX_COLS];
  ST_TRY(stage_input(ctx, &xyz, cols));
  const Batch bt = make_batch(ctx, 1);
  ST_TRY(begin_chain(ctx, n, bt, 1, nullptr, params));
  const uint32_t grid_b = std::max<uint32_t>(1, std::min<uint32_t>(ceil_div(n, BND_THREADS * 4),
                                                                    uint32_t(ctx->num_sms) * 8));
  {
    Launch l(ctx, SRCU_K_BOUNDS);
    k_bounds<<<grid_b, BND_THREADS, 0, ctx->stream>>>(cols[0], cols[1], cols[2], ctx->ctl, nullptr,
                                                       nullptr, ptr<float4>(ctx->in_aos), bt);
  }
  ST_TRY(enqueue_normals(ctx, cols[0], cols[1], cols[2], ptr<const float4>(ctx->in_aos), nullptr, n,
                         bt, nullptr));
  ST_TRY(read_control(ctx));
  ST_TRY(fetch_normals(ctx, out, n, stats));
  CU_TRY(cudaStreamSynchronize(ctx->stream));
  return SRCU_OK;
}

srcu_status srcu_euclidean_cluster_roots(srcu_ctx *ctx, const srcu_cloud *cloud,
                                         float cluster_tolerance, uint32_t *roots) {
  if (!ctx) return SRCU_ERR_INVALID_ARGUMENT;
  ST_TRY(check_cloud(ctx, cloud));
  const uint64_t n = cloud->n;
  if (n == 0) return SRCU_OK;  // uniform_grid.rs:100-102, before the tolerance check
  // uniform_grid.rs:103-105 (an infinite tolerance has no grid here)
  if (!(cluster_tolerance > 0.0f) || cluster_tolerance == INFINITY)
    return fail(ctx, SRCU_ERR_INVALID_ARGUMENT, "cluster_tolerance must be positive and finite");
  CU_TRY(cudaSetDevice(ctx->device));
  if (!roots) return fail(ctx, SRCU_ERR_MISSING_FIELD, "roots is NULL");
  ST_TRY(reserve(ctx, n, 3, needs_staging(cloud), false, true));
  ST_TRY(reserve_batch(ctx, 1));
  ST_TRY(ensure(ctx, ctx->parent, n * 4));
  srcu_cloud xyz = *cloud;
  xyz.n_attrs = 0;
  const float *cols[MAX_COLS];
  ST_TRY(stage_input(ctx, &xyz, cols));
  const Batch bt = make_batch(ctx, 1);
  srcu_normal_params np{};
  np.radius = cluster_tolerance;  // the grid of a radius search with r = tolerance
  np.min_neighbors = 1;
  ST_TRY(begin_chain(ctx, n, bt, 1, nullptr, &np));
  const uint32_t grid_b = std::max<uint32_t>(1, std::min<uint32_t>(ceil_div(n, BND_THREADS * 4),
                                                                    uint32_t(ctx->num_sms) * 8));
  {
    Launch l(ctx, SRCU_K_BOUNDS);
    k_bounds<<<grid_b, BND_THREADS, 0, ctx->stream>>>(cols[0], cols[1], cols[2], ctx->ctl, nullptr,
                                                       nullptr, ptr<float4>(ctx->in_aos), bt);
  }
  ST_TRY(enqueue_grid(ctx, cols[0], cols[1], cols[2], ptr<const float4>(ctx->in_aos), nullptr, n,
                      bt, nullptr));
  const float r2 = cluster_tolerance * cluster_tolerance;  // radius_sq, uniform_grid.rs:109
  const uint32_t grid = std::max<uint32_t>(1, std::min<uint32_t>(ceil_div(n, CL_THREADS),
                                                                  uint32_t(ctx->num_sms) * 8));
  uint32_t *dst = cloud->on_device ? roots : ptr<uint32_t>(ctx->nout[0]);
  {
    Launch l(ctx, SRCU_K_CLUSTER);
    k_cluster_init<<<grid, CL_THREADS, 0, ctx->stream>>>(ctx->ctl, ptr<uint32_t>(ctx->parent),
                                                         nullptr);
    k_cluster_union<<<grid, CL_THREADS, 0, ctx->stream>>>(
        ctx->ctl, ptr<const float4>(ctx->pts), ptr<const uint32_t>(ctx->pt_cell),
        ptr<const uint2>(ctx->ranges), nullptr, r2, ptr<uint32_t>(ctx->parent));
    k_cluster_roots<<<grid, CL_THREADS, 0, ctx->stream>>>(ctx->ctl, ptr<uint32_t>(ctx->parent), dst,
                                                          nullptr);
  }
  CU_TRY(cudaGetLastError());
  ST_TRY(read_control(ctx));
  if (!cloud->on_device) ST_TRY(copy_out(ctx, roots, dst, n * 4, 0));
  CU_TRY(cudaStreamSynchronize(ctx->stream));
  return SRCU_OK;
}

srcu_status srcu_plane_covariances(srcu_ctx *ctx, const srcu_cloud *cloud, float radius,
                                   float epsilon, float *cov, srcu_normal_stats *stats) {
  if (!ctx) return SRCU_ERR_INVALID_ARGUMENT;
  if (stats) memset(stats, 0, sizeof(*stats));
  ST_TRY(check_cloud(ctx, cloud));
  const uint64_t n = cloud->n;
  if (n == 0) return SRCU_OK;  // covariances_grid.rs:228-230, before the radius check
  // covariances_grid.rs:231-233 (an infinite radius has no grid here)
  if (!(radius > 0.0f) || radius == INFINITY)
    return fail(ctx, SRCU_ERR_INVALID_ARGUMENT, "grid radius must be positive and finite");
  CU_TRY(cudaSetDevice(ctx->device));
  if (!cov) return fail(ctx, SRCU_ERR_MISSING_FIELD, "cov is NULL");
  ST_TRY(reserve(ctx, n, 3, needs_staging(cloud), false, true));
  ST_TRY(reserve_batch(ctx, 1));
  float *dst = cov;
  if (!cloud->on_device) {
    ST_TRY(ensure(ctx, ctx->cov6, n * 24));
    dst = ptr<float>(ctx->cov6);
  }
  srcu_cloud xyz = *cloud;
  xyz.n_attrs = 0;
  const float *cols[MAX_COLS];
  ST_TRY(stage_input(ctx, &xyz, cols));
  const Batch bt = make_batch(ctx, 1);
  // The shader's neighbourhood includes the query (covariances_grid.rs:100-121)
  // and needs 3 points (:127-131): the include_self rule of the normals.
  srcu_normal_params np{};
  np.radius = radius;
  np.min_neighbors = 3;
  np.include_self = 1;
  ST_TRY(begin_chain(ctx, n, bt, 1, nullptr, &np));
  const uint32_t grid_b = std::max<uint32_t>(1, std::min<uint32_t>(ceil_div(n, BND_THREADS * 4),
                                                                    uint32_t(ctx->num_sms) * 8));
  {
    Launch l(ctx, SRCU_K_BOUNDS);
    k_bounds<<<grid_b, BND_THREADS, 0, ctx->stream>>>(cols[0], cols[1], cols[2], ctx->ctl, nullptr,
                                                       nullptr, ptr<float4>(ctx->in_aos), bt);
  }
  ST_TRY(enqueue_grid(ctx, cols[0], cols[1], cols[2], ptr<const float4>(ctx->in_aos), nullptr, n,
                      bt, nullptr));
  {
    const bool flat = ctx->neighbor_staging == WALK_PACKED;
    const uint32_t grid_n =
        uint32_t(ctx->num_sms) * uint32_t(flat ? ctx->occ_normals_packed : ctx->occ_normals);
    Launch l(ctx, SRCU_K_NORMALS);
    (flat ? k_normals<false, true, WALK_PACKED> : k_normals<false, true>)<<<grid_n, NM_THREADS, 0, ctx->stream>>>(
        ctx->ctl, ptr<float4>(ctx->pts), ptr<uint32_t>(ctx->pt_cell), ptr<uint2>(ctx->ranges),
        ptr<uint64_t>(ctx->cell_key), bt, nullptr, nullptr, nullptr, nullptr, nullptr, nullptr,
        dst, epsilon);
  }
  CU_TRY(cudaGetLastError());
  ST_TRY(read_control(ctx));
  if (!cloud->on_device) ST_TRY(copy_out(ctx, cov, dst, n * 24, 0));
  ST_TRY(fetch_normals(ctx, nullptr, n, stats));
  CU_TRY(cudaStreamSynchronize(ctx->stream));
  return SRCU_OK;
}

srcu_status srcu_voxel_normals(srcu_ctx *ctx, const srcu_cloud *cloud,
                               const srcu_voxel_params *vparams, const srcu_normal_params *nparams,
                               const srcu_voxel_out *vout, const srcu_normal_out *nout,
                               uint64_t *out_voxels, srcu_normal_stats *stats) {
  if (!ctx) return SRCU_ERR_INVALID_ARGUMENT;
  if (out_voxels) *out_voxels = 0;
  if (stats) memset(stats, 0, sizeof(*stats));
  ST_TRY(check_cloud(ctx, cloud));
  ST_TRY(check_voxel_params(ctx, vparams, cloud));
  ST_TRY(check_normal_params(ctx, nparams));
  CU_TRY(cudaSetDevice(ctx->device));
  const uint64_t n = cloud->n;
  if (n == 0) return SRCU_OK;
  const uint32_t nc = 3 + cloud->n_attrs;
  ST_TRY(reserve(ctx, n, nc, needs_staging(cloud), true, true));
  ST_TRY(reserve_batch(ctx, 1));
  if (vout && vout->keys) ST_TRY(ensure(ctx, ctx->vkeys3, n * 24));
  const float *cols[MAX_COLS];
  ST_TRY(stage_input(ctx, cloud, cols));
  const Batch bt = make_batch(ctx, 1);
  ST_TRY(begin_chain(ctx, n, bt, 1, vparams, nparams));
  ST_TRY(enqueue_voxel(ctx, cols, nc, n, bt));
  // The centroids are final once the voxel stage is done: their read-back
  // runs on the side stream while the normal kernels run.  The host learns V
  // from a small copy of the control-block head taken at that point.
  CU_TRY(cudaMemcpyAsync(ctx->head_host, ctx->ctl, offsetof(Control, n_cells),
                         cudaMemcpyDeviceToHost, ctx->stream));
  CU_TRY(cudaEventRecord(ctx->ev_voxel, ctx->stream));
  // Normals on the centroids (mvp.rs:220-222); the input bounds contain them.
  ST_TRY(enqueue_normals(ctx, ptr<float>(ctx->vout[0]), ptr<float>(ctx->vout[1]),
                         ptr<float>(ctx->vout[2]), ptr<const float4>(ctx->vaos),
                         &ctx->ctl->n_voxels, n, bt, ptr<uint64_t>(ctx->vkeys)));
  if (vout && vout->keys) ST_TRY(unpack_keys(ctx, n));
  bool early = false;
  if (vout) {
    CU_TRY(cudaEventSynchronize(ctx->ev_voxel));
    const Control *head = reinterpret_cast<const Control *>(ctx->head_host);
    if (head->status == 0) {  // otherwise read_control below reports the failure
      CU_TRY(cudaStreamWaitEvent(ctx->side_stream, ctx->ev_voxel, 0));
      ST_TRY(fetch_voxels(ctx, nc, vout, head->n_voxels, ctx->side_stream, false));
      early = true;
    }
  }
  const srcu_status st = read_control(ctx);
  if (early && st != SRCU_OK) cudaStreamSynchronize(ctx->side_stream);  // no copy outlives the call
  if (st != SRCU_OK) return st;
  const uint64_t v = ctx->ctl_host->n_voxels;
  if (!early) ST_TRY(fetch_voxels(ctx, nc, vout, v));
  else if (vout->keys) ST_TRY(copy_out(ctx, vout->keys, ctx->vkeys3.p, v * 24, vout->on_device));
  ST_TRY(fetch_normals(ctx, nout, v, stats));
  CU_TRY(cudaStreamSynchronize(ctx->stream));
  CU_TRY(cudaStreamSynchronize(ctx->side_stream));
  if (out_voxels) *out_voxels = v;
  return SRCU_OK;
}

srcu_status srcu_voxel_normals_enqueue(srcu_ctx *ctx, const srcu_cloud *cloud,
                                       const srcu_voxel_params *vparams,
                                       const srcu_normal_params *nparams) {
  if (!ctx) return SRCU_ERR_INVALID_ARGUMENT;
  ST_TRY(check_cloud(ctx, cloud));
  ST_TRY(check_voxel_params(ctx, vparams));
  ST_TRY(check_normal_params(ctx, nparams));
  if (!cloud->on_device)
    return fail(ctx, SRCU_ERR_INVALID_ARGUMENT, "enqueue needs a device-resident cloud");
  const uint64_t n = cloud->n;
  const uint32_t nc = 3 + cloud->n_attrs;
  ST_TRY(reserve(ctx, n, nc, needs_staging(cloud), true, true));
  ST_TRY(reserve_batch(ctx, 1));
  const float *cols[MAX_COLS];
  ST_TRY(stage_input(ctx, cloud, cols));
  const Batch bt = make_batch(ctx, 1);
  ST_TRY(begin_chain(ctx, n, bt, 1, vparams, nparams));
  if (n > 0) {
    ST_TRY(enqueue_voxel(ctx, cols, nc, n, bt));
    ST_TRY(enqueue_normals(ctx, ptr<float>(ctx->vout[0]), ptr<float>(ctx->vout[1]),
                           ptr<float>(ctx->vout[2]), ptr<const float4>(ctx->vaos),
                           &ctx->ctl->n_voxels, n, bt, ptr<uint64_t>(ctx->vkeys)));
  }
  ctx->last_attrs = cloud->n_attrs;
  CU_TRY(cudaGetLastError());
  return SRCU_OK;
}

srcu_status srcu_voxel_centroid_enqueue(srcu_ctx *ctx, const srcu_cloud *cloud,
                                        const srcu_voxel_params *vparams) {
  if (!ctx) return SRCU_ERR_INVALID_ARGUMENT;
  ST_TRY(check_cloud(ctx, cloud));
  ST_TRY(check_voxel_params(ctx, vparams));
  if (!cloud->on_device)
    return fail(ctx, SRCU_ERR_INVALID_ARGUMENT, "enqueue needs a device-resident cloud");
  const uint64_t n = cloud->n;
  const uint32_t nc = 3 + cloud->n_attrs;
  ST_TRY(reserve(ctx, n, nc, needs_staging(cloud), true, false));
  ST_TRY(reserve_batch(ctx, 1));
  const float *cols[MAX_COLS];
  ST_TRY(stage_input(ctx, cloud, cols));
  const Batch bt = make_batch(ctx, 1);
  ST_TRY(begin_chain(ctx, n, bt, 1, vparams, nullptr));
  if (n > 0) ST_TRY(enqueue_voxel(ctx, cols, nc, n, bt));
  ctx->last_attrs = cloud->n_attrs;
  CU_TRY(cudaGetLastError());
  return SRCU_OK;
}

static srcu_status batch_enqueue(srcu_ctx *ctx, const srcu_cloud *points, const uint64_t *offsets,
                                 uint32_t count, const srcu_voxel_params *vparams,
                                 const srcu_normal_params *nparams, bool stage) {
  if (!ctx) return SRCU_ERR_INVALID_ARGUMENT;
  ST_TRY(check_cloud(ctx, points));
  if (!points->on_device)
    return fail(ctx, SRCU_ERR_INVALID_ARGUMENT, "batch enqueue needs device-resident points");
  if (count == 0 || !offsets || !vparams || !nparams)
    return fail(ctx, SRCU_ERR_INVALID_ARGUMENT, "a batch needs count >= 1, offsets and parameters");
  if (offsets[0] != 0 || offsets[count] != points->n) {
    fail(ctx, SRCU_ERR_LENGTH_MISMATCH, "offsets must run from 0 to the point count %llu",
         (unsigned long long)points->n);
    ctx->mismatch_expected = offsets[0] != 0 ? 0 : points->n;
    ctx->mismatch_found = offsets[0] != 0 ? offsets[0] : offsets[count];
    return SRCU_ERR_LENGTH_MISMATCH;
  }
  for (uint32_t b = 0; b < count; ++b) {
    if (offsets[b + 1] < offsets[b])
      return fail(ctx, SRCU_ERR_INVALID_ARGUMENT, "offsets must be non-decreasing (cloud %u)", b);
    ST_TRY(check_voxel_params(ctx, &vparams[b]));
    ST_TRY(check_normal_params(ctx, &nparams[b]));
  }
  const uint64_t n = points->n;
  const uint32_t nc = 3 + points->n_attrs;
  ST_TRY(reserve(ctx, n, nc, needs_staging(points), true, true));
  ST_TRY(reserve_batch(ctx, count));
  const float *cols[MAX_COLS];
  ST_TRY(stage_input(ctx, points, cols));
  if (stage) ST_TRY(stage_batch(ctx, count, offsets, vparams, nparams));
  const Batch bt = make_batch(ctx, count);
  ST_TRY(begin_chain(ctx, n, bt, 0, nullptr, nullptr));
  ctx->agg_all = to_dev(&vparams[0]).agg;
  for (uint32_t b = 1; b < count; ++b)
    if (to_dev(&vparams[b]).agg != ctx->agg_all) ctx->agg_all = -1;
  ctx->count_shell = false;
  for (uint32_t b = 0; b < count; ++b) ctx->count_shell |= nparams[b].count_shell != 0;
  if (n > 0) {
    ST_TRY(enqueue_voxel(ctx, cols, nc, n, bt));
    ST_TRY(enqueue_normals(ctx, ptr<float>(ctx->vout[0]), ptr<float>(ctx->vout[1]),
                           ptr<float>(ctx->vout[2]), ptr<const float4>(ctx->vaos),
                           &ctx->ctl->n_voxels, n, bt, ptr<uint64_t>(ctx->vkeys)));
  }
  ctx->last_attrs = points->n_attrs;
  CU_TRY(cudaGetLastError());
  return SRCU_OK;
}

srcu_status srcu_batch_voxel_normals_enqueue(srcu_ctx *ctx, const srcu_cloud *points,
                                             const uint64_t *offsets, uint32_t count,
                                             const srcu_voxel_params *vparams,
                                             const srcu_normal_params *nparams) {
  return batch_enqueue(ctx, points, offsets, count, vparams, nparams, true);
}

struct srcu_graph {
  cudaGraph_t graph = nullptr;
  cudaGraphExec_t exec = nullptr;
  uint32_t clouds = 1;
  uint32_t attrs = 0;
};

srcu_status srcu_chain_graph_create(srcu_ctx *ctx, const srcu_cloud *points,
                                    const uint64_t *offsets, uint32_t count,
                                    const srcu_voxel_params *vparams,
                                    const srcu_normal_params *nparams, srcu_graph **out) {
  if (!ctx || !out) return SRCU_ERR_INVALID_ARGUMENT;
  *out = nullptr;
  if (ctx->stream == ctx->own_stream || ctx->stream == nullptr) {
    // capture needs a stream; the context's own stream is fine
  }
  const uint64_t single_off[2] = {0, points ? points->n : 0};
  const uint64_t *off = offsets ? offsets : single_off;
  const uint32_t cnt = offsets ? count : 1;
  // 1) one uncaptured run sizes every buffer and stages the parameters
  ST_TRY(batch_enqueue(ctx, points, off, cnt, vparams, nparams, true));
  CU_TRY(cudaStreamSynchronize(ctx->stream));
  ST_TRY(read_control(ctx));
  // 2) capture the kernels only (the staged parameters stay in the batch arrays)
  srcu_graph *g = new srcu_graph();
  g->clouds = cnt;
  g->attrs = points->n_attrs;
  const uint64_t mask = ctx->prof_mask;
  ctx->prof_mask = 0;  // no timing events inside a graph
  cudaError_t e = cudaStreamBeginCapture(ctx->stream, cudaStreamCaptureModeThreadLocal);
  srcu_status st = SRCU_OK;
  if (e == cudaSuccess) {
    ctx->capturing = true;
    st = batch_enqueue(ctx, points, off, cnt, vparams, nparams, false);
    ctx->capturing = false;
    e = cudaStreamEndCapture(ctx->stream, &g->graph);
  }
  ctx->prof_mask = mask;
  if (e == cudaSuccess && st == SRCU_OK) e = cudaGraphInstantiate(&g->exec, g->graph, 0);
  if (e != cudaSuccess || st != SRCU_OK) {
    cudaGetLastError();
    if (g->exec) cudaGraphExecDestroy(g->exec);
    if (g->graph) cudaGraphDestroy(g->graph);
    delete g;
    if (st != SRCU_OK) return st;
    return fail(ctx, SRCU_ERR_CUDA, "graph capture failed: %s", cudaGetErrorString(e));
  }
  *out = g;
  return SRCU_OK;
}

srcu_status srcu_graph_launch(srcu_ctx *ctx, srcu_graph *g) {
  if (!ctx || !g) return SRCU_ERR_INVALID_ARGUMENT;
  ST_TRY(epoch_guard(ctx));  // the graph's k_begin advances the epoch once
  CU_TRY(cudaGraphLaunch(g->exec, ctx->stream));
  ctx->last_clouds = g->clouds;
  ctx->last_attrs = g->attrs;
  return SRCU_OK;
}

void srcu_graph_destroy(srcu_graph *g) {
  if (!g) return;
  if (g->exec) cudaGraphExecDestroy(g->exec);
  if (g->graph) cudaGraphDestroy(g->graph);
  delete g;
}

srcu_status srcu_batch_voxel_offsets(srcu_ctx *ctx, uint64_t *voxel_offsets) {
  if (!ctx || !voxel_offsets) return SRCU_ERR_INVALID_ARGUMENT;
  const uint32_t count = ctx->last_clouds;
  std::vector<uint32_t> tmp(count + 1);
  if (count > 1)
    CU_TRY(cudaMemcpyAsync(tmp.data(), ctx->b_voff.p, (count + 1) * 4, cudaMemcpyDeviceToHost,
                           ctx->stream));
  ST_TRY(read_control(ctx));
  if (count <= 1) {
    tmp[0] = 0;
    tmp[count] = uint32_t(ctx->ctl_host->n_voxels);
  }
  for (uint32_t b = 0; b <= count; ++b) voxel_offsets[b] = tmp[b];
  return SRCU_OK;
}

srcu_status srcu_frame_view_get(srcu_ctx *ctx, srcu_frame_view *view) {
  if (!ctx || !view) return SRCU_ERR_INVALID_ARGUMENT;
  view->x = ptr<const float>(ctx->vout[0]);
  view->y = ptr<const float>(ctx->vout[1]);
  view->z = ptr<const float>(ctx->vout[2]);
  for (uint32_t a = 0; a < ctx->last_attrs; ++a) ctx->frame_attr_ptrs[a] = ptr<const float>(ctx->vout[3 + a]);
  view->attrs = ctx->frame_attr_ptrs;
  view->n_attrs = ctx->last_attrs;
  view->nx = ptr<const float>(ctx->nout[0]);
  view->ny = ptr<const float>(ctx->nout[1]);
  view->nz = ptr<const float>(ctx->nout[2]);
  view->curvature = ptr<const float>(ctx->nout[3]);
  view->counts = ptr<const uint32_t>(ctx->vcounts);
  view->voxel_count = reinterpret_cast<const uint64_t *>(&ctx->ctl->n_voxels);
  return SRCU_OK;
}

srcu_status srcu_frame_check(srcu_ctx *ctx, uint64_t *out_voxels, srcu_normal_stats *stats) {
  if (!ctx) return SRCU_ERR_INVALID_ARGUMENT;
  ST_TRY(read_control(ctx));
  if (out_voxels) *out_voxels = ctx->ctl_host->n_voxels;
  return fetch_normals(ctx, nullptr, 0, stats);
}

srcu_status srcu_frame_fetch(srcu_ctx *ctx, const srcu_voxel_out *vout, const srcu_normal_out *nout,
                             uint64_t *out_voxels, srcu_normal_stats *stats) {
  if (!ctx) return SRCU_ERR_INVALID_ARGUMENT;
  ST_TRY(read_control(ctx));
  const uint64_t v = ctx->ctl_host->n_voxels;
  if (vout && vout->keys)
    return fail(ctx, SRCU_ERR_INVALID_ARGUMENT, "frame read-back does not unpack voxel keys");
  ST_TRY(fetch_voxels(ctx, 3 + ctx->last_attrs, vout, v));
  ST_TRY(fetch_normals(ctx, nout, v, stats));
  CU_TRY(cudaStreamSynchronize(ctx->stream));
  if (out_voxels) *out_voxels = v;
  return SRCU_OK;
}

srcu_status srcu_chain_info_get(srcu_ctx *ctx, srcu_chain_info *info) {
  if (!ctx || !info) return SRCU_ERR_INVALID_ARGUMENT;
  CU_TRY(cudaMemcpyAsync(ctx->ctl_host, ctx->ctl, sizeof(Control), cudaMemcpyDeviceToHost,
                         ctx->stream));
  CU_TRY(cudaStreamSynchronize(ctx->stream));
  const Control &c = *ctx->ctl_host;
  info->points = c.n_points;
  info->voxels = c.n_voxels;
  info->cells = c.n_cells;
  info->voxel_key_bits = c.vkey_bits + c.cloud_bits;
  info->cell_key_bits = c.ckey_bits + c.cloud_bits;
  info->voxel_sort_passes = c.vsort.passes;
  info->cell_sort_passes = c.csort.passes;
  CellPlan first{};
  CU_TRY(cudaMemcpy(&first, ctx->b_cplans.p, sizeof(CellPlan), cudaMemcpyDeviceToHost));
  info->cell_size = first.h;
  return SRCU_OK;
}

srcu_status srcu_debug_set_epoch(srcu_ctx *ctx, uint32_t epoch) {
  if (!ctx) return SRCU_ERR_INVALID_ARGUMENT;
  if (epoch % EPOCHS_PER_RUN != 0)
    return fail(ctx, SRCU_ERR_INVALID_ARGUMENT, "the epoch must be a multiple of %u", EPOCHS_PER_RUN);
  CU_TRY(cudaSetDevice(ctx->device));
  CU_TRY(cudaStreamSynchronize(ctx->stream));
  CU_TRY(cudaMemcpy(&ctx->ctl->epoch, &epoch, sizeof(epoch), cudaMemcpyHostToDevice));
  ctx->epoch_host = epoch;
  return SRCU_OK;
}

srcu_status srcu_debug_get_epoch(srcu_ctx *ctx, uint32_t *epoch, uint64_t *restarts) {
  if (!ctx) return SRCU_ERR_INVALID_ARGUMENT;
  CU_TRY(cudaSetDevice(ctx->device));
  CU_TRY(cudaStreamSynchronize(ctx->stream));
  uint32_t dev = 0;
  CU_TRY(cudaMemcpy(&dev, &ctx->ctl->epoch, sizeof(dev), cudaMemcpyDeviceToHost));
  if (dev != ctx->epoch_host)
    return fail(ctx, SRCU_ERR_CUDA, "device epoch %u differs from the host mirror %u", dev,
                ctx->epoch_host);
  if (epoch) *epoch = dev;
  if (restarts) *restarts = ctx->epoch_restarts;
  return SRCU_OK;
}

srcu_status srcu_profile_enable(srcu_ctx *ctx, uint64_t timed_kernel_mask) {
  if (!ctx) return SRCU_ERR_INVALID_ARGUMENT;
  ctx->prof_mask = timed_kernel_mask;
  return SRCU_OK;
}

int srcu_profile_read(srcu_ctx *ctx, srcu_kernel_stat *out, int max_entries, int reset) {
  if (!ctx || (!out && max_entries > 0)) return -int(SRCU_ERR_INVALID_ARGUMENT);
  if (cudaStreamSynchronize(ctx->stream) != cudaSuccess) return -int(SRCU_ERR_CUDA);
  for (size_t r = 0; r < ctx->ev_pending.size(); ++r) {
    float ms = 0.f;
    if (cudaEventElapsedTime(&ms, ctx->ev_pool[2 * r], ctx->ev_pool[2 * r + 1]) == cudaSuccess) {
      ctx->timed_ms[ctx->ev_pending[r]] += double(ms);
      ctx->timed[ctx->ev_pending[r]] += 1;
    }
  }
  ctx->ev_pending.clear();
  const int n = std::min<int>(max_entries, SRCU_K_COUNT);
  for (int i = 0; i < n; ++i) {
    memset(&out[i], 0, sizeof(out[i]));
    strncpy(out[i].name, kKernelNames[i], sizeof(out[i].name) - 1);
    out[i].launches = ctx->launches[i];
    out[i].timed_regions = ctx->timed[i];
    out[i].total_ms = ctx->timed_ms[i];
  }
  if (reset) {
    for (int i = 0; i < SRCU_K_COUNT; ++i) {
      ctx->launches[i] = 0;
      ctx->timed[i] = 0;
      ctx->timed_ms[i] = 0.0;
    }
  }
  return n;
}

}  // extern "C"

// The allocation-free variant of the voxel chain shares this translation unit's kernels.
#include "noalloc.cu"
// So do the bounded streaming voxel and the LAS record decoder.
#include "stream.cu"
#include "las.cu"
#include "ransac.cu"
