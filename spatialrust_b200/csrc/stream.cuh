// stream.cuh -- bounded streaming voxel centroids on the device, the
// counterpart of StreamingVoxelSource
// (crates/spatialrust-pipeline/src/streaming.rs:334-700).
//
// Semantics followed (streaming.rs):
//   - the voxel of a point is floor(f64(v) / f64(leaf)) per axis, no origin
//     (voxel_coordinate, :986-994); a coordinate outside the i64 range is an
//     error;
//   - points with a non-finite coordinate are skipped (:464-466);
//   - every column of a voxel is averaged in FP64 over all its points of the
//     whole stream, sum / count (:852-858, :631-633);
//   - voxels come out in ascending (ix, iy, iz) order (:805-838).
//
// Device design.  Chunks fill a device run buffer.  A full run is sorted by
// packed key with the onesweep sort (stable, so a voxel's points stay in
// stream order) and reduced to partial records -- key, count and a
// compensated FP64 sum of every column -- appended to a device record store.
// finish() sorts all partial records by key (stable, so runs stay in stream
// order) and reduces them again into the final records.  Only reduced runs
// stay resident: device memory grows with the distinct voxels of each run,
// not with the length of the stream.
//
// A voxel's sum is compensated (Kahan) within each run and across runs, as
// the reference's CompensatedSum is over the whole stream (:240-262); the
// grouping differs, so means agree to FP64 rounding, not bit for bit.
#pragma once

#include <climits>

#include "radix.cuh"

namespace srcu {

constexpr int SV_THREADS = 256;
constexpr int SV_ITEMS = 4;
constexpr int SV_TILE = SV_THREADS * SV_ITEMS;  // sorted positions per tile
constexpr uint32_t SV_SHORT = 64;  // longer segments are reduced by a whole block
constexpr double SV_I64_EDGE = 9223372036854775808.0;  // 2^63: i64::MIN and i64::MAX as f64

// Packing of one sort: per-axis key minimum and bit widths.  Bit total_bits
// of a packed key marks a skipped (non-finite) point, which sorts last.
struct StreamPlan {
  long long kmin[3];
  uint32_t bits[3];
  uint32_t shift_y, shift_x;
  uint32_t total_bits;
  uint32_t any;  // 1: the sort holds at least one finite point
  uint32_t pad;
};

// Device state of one stream.
struct StreamState {
  long long gmin[3], gmax[3];      // key range over every run's finite points
  unsigned long long finite;       // finite points over all runs
  unsigned long long segments;     // records written by the last reduction
  unsigned long long long_count;   // long segments of the last reduction
  uint32_t overflow;               // 1: a key leaves the i64 range; 2: packed key > 63 bits
  uint32_t pad;
};

// One reduction's inputs: f32 or f64 point columns (bit c of f64_mask), or
// the partial records' FP64 sums and counts.
struct StreamIn {
  const void *col[MAX_COLS];
  uint32_t nc;
  uint32_t f64_mask;
  const unsigned long long *cnt;  // records only
};

// Record store (partial or final): SoA, written at base + slot < cap.
struct StreamOut {
  long long *kx, *ky, *kz;
  unsigned long long *cnt;
  double *sum[MAX_COLS];
  unsigned long long base, cap;
};

// floor(v / leaf) in FP64 as an i64 (streaming.rs:986-994): false when the
// result leaves the range; 2^63 itself saturates like Rust's `as i64`.
__device__ __forceinline__ bool stream_axis_key(float v, double leaf, long long &k) {
  const double c = floor(__ddiv_rn(double(v), leaf));
  if (c < -SV_I64_EDGE || c > SV_I64_EDGE) return false;
  k = c >= SV_I64_EDGE ? LLONG_MAX : (long long)c;
  return true;
}

__device__ __forceinline__ uint64_t stream_pack(const StreamPlan &pl, long long kx, long long ky,
                                                long long kz) {
  const uint64_t fx = uint64_t(kx) - uint64_t(pl.kmin[0]);
  const uint64_t fy = uint64_t(ky) - uint64_t(pl.kmin[1]);
  const uint64_t fz = uint64_t(kz) - uint64_t(pl.kmin[2]);
  return (fx << pl.shift_x) | (fy << pl.shift_y) | fz;
}

__device__ __forceinline__ void stream_unpack(const StreamPlan &pl, uint64_t key, long long &kx,
                                              long long &ky, long long &kz) {
  const uint64_t mz = pl.bits[2] ? (~0ull >> (64 - pl.bits[2])) : 0ull;
  const uint64_t my = pl.bits[1] ? (~0ull >> (64 - pl.bits[1])) : 0ull;
  kz = (long long)(uint64_t(pl.kmin[2]) + (key & mz));
  ky = (long long)(uint64_t(pl.kmin[1]) + ((key >> pl.shift_y) & my));
  kx = (long long)(uint64_t(pl.kmin[0]) + (pl.shift_x < 64 ? (key >> pl.shift_x) : 0ull));
}

__device__ __forceinline__ bool finite3(float x, float y, float z) {
  return isfinite(x) && isfinite(y) && isfinite(z);
}

// Per-axis min/max over the points whose three coordinates are finite (the
// points the stream keeps) of the current run (ctl->n_points of them):
// warp then block reductions, six atomics per block.
__global__ void __launch_bounds__(256) k_stream_bounds(Control *ctl, const float *x, const float *y,
                                                       const float *z, Bounds *out) {
  __shared__ uint32_t red[6][8];
  if (ld_relaxed_u32(&ctl->status)) return;
  const uint64_t n = ctl->n_points;
  uint32_t v6[6] = {0xffffffffu, 0xffffffffu, 0xffffffffu, 0u, 0u, 0u};  // mn xyz, mx xyz
  for (uint64_t i = blockIdx.x * uint64_t(blockDim.x) + threadIdx.x; i < n;
       i += uint64_t(gridDim.x) * blockDim.x) {
    const float v[3] = {x[i], y[i], z[i]};
    if (!finite3(v[0], v[1], v[2])) continue;
#pragma unroll
    for (int a = 0; a < 3; ++a) {
      const uint32_t o = f2ord(v[a]);
      v6[a] = min(v6[a], o);
      v6[3 + a] = max(v6[3 + a], o);
    }
  }
  const uint32_t lane = threadIdx.x & 31u, warp = threadIdx.x >> 5;
#pragma unroll
  for (int a = 0; a < 3; ++a) {
    v6[a] = __reduce_min_sync(FULL_MASK, v6[a]);
    v6[3 + a] = __reduce_max_sync(FULL_MASK, v6[3 + a]);
  }
  if (lane == 0)
    for (int k = 0; k < 6; ++k) red[k][warp] = v6[k];
  __syncthreads();
  if (threadIdx.x == 0) {
    const uint32_t warps = blockDim.x >> 5;
    for (int a = 0; a < 3; ++a) {
      uint32_t mn = red[a][0], mx = red[3 + a][0];
      for (uint32_t w = 1; w < warps; ++w) {
        mn = min(mn, red[a][w]);
        mx = max(mx, red[3 + a][w]);
      }
      if (mn != 0xffffffffu) {
        atomicMin(&out->mn[a], mn);
        atomicMax(&out->mx[a], mx);
      }
    }
  }
}

__device__ __forceinline__ void stream_plan_finish(StreamPlan &pl, const long long (&kmax)[3],
                                                   Control *ctl, StreamState *st) {
  uint32_t total = 0;
  for (int a = 0; a < 3; ++a) {
    pl.bits[a] = bit_width_u64(uint64_t(kmax[a]) - uint64_t(pl.kmin[a]));
    total += pl.bits[a];
  }
  pl.shift_y = pl.bits[2];
  pl.shift_x = pl.bits[1] + pl.bits[2];
  pl.total_bits = total;
  if (total > 63) {
    st->overflow = 2;
    atomicOr(&ctl->status, ST_KEY_OVERFLOW);
  }
}

// Plan of one run from its bounds; widens the stream's key range.  One thread.
__global__ void k_stream_plan(Control *ctl, const Bounds *bd, double leaf, StreamPlan *plan,
                              StreamState *st) {
  if (threadIdx.x != 0 || ld_relaxed_u32(&ctl->status)) return;
  StreamPlan pl{};
  const Bounds b = *bd;
  pl.any = (b.mn[0] != 0xffffffffu) ? 1u : 0u;  // all three axes or none
  long long kmax[3] = {0, 0, 0};
  if (pl.any) {
    for (int a = 0; a < 3; ++a) {
      long long lo, hi;
      if (!stream_axis_key(ord2f(b.mn[a]), leaf, lo) || !stream_axis_key(ord2f(b.mx[a]), leaf, hi)) {
        st->overflow = 1;
        atomicOr(&ctl->status, ST_KEY_OVERFLOW);
        return;
      }
      pl.kmin[a] = lo;
      kmax[a] = hi;
      atomicMin(&st->gmin[a], lo);
      atomicMax(&st->gmax[a], hi);
    }
  }
  stream_plan_finish(pl, kmax, ctl, st);
  *plan = pl;
}

// Plan of the final merge: the key range of every run.  One thread.
__global__ void k_stream_merge_plan(Control *ctl, StreamPlan *plan, StreamState *st) {
  if (threadIdx.x != 0 || ld_relaxed_u32(&ctl->status)) return;
  StreamPlan pl{};
  long long kmax[3] = {0, 0, 0};
  pl.any = st->gmin[0] <= st->gmax[0] ? 1u : 0u;
  if (pl.any)
    for (int a = 0; a < 3; ++a) {
      pl.kmin[a] = st->gmin[a];
      kmax[a] = st->gmax[a];
    }
  stream_plan_finish(pl, kmax, ctl, st);
  *plan = pl;
}

// Sort key of a run's points (ctl->n_points of them).
struct StreamPointSrc {
  const float *x, *y, *z;
  const StreamPlan *plan_ptr;
  double leaf;
  StreamPlan pl;
  __device__ __forceinline__ void prepare(const Control *) { pl = *plan_ptr; }
  __device__ __forceinline__ uint32_t count(const Control *ctl) const { return uint32_t(ctl->n_points); }
  __device__ __forceinline__ uint32_t key_bits() const { return pl.total_bits + 1; }
  __device__ __forceinline__ uint64_t key(uint32_t i) const {
    const float px = x[i], py = y[i], pz = z[i];
    long long kx, ky, kz;
    // a finite point lies inside the run's bounds, so its keys are in range
    if (!finite3(px, py, pz) || !stream_axis_key(px, leaf, kx) || !stream_axis_key(py, leaf, ky) ||
        !stream_axis_key(pz, leaf, kz))
      return 1ull << pl.total_bits;
    return stream_pack(pl, kx, ky, kz);
  }
};

// Sort key of the partial records (ctl->n_points of them).
struct StreamRecordSrc {
  const long long *kx, *ky, *kz;
  const StreamPlan *plan_ptr;
  StreamPlan pl;
  __device__ __forceinline__ void prepare(const Control *) { pl = *plan_ptr; }
  __device__ __forceinline__ uint32_t count(const Control *ctl) const { return uint32_t(ctl->n_points); }
  __device__ __forceinline__ uint32_t key_bits() const { return pl.total_bits + 1; }
  __device__ __forceinline__ uint64_t key(uint32_t i) const {
    return stream_pack(pl, kx[i], ky[i], kz[i]);
  }
};

// A sorted position starts a voxel: kept, and first or unlike its predecessor.
__device__ __forceinline__ bool stream_head(const SortedView &sv, uint64_t flag, uint32_t i,
                                            uint64_t &key) {
  key = sv.key(i);
  if (key & flag) return false;
  return i == 0 || sv.key(i - 1) != key;
}

// Voxel starts per tile of SV_TILE sorted positions (thread t owns positions
// 4t .. 4t+3 of the tile); kept points into st->finite when count_finite.
__global__ void __launch_bounds__(SV_THREADS) k_stream_flags(Control *ctl, SortBuffers sort,
                                                             const SortState *ss,
                                                             const StreamPlan *plan,
                                                             uint32_t *tile_heads, StreamState *st,
                                                             int count_finite) {
  __shared__ uint32_t scratch[SV_THREADS / 32];
  if (ld_relaxed_u32(&ctl->status)) return;
  const uint32_t n = uint32_t(ctl->n_points);
  const uint32_t tiles = (n + SV_TILE - 1) / SV_TILE;
  const SortedView sv = sorted_view(sort, *ss);
  const uint64_t flag = 1ull << plan->total_bits;
  for (uint32_t tile = blockIdx.x; tile < tiles; tile += gridDim.x) {
    uint32_t heads = 0, kept = 0;
#pragma unroll
    for (int k = 0; k < SV_ITEMS; ++k) {
      const uint32_t i = tile * SV_TILE + threadIdx.x * SV_ITEMS + k;
      if (i >= n) break;
      uint64_t key;
      heads += stream_head(sv, flag, i, key) ? 1u : 0u;
      kept += (key & flag) ? 0u : 1u;
    }
    uint32_t total_heads, total_kept;
    block_exclusive_sum<SV_THREADS>(heads, scratch, &total_heads);
    block_exclusive_sum<SV_THREADS>(kept, scratch, &total_kept);
    if (threadIdx.x == 0) {
      tile_heads[tile] = total_heads;
      if (count_finite && total_kept) atomicAdd(&st->finite, (unsigned long long)total_kept);
    }
  }
}

// Exclusive scan of the tile counts (one block of 1024 threads); the total
// is the number of records the reduction writes.
__global__ void __launch_bounds__(1024) k_stream_scan(Control *ctl, const uint32_t *tile_heads,
                                                      uint32_t *tile_off, StreamState *st) {
  __shared__ uint32_t scratch[32];
  if (ld_relaxed_u32(&ctl->status)) return;
  const uint32_t n = uint32_t(ctl->n_points);
  const uint32_t tiles = (n + SV_TILE - 1) / SV_TILE;
  const uint32_t per = (tiles + 1023) / 1024;
  const uint32_t lo = min(tiles, threadIdx.x * per), hi = min(tiles, lo + per);
  uint32_t local = 0;
  for (uint32_t t = lo; t < hi; ++t) local += tile_heads[t];
  uint32_t total;
  uint32_t run = block_exclusive_sum<1024>(local, scratch, &total);
  for (uint32_t t = lo; t < hi; ++t) {
    tile_off[t] = run;
    run += tile_heads[t];
  }
  if (threadIdx.x == 0) {
    st->segments = total;
    st->long_count = 0;
    ctl->n_voxels = total;
  }
}

template <bool Records>
__device__ __forceinline__ double stream_value(const StreamIn &in, uint32_t c, uint32_t v) {
  if (Records || ((in.f64_mask >> c) & 1u)) return static_cast<const double *>(in.col[c])[v];
  return double(static_cast<const float *>(in.col[c])[v]);
}

// Compensated sum (Kahan): the running correction is subtracted from each
// addend, as CompensatedSum::add does (streaming.rs:246-257).
struct Kahan {
  double s = 0.0, c = 0.0;
  __device__ __forceinline__ void add(double v) {
    const double y = __dsub_rn(v, c);
    const double t = __dadd_rn(s, y);
    c = __dsub_rn(__dsub_rn(t, s), y);
    s = t;
  }
};

// Writes the record of the voxel at sorted positions [i, j), reduced by one
// thread in sorted order.
template <bool Records>
__device__ void stream_reduce_short(Control *ctl, const SortedView &sv, const StreamPlan &pl,
                                    const StreamIn &in, const StreamOut &out, uint64_t key,
                                    uint32_t i, uint32_t j, uint64_t slot) {
  const uint64_t r = out.base + slot;
  if (r >= out.cap) {
    atomicOr(&ctl->status, ST_INTERNAL);
    return;
  }
  long long kx, ky, kz;
  stream_unpack(pl, key, kx, ky, kz);
  out.kx[r] = kx;
  out.ky[r] = ky;
  out.kz[r] = kz;
  if (j == i + 1) {
    // one item (the common case): every column's value is its sum, and the
    // column loads are independent, so they are all issued before any is used
    const uint32_t v = sv.val(i);
    out.cnt[r] = Records ? in.cnt[v] : 1ull;
    for (uint32_t c0 = 0; c0 < in.nc; c0 += 4) {
      double val[4];
#pragma unroll
      for (uint32_t k = 0; k < 4; ++k)
        if (c0 + k < in.nc) val[k] = stream_value<Records>(in, c0 + k, v);
#pragma unroll
      for (uint32_t k = 0; k < 4; ++k)
        if (c0 + k < in.nc) out.sum[c0 + k][r] = val[k];
    }
    return;
  }
  unsigned long long cnt = j - i;
  if (Records) {
    cnt = 0;
    for (uint32_t p = i; p < j; ++p) cnt += in.cnt[sv.val(p)];
  }
  out.cnt[r] = cnt;
  for (uint32_t c = 0; c < in.nc; ++c) {
    Kahan k;
    for (uint32_t p = i; p < j; ++p) k.add(stream_value<Records>(in, c, sv.val(p)));
    out.sum[c][r] = k.s;
  }
}

// Records of the voxels that start in each tile: a voxel of at most SV_SHORT
// positions is reduced by the thread holding its start; a longer one is
// queued for k_stream_long.
template <bool Records>
__global__ void __launch_bounds__(SV_THREADS) k_stream_emit(Control *ctl, SortBuffers sort,
                                                            const SortState *ss,
                                                            const StreamPlan *plan,
                                                            const uint32_t *tile_off, StreamIn in,
                                                            StreamOut out, StreamState *st,
                                                            ulonglong2 *long_list,
                                                            uint32_t long_cap) {
  __shared__ uint32_t scratch[SV_THREADS / 32];
  if (ld_relaxed_u32(&ctl->status)) return;
  const uint32_t n = uint32_t(ctl->n_points);
  const uint32_t tiles = (n + SV_TILE - 1) / SV_TILE;
  const SortedView sv = sorted_view(sort, *ss);
  const StreamPlan pl = *plan;
  const uint64_t flag = 1ull << pl.total_bits;
  for (uint32_t tile = blockIdx.x; tile < tiles; tile += gridDim.x) {
    uint32_t heads = 0;
    uint64_t keys[SV_ITEMS];
    bool is_head[SV_ITEMS];
#pragma unroll
    for (int k = 0; k < SV_ITEMS; ++k) {
      const uint32_t i = tile * SV_TILE + threadIdx.x * SV_ITEMS + k;
      is_head[k] = i < n && stream_head(sv, flag, i, keys[k]);
      heads += is_head[k] ? 1u : 0u;
    }
    uint32_t total;
    uint32_t rank = block_exclusive_sum<SV_THREADS>(heads, scratch, &total);
#pragma unroll
    for (int k = 0; k < SV_ITEMS; ++k) {
      if (!is_head[k]) continue;
      const uint32_t i = tile * SV_TILE + threadIdx.x * SV_ITEMS + k;
      const uint64_t slot = uint64_t(tile_off[tile]) + rank++;
      uint32_t j = i + 1;
      while (j < n && j - i < SV_SHORT && sv.key(j) == keys[k]) ++j;
      if (j < n && j - i == SV_SHORT && sv.key(j) == keys[k]) {
        const unsigned long long q = atomicAdd(&st->long_count, 1ull);
        if (q < long_cap) long_list[q] = make_ulonglong2(i, slot);
        else atomicOr(&ctl->status, ST_INTERNAL);
        continue;
      }
      stream_reduce_short<Records>(ctl, sv, pl, in, out, keys[k], i, j, slot);
    }
  }
}

// One block per queued long voxel: finds its end, then reduces every column
// with per-thread compensated sums combined in thread order.
template <bool Records>
__global__ void __launch_bounds__(SV_THREADS) k_stream_long(Control *ctl, SortBuffers sort,
                                                            const SortState *ss,
                                                            const StreamPlan *plan, StreamIn in,
                                                            StreamOut out, const StreamState *st,
                                                            const ulonglong2 *long_list) {
  __shared__ unsigned long long end_s;
  __shared__ double red[SV_THREADS];
  __shared__ unsigned long long redc[SV_THREADS];
  if (ld_relaxed_u32(&ctl->status)) return;
  const uint32_t n = uint32_t(ctl->n_points);
  const SortedView sv = sorted_view(sort, *ss);
  const StreamPlan pl = *plan;
  const unsigned long long count = st->long_count;
  const uint32_t t = threadIdx.x;
  for (unsigned long long e = blockIdx.x; e < count; e += gridDim.x) {
    const ulonglong2 item = long_list[e];
    const uint32_t start = uint32_t(item.x);
    const uint64_t key = sv.key(start);
    if (t == 0) end_s = n;
    __syncthreads();
    for (uint32_t base = start; base < n; base += SV_THREADS) {
      const uint32_t p = base + t;
      if (p < n && sv.key(p) != key) atomicMin(&end_s, (unsigned long long)p);
      __syncthreads();
      const unsigned long long e_s = end_s;
      __syncthreads();
      if (e_s < base + SV_THREADS) break;
    }
    const uint32_t end = uint32_t(end_s);
    const uint64_t r = out.base + item.y;
    const bool ok = r < out.cap;
    unsigned long long cnt = 0;
    for (uint32_t p = start + t; p < end; p += SV_THREADS) cnt += Records ? in.cnt[sv.val(p)] : 1ull;
    redc[t] = cnt;
    __syncthreads();
    for (uint32_t w = SV_THREADS / 2; w > 0; w >>= 1) {
      if (t < w) redc[t] += redc[t + w];
      __syncthreads();
    }
    if (t == 0) {
      if (ok) {
        long long kx, ky, kz;
        stream_unpack(pl, key, kx, ky, kz);
        out.kx[r] = kx;
        out.ky[r] = ky;
        out.kz[r] = kz;
        out.cnt[r] = redc[0];
      } else {
        atomicOr(&ctl->status, ST_INTERNAL);
      }
    }
    for (uint32_t c = 0; c < in.nc; ++c) {
      Kahan k;
      for (uint32_t p = start + t; p < end; p += SV_THREADS)
        k.add(stream_value<Records>(in, c, sv.val(p)));
      red[t] = k.s;
      __syncthreads();
      if (t == 0) {
        Kahan tot;
        for (uint32_t w = 0; w < SV_THREADS; ++w) tot.add(red[w]);
        if (ok) out.sum[c][r] = tot.s;
      }
      __syncthreads();
    }
  }
}

// Outputs of finish(): positions as f32, the other columns' means in FP64,
// (ix, iy, iz) triples.
struct StreamFinal {
  float *pos[3];
  double *attr[MAX_COLS];
  long long *keys3;
};

// Final records -> outputs: positions (sum / count) as f32, the other
// columns' means in FP64 (narrowed by the caller per field type, as
// push_scalar does, streaming.rs:922-938).
__global__ void __launch_bounds__(256) k_stream_finalize(Control *ctl, StreamOut fin, uint32_t nc,
                                                         StreamFinal o) {
  if (ld_relaxed_u32(&ctl->status)) return;
  const unsigned long long v = ctl->n_voxels;
  for (unsigned long long r = blockIdx.x * uint64_t(blockDim.x) + threadIdx.x; r < v;
       r += uint64_t(gridDim.x) * blockDim.x) {
    const double cnt = __ull2double_rn(fin.cnt[r]);
    for (uint32_t c = 0; c < 3; ++c) o.pos[c][r] = __double2float_rn(__ddiv_rn(fin.sum[c][r], cnt));
    for (uint32_t c = 3; c < nc; ++c) o.attr[c - 3][r] = __ddiv_rn(fin.sum[c][r], cnt);
    o.keys3[3 * r] = fin.kx[r];
    o.keys3[3 * r + 1] = fin.ky[r];
    o.keys3[3 * r + 2] = fin.kz[r];
  }
}

}  // namespace srcu
