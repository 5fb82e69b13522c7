// voxel.cuh -- bounds, voxel-key plan, and the fused segment + centroid
// reduction of the VoxelGrid centroid downsample.
#pragma once

#include "radix.cuh"

namespace srcu {

constexpr int BND_THREADS = 256;

// k_begin: zeroes the control block for a new chain, advances the epoch and
// resets the per-cloud bounds.  For a single cloud it also writes the batch
// arrays (offsets {0, n} and the cloud's parameters) so that no host copy is
// needed.
__global__ void k_begin(Control *ctl, unsigned long long n_points, Batch bt, uint32_t cloud_bits,
                        int single, VoxelParamsDev vp0, NormalParamsDev np0) {
  const uint32_t t = threadIdx.x;
  if (single && t == 0) {
    uint32_t *off = const_cast<uint32_t *>(bt.offsets);
    off[0] = 0;
    off[1] = uint32_t(n_points);
    if (bt.vparams) *const_cast<VoxelParamsDev *>(bt.vparams) = vp0;
    if (bt.nparams) *const_cast<NormalParamsDev *>(bt.nparams) = np0;
  }
  uint32_t *w = reinterpret_cast<uint32_t *>(ctl);
  const uint32_t words = sizeof(Control) / 4;
  // word 0 is the epoch
  for (uint32_t i = 1 + t; i < words; i += blockDim.x) w[i] = 0;
  for (uint32_t b = t; b < bt.clouds; b += blockDim.x) {
    Bounds z;
    for (int a = 0; a < 3; ++a) {
      z.mn[a] = 0xffffffffu;  // atomicMin target
      z.mx[a] = 0u;
    }
    z.flags = 0;
    z.pad = 0;
    bt.bounds[b] = z;
  }
  __syncthreads();
  if (t == 0) {
    ctl->epoch += EPOCHS_PER_RUN;
    ctl->n_points = n_points;
    ctl->clouds = bt.clouds;
    ctl->cloud_bits = cloud_bits;
  }
}

struct BoundsAcc {
  uint32_t mn[3], mx[3], flags;
  __device__ __forceinline__ void reset() {
    for (int a = 0; a < 3; ++a) {
      mn[a] = 0xffffffffu;
      mx[a] = 0u;
    }
    flags = 0;
  }
  __device__ __forceinline__ void add(float x, float y, float z) {
    const float v[3] = {x, y, z};
#pragma unroll
    for (int a = 0; a < 3; ++a) {
      if (isnan(v[a])) {
        flags |= 1u << a;
      } else if (isinf(v[a])) {
        flags |= 8u << a;
      } else {
        const uint32_t o = f2ord(v[a]);
        mn[a] = min(mn[a], o);
        mx[a] = max(mx[a], o);
      }
    }
  }
  __device__ __forceinline__ void flush(Bounds &b) const {
#pragma unroll
    for (int a = 0; a < 3; ++a) {
      if (mn[a] != 0xffffffffu) atomicMin(&b.mn[a], mn[a]);
      if (mx[a] != 0u) atomicMax(&b.mx[a], mx[a]);
    }
    if (flags) atomicOr(&b.flags, flags);
  }
};

constexpr uint32_t BND_CHUNK = 32;  // points per lane of a warp span in the multi-cloud case

// Interleaved input records (srcu_cloud.stride > 1) -> packed columns.
struct Interleaved {
  const float *src[MAX_COLS];
  float *dst[MAX_COLS];
  uint32_t nc, stride;
};

__global__ void k_deinterleave(Interleaved iv, uint64_t n) {
  for (uint64_t i = blockIdx.x * uint64_t(blockDim.x) + threadIdx.x; i < n;
       i += uint64_t(gridDim.x) * blockDim.x)
    for (uint32_t c = 0; c < iv.nc; ++c) iv.dst[c][i] = iv.src[c][i * iv.stride];
}

// Per-cloud min/max over finite coordinates plus NaN / inf flags
// (compute_bounds, voxel.rs:1067-1079, ignores NaN through f32::min/max).
// The point count comes from *count_dev when non-null, else ctl->n_points.
// Optionally writes an AoS copy (x, y, z, first attribute) so that later
// gathers by point index touch one 32-byte sector per point.
__global__ void __launch_bounds__(BND_THREADS) k_bounds(const float *x, const float *y,
                                                        const float *z, Control *ctl,
                                                        const unsigned long long *count_dev,
                                                        const float *a0, float4 *aos, Batch bt) {
  if (ld_relaxed_u32(&ctl->status)) return;
  const uint64_t n = count_dev ? *count_dev : ctl->n_points;
  if (bt.clouds == 1) {
    BoundsAcc acc;
    acc.reset();
    const uint64_t stride = uint64_t(gridDim.x) * BND_THREADS;
    uint64_t i = blockIdx.x * uint64_t(BND_THREADS) + threadIdx.x;
    // four points per thread in flight: all loads first, then the stores
    for (; i + 3 * stride < n; i += 4 * stride) {
      float px[4], py[4], pz[4], pa[4];
#pragma unroll
      for (int q = 0; q < 4; ++q) {
        const uint64_t k = i + uint64_t(q) * stride;
        px[q] = x[k];
        py[q] = y[k];
        pz[q] = z[k];
        pa[q] = a0 ? a0[k] : 0.0f;
      }
#pragma unroll
      for (int q = 0; q < 4; ++q) {
        if (aos) aos[i + uint64_t(q) * stride] = make_float4(px[q], py[q], pz[q], pa[q]);
        acc.add(px[q], py[q], pz[q]);
      }
    }
    for (; i < n; i += stride) {
      const float xi = x[i], yi = y[i], zi = z[i];
      if (aos) aos[i] = make_float4(xi, yi, zi, a0 ? a0[i] : 0.0f);
      acc.add(xi, yi, zi);
    }
#pragma unroll
    for (int a = 0; a < 3; ++a) {
#pragma unroll
      for (int o = 16; o > 0; o >>= 1) {
        acc.mn[a] = min(acc.mn[a], __shfl_xor_sync(FULL_MASK, acc.mn[a], o));
        acc.mx[a] = max(acc.mx[a], __shfl_xor_sync(FULL_MASK, acc.mx[a], o));
      }
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) acc.flags |= __shfl_xor_sync(FULL_MASK, acc.flags, o);
    // one flush per block: warp results meet in shared memory first
    __shared__ uint32_t sred[BND_THREADS / 32][7];
    const uint32_t lane = threadIdx.x & 31u, warp = threadIdx.x >> 5;
    if (lane == 0) {
      for (int a = 0; a < 3; ++a) {
        sred[warp][a] = acc.mn[a];
        sred[warp][3 + a] = acc.mx[a];
      }
      sred[warp][6] = acc.flags;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
      for (uint32_t w = 1; w < BND_THREADS / 32; ++w) {
        for (int a = 0; a < 3; ++a) {
          acc.mn[a] = min(acc.mn[a], sred[w][a]);
          acc.mx[a] = max(acc.mx[a], sred[w][3 + a]);
        }
        acc.flags |= sred[w][6];
      }
      acc.flush(bt.bounds[0]);
    }
    return;
  }
  // Many clouds: each warp owns a span of 32 * BND_CHUNK consecutive points,
  // read coalesced.  A span inside one cloud (all but at most one span per
  // cloud boundary) reduces across the warp and flushes once; a span that
  // crosses a boundary flushes per lane whenever its cloud changes.
  const uint32_t lane = threadIdx.x & 31u;
  const uint64_t span = 32ull * BND_CHUNK;
  const uint64_t spans = (n + span - 1) / span;
  const uint64_t warps = uint64_t(gridDim.x) * (BND_THREADS / 32);
  for (uint64_t sp = blockIdx.x * uint64_t(BND_THREADS / 32) + (threadIdx.x >> 5); sp < spans;
       sp += warps) {
    const uint64_t s0 = sp * span;
    const uint64_t s1 = s0 + span < n ? s0 + span : n;
    const uint32_t b0 = cloud_of(bt, uint32_t(s0));
    const uint32_t b1 = cloud_of(bt, uint32_t(s1 - 1));
    BoundsAcc acc;
    acc.reset();
    if (b0 == b1) {
      uint64_t i = s0 + lane;
      // four points per lane in flight: all loads first, then the stores
      for (; i + 96 < s1; i += 128) {
        float px[4], py[4], pz[4], pa[4];
#pragma unroll
        for (int q = 0; q < 4; ++q) {
          const uint64_t k = i + 32u * q;
          px[q] = x[k];
          py[q] = y[k];
          pz[q] = z[k];
          pa[q] = a0 ? a0[k] : 0.0f;
        }
#pragma unroll
        for (int q = 0; q < 4; ++q) {
          if (aos) aos[i + 32u * q] = make_float4(px[q], py[q], pz[q], pa[q]);
          acc.add(px[q], py[q], pz[q]);
        }
      }
      for (; i < s1; i += 32) {
        const float xi = x[i], yi = y[i], zi = z[i];
        if (aos) aos[i] = make_float4(xi, yi, zi, a0 ? a0[i] : 0.0f);
        acc.add(xi, yi, zi);
      }
#pragma unroll
      for (int a = 0; a < 3; ++a) {
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) {
          acc.mn[a] = min(acc.mn[a], __shfl_xor_sync(FULL_MASK, acc.mn[a], o));
          acc.mx[a] = max(acc.mx[a], __shfl_xor_sync(FULL_MASK, acc.mx[a], o));
        }
      }
#pragma unroll
      for (int o = 16; o > 0; o >>= 1) acc.flags |= __shfl_xor_sync(FULL_MASK, acc.flags, o);
      if (lane == 0) acc.flush(bt.bounds[b0]);
    } else {
      uint32_t b = b0;
      uint32_t next = __ldg(bt.offsets + b + 1);
      for (uint64_t i = s0 + lane; i < s1; i += 32) {
        while (i >= next) {  // crossed into a later cloud (skipping empty ones)
          acc.flush(bt.bounds[b]);
          acc.reset();
          ++b;
          next = __ldg(bt.offsets + b + 1);
        }
        const float xi = x[i], yi = y[i], zi = z[i];
        if (aos) aos[i] = make_float4(xi, yi, zi, a0 ? a0[i] : 0.0f);
        acc.add(xi, yi, zi);
      }
      acc.flush(bt.bounds[b]);
    }
  }
}

// One voxel-key plan per cloud from its bounds and parameters
// (filter_internal, voxel.rs:266-275).  The per-cloud key widths are reduced
// to their maximum (ctl->vkey_bits); a cloud whose key plus the cloud id does
// not fit in 64 bits stops the chain with ST_KEY_OVERFLOW.
__global__ void k_voxel_plans(Control *ctl, Batch bt) {
  if (ld_relaxed_u32(&ctl->status)) return;
  const uint32_t b = blockIdx.x * blockDim.x + threadIdx.x;
  if (b >= bt.clouds) return;
  const VoxelParamsDev prm = bt.vparams[b];
  VoxelPlan pl{};
  pl.inv_leaf = __fdiv_rn(1.0f, prm.leaf);  // f32 IEEE division, voxel.rs:267
  pl.floor_mode = prm.has_origin ? 1 : 0;
  const Bounds bd = bt.bounds[b];
  float lo[3], hi[3];
  for (int a = 0; a < 3; ++a) {
    const bool any = bd.mn[a] != 0xffffffffu;
    lo[a] = any ? ord2f(bd.mn[a]) : __int_as_float(0x7fc00000);  // all-NaN axis -> NaN
    hi[a] = any ? ord2f(bd.mx[a]) : __int_as_float(0x7fc00000);
  }
  for (int a = 0; a < 3; ++a) pl.origin[a] = prm.has_origin ? prm.origin[a] : lo[a];
  bool ok = (bd.flags & (7u << 3)) == 0;  // an infinite coordinate saturates the key
  uint32_t total = 0;
  for (int a = 0; a < 3; ++a) {
    int64_t k0 = voxel_axis_key(lo[a], pl.origin[a], pl.inv_leaf, pl.floor_mode);
    int64_t k1 = voxel_axis_key(hi[a], pl.origin[a], pl.inv_leaf, pl.floor_mode);
    if (isnan(lo[a])) k0 = k1 = 0;
    if (bd.flags & (1u << a)) {  // NaN coordinates get key 0 (saturating cast)
      k0 = min(k0, int64_t(0));
      k1 = max(k1, int64_t(0));
    }
    pl.kmin[a] = k0;
    const uint64_t range = uint64_t(k1) - uint64_t(k0);
    pl.bits[a] = bit_width_u64(range);
    total += pl.bits[a];
  }
  pl.shift_y = pl.bits[2];
  pl.shift_x = pl.bits[1] + pl.bits[2];
  pl.total_bits = total;
  pl.num_digits = total == 0 ? 1u : (total + RADIX_BITS - 1) / RADIX_BITS;
  if (total + ctl->cloud_bits > 64) ok = false;
  if (ctl->n_points > LB_MAX_COUNT) {
    atomicOr(&ctl->status, ST_TOO_MANY_POINTS);
    ok = false;
  }
  pl.valid = ok ? 1u : 0u;
  bt.vplans[b] = pl;
  atomicMax(&ctl->vkey_bits, total);
  if (!ok) atomicOr(&ctl->status, ST_KEY_OVERFLOW);
}

// Key source for the voxel sort: the reference's voxel key of point i,
// packed, with its cloud id above the per-cloud key bits.
struct VoxelKeySrc {
  const float *x, *y, *z;
  Batch bt;
  VoxelPlan pl;  // the plan when there is one cloud
  uint32_t local_bits;
  uint32_t cloud_bits;
  __device__ __forceinline__ void prepare(const Control *ctl) {
    local_bits = ctl->vkey_bits;
    cloud_bits = ctl->cloud_bits;
    if (bt.clouds == 1) pl = bt.vplans[0];
  }
  __device__ __forceinline__ uint32_t count(const Control *ctl) const {
    return uint32_t(ctl->n_points);
  }
  __device__ __forceinline__ uint32_t key_bits() const { return local_bits + cloud_bits; }
  __device__ __forceinline__ uint64_t key(uint32_t i) const {
    if (bt.clouds == 1) return voxel_pack(pl, x[i], y[i], z[i]);
    const uint32_t b = cloud_of(bt, i);
    return with_cloud(voxel_pack(bt.vplans[b], x[i], y[i], z[i]), b, local_bits);
  }
};

template <int NC>
struct Columns {
  const float *in[NC];
  float *out[NC];
};

constexpr int SEG_THREADS = 256;
constexpr int SEG_ITEMS = 4;
constexpr int SEG_TILE = SEG_THREADS * SEG_ITEMS;  // 1024 sorted positions per tile
constexpr uint32_t SEG_SHORT = 32;  // longer voxels are reduced by a whole warp

// Shared memory of k_voxel_segments<NC>: the tile's keys (plus one before and
// one after), the scan scratch, and the tile's gathered point columns.
struct SegmentSmemHead {
  uint64_t keys[SEG_TILE + 2];  // keys[0] = key before the tile, keys[1 + tile_n] = key after it
  uint32_t scratch[SEG_THREADS / 32];
  uint32_t tile;
  uint32_t pad;
};
__host__ __device__ constexpr size_t segment_smem_bytes(int nc) {
  return sizeof(SegmentSmemHead) + size_t(nc) * SEG_TILE * sizeof(float);
}

// Aggregation of the voxel whose packed key is `key`: agg_all when the host
// knows every cloud of the chain shares one, else the voxel's cloud's mode.
__device__ __forceinline__ int32_t voxel_agg(const Batch &bt, uint64_t key, uint32_t vkey_bits,
                                             int32_t agg_all) {
  if (agg_all >= 0) return agg_all;
  const uint32_t b = (bt.clouds == 1 || vkey_bits >= 64) ? 0u : uint32_t(key >> vkey_bits);
  return bt.vparams[b < bt.clouds ? b : 0].agg;
}

// Writes one voxel.  s: FP64 sums of every column in ascending point order;
// first(c): column c of the voxel's first point, read only by the modes that
// use it (so the default mode keeps no extra registers live).
//   AGG_FAST            (sum * (1.0 / count)) as f32, voxel.rs:531-536
//   AGG_CENTROID_FIRST  positions (sum / count) as f32 (average_field,
//                       voxel.rs:1156-1165), other fields from the first point
//   AGG_FIRST           every field from the first point (voxel.rs:1144-1146)
template <int NC, class First>
__device__ __forceinline__ void write_centroid(const Columns<NC> &cols, const double (&s)[NC],
                                               First first, int32_t agg,
                                               uint32_t cnt, uint32_t seg, uint64_t key,
                                               uint64_t *out_keys, uint32_t *out_counts,
                                               uint32_t n, uint32_t *status, float4 *aos_out) {
  if (seg >= n) {  // cannot happen for a consistent sort; never write out of bounds
    atomicOr(status, ST_INTERNAL);
    return;
  }
  const double inv = 1.0 / double(cnt);
  float o[NC];
#pragma unroll
  for (int c = 0; c < NC; ++c) {
    if (agg == AGG_FAST) o[c] = __double2float_rn(__dmul_rn(s[c], inv));
    else if (agg == AGG_CENTROID_FIRST && c < 3)
      o[c] = __double2float_rn(__ddiv_rn(s[c], double(cnt)));
    else o[c] = first(c);
    cols.out[c][seg] = o[c];
  }
  if (aos_out) aos_out[seg] = make_float4(o[0], o[1], o[2], 0.0f);
  out_keys[seg] = key;
  out_counts[seg] = cnt;
}

// Fused segment discovery + FP64 centroid reduction over the sorted
// (key, index) pairs.  Each tile gathers its points' columns into shared
// memory with all threads at once (independent loads, so the random gather
// overlaps), flags voxel starts, numbers them with a block scan plus
// decoupled look-back, and reduces every voxel that starts in it: one thread
// per short voxel (sequential FP64 sum in ascending point index, the
// reference's order, voxel.rs:502-520), one warp per long voxel or per voxel
// that runs past the tile end.
template <int NC>
__global__ void __launch_bounds__(SEG_THREADS, 5) k_voxel_segments(Control *ctl, SortBuffers sort,
                                                                 const SortState *sort_state,
                                                                 Columns<NC> cols,
                                                                 uint64_t *out_keys,
                                                                 uint32_t *out_counts,
                                                                 uint64_t *lookback,
                                                                 const float4 *aos_in,
                                                                 float4 *aos_out, Batch bt,
                                                                 int32_t agg_all) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  SegmentSmemHead &sm = *reinterpret_cast<SegmentSmemHead *>(smem_raw);
  float *scol = reinterpret_cast<float *>(smem_raw + sizeof(SegmentSmemHead));  // [NC][SEG_TILE]
  if (ld_relaxed_u32(&ctl->status)) return;
  const uint32_t n = uint32_t(ctl->n_points);
  if (n == 0) return;
  const SortedView sv = sorted_view(sort, *sort_state);
  const uint32_t epoch = ctl->epoch + EP_VSEG;
  const uint32_t num_tiles = (n + SEG_TILE - 1) / SEG_TILE;
  const uint32_t t = threadIdx.x, lane = t & 31u;

  for (;;) {
    if (t == 0) sm.tile = atomicAdd(&ctl->work[WK_VSEG], 1u);
    __syncthreads();
    const uint32_t tile = sm.tile;
    if (tile >= num_tiles) break;
    const uint32_t base = tile * SEG_TILE;
    const uint32_t tile_n = min(uint32_t(SEG_TILE), n - base);
    // The tile's sorted items, then their points: every thread issues all of
    // its SEG_ITEMS item loads, then all of its random point gathers, before
    // any of them is consumed, so the gathers' latencies overlap.
    uint64_t ik[SEG_ITEMS];
    uint32_t iv[SEG_ITEMS];
    uint64_t k_before = 0, k_after = 0;  // the keys either side of the tile (thread 0)
    if (t == 0) {
      k_before = base > 0 ? sv.key(base - 1) : ~sv.key(0);
      k_after = base + tile_n < n ? sv.key(base + tile_n) : ~sv.key(n - 1);
    }
#pragma unroll
    for (int q = 0; q < SEG_ITEMS; ++q) {
      const uint32_t j = t + uint32_t(q) * SEG_THREADS;
      ik[q] = 0;
      iv[q] = n;  // out of range: no gather
      if (j < tile_n) sv.get(base + j, ik[q], iv[q]);
    }
    if (aos_in) {  // columns 0..3 from the AoS copy: one sector per point
      float4 pt[SEG_ITEMS];
#pragma unroll
      for (int q = 0; q < SEG_ITEMS; ++q)
        pt[q] = iv[q] < n ? aos_in[iv[q]] : make_float4(0.f, 0.f, 0.f, 0.f);
#pragma unroll
      for (int q = 0; q < SEG_ITEMS; ++q) {
        const uint32_t j = t + uint32_t(q) * SEG_THREADS;
        if (j >= tile_n) continue;
        scol[0 * SEG_TILE + j] = pt[q].x;
        scol[1 * SEG_TILE + j] = pt[q].y;
        scol[2 * SEG_TILE + j] = pt[q].z;
        if (NC > 3) scol[3 * SEG_TILE + j] = pt[q].w;
      }
    }
#pragma unroll
    for (int q = 0; q < SEG_ITEMS; ++q) {
      const uint32_t j = t + uint32_t(q) * SEG_THREADS;
      if (j >= tile_n) continue;
      sm.keys[1 + j] = ik[q];
      const uint32_t v = iv[q];
      if (v < n) {
#pragma unroll
        for (int c = aos_in ? 4 : 0; c < NC; ++c) scol[c * SEG_TILE + j] = cols.in[c][v];
      } else {  // a consistent sort never produces this; never read out of bounds
        atomicOr(&ctl->status, ST_INTERNAL);
#pragma unroll
        for (int c = 0; c < NC; ++c) scol[c * SEG_TILE + j] = 0.0f;
      }
    }
    if (t == 0) {
      sm.keys[0] = k_before;
      sm.keys[1 + tile_n] = k_after;
    }
    __syncthreads();

    const uint32_t j0 = t * SEG_ITEMS;
    uint32_t flags = 0;
#pragma unroll
    for (int i = 0; i < SEG_ITEMS; ++i) {
      const uint32_t j = j0 + i;
      if (j < tile_n && sm.keys[1 + j] != sm.keys[j]) flags |= 1u << i;
    }
    uint32_t tile_count;
    const uint32_t local = block_exclusive_sum<SEG_THREADS>(__popc(flags), sm.scratch, &tile_count);
    uint32_t seg_base = 0;
    if (t < 32) {
      seg_base = lookback_exclusive_warp(lookback, tile, tile_count, epoch, &ctl->status);
      if (t == 0) sm.scratch[0] = seg_base;
    }
    __syncthreads();
    seg_base = sm.scratch[0];
    if (t == 0 && tile == num_tiles - 1) ctl->n_voxels = seg_base + tile_count;

    // Short voxels: the owning thread reduces sequentially from shared memory.
    // At most one voxel per thread (its last start) can be long or run past
    // the tile.
    bool deferred = false;
    uint32_t def_pos = 0, def_seg = 0;
    uint32_t seg = seg_base + local;
    for (int i = 0; i < SEG_ITEMS; ++i) {
      if (!(flags & (1u << i))) continue;
      const uint32_t j = j0 + i;
      const uint64_t key = sm.keys[1 + j];
      uint32_t e = j + 1;
      while (e < tile_n && e - j <= SEG_SHORT && sm.keys[1 + e] == key) ++e;
      const bool closed = sm.keys[1 + e] != key;  // keys[1 + tile_n] is the key after the tile
      if (closed && e - j <= SEG_SHORT) {
        double s[NC];
#pragma unroll
        for (int c = 0; c < NC; ++c) s[c] = 0.0;
        for (uint32_t m = j; m < e; ++m) {
#pragma unroll
          for (int c = 0; c < NC; ++c) s[c] += double(scol[c * SEG_TILE + m]);
        }
        write_centroid<NC>(cols, s, [&](int c) { return scol[c * SEG_TILE + j]; },
                           voxel_agg(bt, key, ctl->vkey_bits, agg_all), e - j, seg, key, out_keys,
                           out_counts, n, &ctl->status, aos_out);
      } else {
        deferred = true;
        def_pos = base + j;
        def_seg = seg;
      }
      ++seg;
    }
    // Long voxels: the whole warp finds the end and reduces from global memory.
    uint32_t pending = __ballot_sync(FULL_MASK, deferred);
    while (pending) {
      const uint32_t src_lane = __ffs(pending) - 1;
      pending &= pending - 1;
      const uint32_t p = __shfl_sync(FULL_MASK, def_pos, src_lane);
      const uint32_t sg = __shfl_sync(FULL_MASK, def_seg, src_lane);
      const uint64_t key = sv.key(p);
      uint32_t e = p + 1;
      for (;;) {
        const uint32_t idx = e + lane;
        const bool stop = idx >= n || sv.key(idx) != key;
        const uint32_t b = __ballot_sync(FULL_MASK, stop);
        if (b) {
          e += __ffs(b) - 1;
          break;
        }
        e += 32;
      }
      double s[NC];
#pragma unroll
      for (int c = 0; c < NC; ++c) s[c] = 0.0;
      for (uint32_t m = p + lane; m < e; m += 32) {
        const uint32_t v = sv.val(m);
        if (v >= n) {
          atomicOr(&ctl->status, ST_INTERNAL);
          continue;
        }
#pragma unroll
        for (int c = 0; c < NC; ++c) s[c] += double(cols.in[c][v]);
      }
#pragma unroll
      for (int c = 0; c < NC; ++c)
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) s[c] += __shfl_xor_sync(FULL_MASK, s[c], o);
      if (lane == 0) {
        // the voxel's first point is the first sorted item (stable sort)
        auto first = [&](int c) {
          const uint32_t v0 = sv.val(p);
          return v0 < n ? cols.in[c][v0] : 0.0f;
        };
        write_centroid<NC>(cols, s, first, voxel_agg(bt, key, ctl->vkey_bits, agg_all), e - p, sg,
                           key, out_keys, out_counts, n, &ctl->status, aos_out);
      }
    }
    __syncthreads();
  }
}

// Opts every k_voxel_segments<NC> instantiation into the shared memory it
// needs (more than 48 KB for many attribute columns).
template <int NC>
inline cudaError_t configure_segments_nc() {
  return cudaFuncSetAttribute(k_voxel_segments<NC>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                              int(segment_smem_bytes(NC)));
}
inline cudaError_t configure_segment_kernels() {
  cudaError_t e = cudaSuccess;
  const cudaError_t all[] = {configure_segments_nc<3>(),  configure_segments_nc<4>(),
                             configure_segments_nc<5>(),  configure_segments_nc<6>(),
                             configure_segments_nc<7>(),  configure_segments_nc<8>(),
                             configure_segments_nc<9>(),  configure_segments_nc<10>(),
                             configure_segments_nc<11>(), configure_segments_nc<12>()};
  for (cudaError_t x : all)
    if (x != cudaSuccess) e = x;
  return e;
}

// ---- the reference's plain-xyz fast path --------------------------------------
// filter_cpu_xyz_centroid_fast (crates/spatialrust-filtering/src/voxel.rs:550-636)
// runs for clouds whose only fields are x, y, z: per voxel it sums x, y, z in
// f32 in input order, emits sum * (1 / count) in f32, and emits the voxels in
// the order of their first point.  After the segment kernel (same voxels, same
// counts, key order), k_voxel_xyz_f32 recomputes those sums -- the stable sort
// keeps each voxel's points in input order -- and records each voxel's first
// point; a sort of the voxels by first point (FirstSeenSrc) and a gather then
// put them in first-seen order.

// One thread per voxel start among the sorted items.
__global__ void k_voxel_xyz_f32(Control *ctl, SortBuffers sort, const SortState *sort_state,
                                const float *x, const float *y, const float *z,
                                const uint64_t *vkeys, const uint32_t *vcounts, float *ox,
                                float *oy, float *oz, uint32_t *first) {
  if (ld_relaxed_u32(&ctl->status)) return;
  const uint32_t n = uint32_t(ctl->n_points);
  const uint32_t nv = uint32_t(ctl->n_voxels);
  const SortedView sv = sorted_view(sort, *sort_state);
  for (uint32_t m = blockIdx.x * blockDim.x + threadIdx.x; m < n; m += gridDim.x * blockDim.x) {
    const uint64_t key = sv.key(m);
    if (m > 0 && sv.key(m - 1) == key) continue;
    uint32_t lo = 0, hi = nv;  // the voxel of this key among the key-ordered voxels
    while (lo < hi) {
      const uint32_t mid = (lo + hi) >> 1;
      if (vkeys[mid] < key) lo = mid + 1;
      else hi = mid;
    }
    if (lo >= nv || vkeys[lo] != key || vcounts[lo] == 0 || vcounts[lo] > n - m) {
      atomicOr(&ctl->status, ST_INTERNAL);  // cannot happen for a consistent chain
      continue;
    }
    const uint32_t cnt = vcounts[lo];
    float sx = 0.0f, sy = 0.0f, sz = 0.0f;
    uint32_t i0 = 0;
    bool ok = true;
    for (uint32_t q = 0; q < cnt; ++q) {
      const uint32_t i = sv.val(m + q);
      if (i >= n) {
        ok = false;
        break;
      }
      if (q == 0) i0 = i;
      sx = __fadd_rn(sx, x[i]);
      sy = __fadd_rn(sy, y[i]);
      sz = __fadd_rn(sz, z[i]);
    }
    if (!ok) {
      atomicOr(&ctl->status, ST_INTERNAL);
      continue;
    }
    const float inv = 1.0f / float(cnt);  // IEEE division: the library is built without fast math
    ox[lo] = __fmul_rn(sx, inv);
    oy[lo] = __fmul_rn(sy, inv);
    oz[lo] = __fmul_rn(sz, inv);
    first[lo] = i0;
  }
}

// Sort key of the first-seen order: each voxel's first point index.
struct FirstSeenSrc {
  const uint32_t *first;
  uint32_t bits;  // bits of the largest point index
  __device__ __forceinline__ void prepare(const Control *) {}
  __device__ __forceinline__ uint32_t count(const Control *ctl) const {
    return uint32_t(ctl->n_voxels);
  }
  __device__ __forceinline__ uint32_t key_bits() const { return bits; }
  __device__ __forceinline__ uint64_t key(uint32_t v) const { return first[v]; }
};

// Voxel j of the first-seen order <- voxel val(j) of the key order.
__global__ void k_voxel_first_seen_gather(Control *ctl, SortBuffers sort, const SortState *order,
                                          const float *ix, const float *iy, const float *iz,
                                          const uint32_t *icnt, const uint64_t *ikey, float *ox,
                                          float *oy, float *oz, uint32_t *ocnt, uint64_t *okey) {
  if (ld_relaxed_u32(&ctl->status)) return;
  const uint32_t nv = uint32_t(ctl->n_voxels);
  const SortedView sv = sorted_view(sort, *order);
  for (uint32_t j = blockIdx.x * blockDim.x + threadIdx.x; j < nv; j += gridDim.x * blockDim.x) {
    const uint32_t v = sv.val(j);
    if (v >= nv) {
      atomicOr(&ctl->status, ST_INTERNAL);
      continue;
    }
    ox[j] = ix[v];
    oy[j] = iy[v];
    oz[j] = iz[v];
    ocnt[j] = icnt[v];
    okey[j] = ikey[v];
  }
}

// The gathered voxels back into the chain's voxel buffers (and the AoS copy
// the normals stage reads).
__global__ void k_voxel_copy_back(const Control *ctl, const float *ix, const float *iy,
                                  const float *iz, const uint32_t *icnt, const uint64_t *ikey,
                                  float *ox, float *oy, float *oz, uint32_t *ocnt, uint64_t *okey,
                                  float4 *aos) {
  if (ld_relaxed_u32(&ctl->status)) return;
  const uint32_t nv = uint32_t(ctl->n_voxels);
  for (uint32_t j = blockIdx.x * blockDim.x + threadIdx.x; j < nv; j += gridDim.x * blockDim.x) {
    ox[j] = ix[j];
    oy[j] = iy[j];
    oz[j] = iz[j];
    ocnt[j] = icnt[j];
    okey[j] = ikey[j];
    if (aos) aos[j] = make_float4(ix[j], iy[j], iz[j], 0.0f);
  }
}

// Unpacks packed voxel keys into the reference's (ix, iy, iz) int64 triples.
__global__ void k_unpack_voxel_keys(const Control *ctl, const uint64_t *packed, int64_t *out,
                                    Batch bt) {
  if (ctl->status) return;
  const uint64_t v = ctl->n_voxels;
  const uint32_t lb = ctl->vkey_bits;
  const uint64_t mask = lb >= 64 ? ~0ull : ((1ull << lb) - 1);
  for (uint64_t i = blockIdx.x * uint64_t(blockDim.x) + threadIdx.x; i < v;
       i += uint64_t(gridDim.x) * blockDim.x) {
    const uint64_t key = packed[i];
    const uint32_t b = lb >= 64 ? 0u : uint32_t(key >> lb);
    int64_t k[3];
    voxel_unpack(bt.vplans[b < bt.clouds ? b : 0], key & mask, k);
    out[3 * i] = k[0];
    out[3 * i + 1] = k[1];
    out[3 * i + 2] = k[2];
  }
}

// Voxel range of every cloud in the key-ordered output: voxel_offsets[b] is
// the first voxel whose key carries cloud id >= b (binary search).
__global__ void k_voxel_offsets(const Control *ctl, const uint64_t *packed, Batch bt) {
  if (ctl->status) return;
  const uint32_t b = blockIdx.x * blockDim.x + threadIdx.x;
  if (b > bt.clouds) return;
  const uint64_t v = ctl->n_voxels;
  const uint32_t lb = ctl->vkey_bits;
  uint64_t lo = 0, hi = v;
  if (b == 0) hi = 0;
  else if (b == bt.clouds) lo = v;
  else {
    const uint64_t target = uint64_t(b) << lb;  // lb < 64 whenever there are 2+ clouds
    while (lo < hi) {
      const uint64_t mid = (lo + hi) >> 1;
      if (packed[mid] < target) lo = mid + 1;
      else hi = mid;
    }
  }
  bt.voxel_offsets[b] = uint32_t(lo);
}

}  // namespace srcu
