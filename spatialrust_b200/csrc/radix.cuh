// radix.cuh -- onesweep LSD radix sort of keys with their point indices, as
// one persistent cooperative kernel per sort.
//
// Phase 1 computes every key once (kept for the first pass) and histograms
// its 8-bit digits (shared-memory atomics, which B200 executes at full rate
// even when lanes collide).  After a grid
// barrier, each digit pass that is not trivial (some key differs in that
// digit) ranks 4096-key tiles with a warp-level multi-split, resolves the
// tile's global digit offsets by decoupled look-back over earlier tiles, and
// scatters through shared memory so global writes are coalesced runs
// (Adinets & Merrill, "Onesweep", 2022); a grid barrier separates passes.
// Only the passes that are needed run, and the host never learns how many.
//
// Items are packed as (key << index_bits) | index in one u64 when the key and
// point-index bits fit in 64 (8 bytes per item per pass), otherwise kept as a
// u64 key and a separate u32 index (12 bytes).
//
// The sort is stable: within a tile items are ranked in input order, and
// tiles are ordered by index.  Because the first pass reads indices 0..n-1
// in order, equal keys keep ascending point index -- the order in which the
// reference accumulates a voxel's points (voxel.rs:502-520).
//
// Tiles are claimed through an atomic counter, so look-back only waits on
// tiles that are already running, and the cooperative launch keeps every
// block resident for the barriers; every wait is bounded.
#pragma once

#include "plans.cuh"

namespace srcu {

constexpr int OS_THREADS = 256;
constexpr int OS_WARPS = OS_THREADS / 32;
constexpr int OS_ITEMS = 16;
constexpr int OS_WARP_ITEMS = OS_ITEMS * 32;
constexpr int OS_TILE = OS_THREADS * OS_ITEMS;  // 4096 keys per tile
constexpr int HIST_COPIES = 2;                  // shared histogram copies (by warp parity)
constexpr int LB_WIDTH = 8;                     // look-back words read per step

template <int TILE>
struct OnesweepTileSmem {
  uint64_t keys[TILE];
  uint32_t vals[TILE];
};

// Shared memory of one sort block of WARPS warps for tiles of TILE keys.
template <int TILE, int WARPS = OS_WARPS>
struct OnesweepSmemT {
  union {
    OnesweepTileSmem<TILE> tile;
    uint32_t hist[HIST_COPIES][MAX_DIGITS][RADIX_BINS];
  } u;
  uint32_t whist[WARPS][RADIX_BINS];
  uint32_t match[WARPS][RADIX_BINS];  // per-warp peer masks, zero between uses
  uint32_t digit_start[RADIX_BINS];
  uint32_t tile_excl[RADIX_BINS];
  uint32_t gbase[RADIX_BINS];
  uint32_t scratch[WARPS];
  uint32_t trivial[MAX_DIGITS];
  uint32_t active[MAX_DIGITS];
  uint32_t num_active;
  uint32_t tile;
};
using OnesweepSmem = OnesweepSmemT<OS_TILE>;

// The sort's launch shapes the library is built with: keys per thread, the
// blocks per SM the registers are capped for, and threads per block (8-bit
// digits throughout: the first 256 threads of a block own one digit each).
// The autotuner picks among them per input size (srcu_set_sort_tuning).
constexpr int SORT_CONFIGS = 6;
constexpr int kSortItems[SORT_CONFIGS] = {16, 8, 12, 8, 8, 12};
constexpr int kSortMinBlocks[SORT_CONFIGS] = {2, 3, 3, 4, 2, 1};
constexpr int kSortThreads[SORT_CONFIGS] = {256, 256, 256, 256, 512, 512};
constexpr int SORT_MIN_TILE = 2048;  // the smallest tile (keys) the look-back buffer is sized for

// Ping-pong buffers of one sort.
struct SortBuffers {
  uint64_t *keys[2];
  uint32_t *vals[2];
  uint64_t *lookback;  // >= num_tiles * 256 words, zeroed once at allocation
};

// Read access to a finished sort.
struct SortedView {
  const uint64_t *keys;
  const uint32_t *vals;
  uint32_t packed;
  uint32_t idx_bits;
  __device__ __forceinline__ uint64_t key(uint32_t i) const {
    return packed ? (keys[i] >> idx_bits) : keys[i];
  }
  __device__ __forceinline__ uint32_t val(uint32_t i) const {
    return packed ? uint32_t(keys[i] & ((1ull << idx_bits) - 1)) : vals[i];
  }
  // key and value of item i with one load of a packed item
  __device__ __forceinline__ void get(uint32_t i, uint64_t &k, uint32_t &v) const {
    const uint64_t w = keys[i];
    if (packed) {
      k = w >> idx_bits;
      v = uint32_t(w & ((1ull << idx_bits) - 1));
    } else {
      k = w;
      v = vals[i];
    }
  }
};

__device__ __forceinline__ SortedView sorted_view(const SortBuffers &b, const SortState &s) {
  SortedView v;
  v.keys = b.keys[s.final_buf];
  v.vals = b.vals[s.final_buf];
  v.packed = s.packed;
  v.idx_bits = s.idx_bits;
  return v;
}

// Grid-wide barrier for a cooperative launch.  Bounded: a waiter that gives
// up sets ST_TIMEOUT and continues.
__device__ __forceinline__ void grid_barrier(SortState *st, uint32_t *status) {
  __syncthreads();
  if (threadIdx.x == 0) {
    const uint32_t gen = ld_relaxed_u32(&st->bar_gen);
    __threadfence();
    const uint32_t arrived = atomicAdd(&st->bar_count, 1u) + 1u;
    if (arrived == gridDim.x) {
      atomicExch(&st->bar_count, 0u);
      __threadfence();
      atomicAdd(&st->bar_gen, 1u);
    } else {
      uint32_t spins = 0;
      while (ld_relaxed_u32(&st->bar_gen) == gen) {
        if (++spins > SPIN_LIMIT) {
          atomicOr(status, ST_TIMEOUT);
          break;
        }
        __nanosleep(64);
      }
    }
    __threadfence();
  }
  __syncthreads();
}

template <class Src, int ITEMS = OS_ITEMS, int MINB = 2, int THREADS = OS_THREADS>
__global__ void __launch_bounds__(THREADS, MINB) k_sort(Src src, Control *ctl, uint32_t *hist,
                                                     SortBuffers buf, uint32_t epoch_off,
                                                     int work_slot, SortState *st) {
  static_assert(THREADS >= RADIX_BINS && THREADS % 32 == 0, "a thread per digit at least");
  constexpr int WARPS = THREADS / 32;
  constexpr int TILE = THREADS * ITEMS;
  constexpr int WARP_ITEMS = ITEMS * 32;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  OnesweepSmemT<TILE, WARPS> &sm = *reinterpret_cast<OnesweepSmemT<TILE, WARPS> *>(smem_raw);
  if (ld_relaxed_u32(&ctl->status)) return;  // before any barrier: every block agrees
  src.prepare(ctl);
  const uint32_t n = src.count(ctl);
  const uint32_t kbits = src.key_bits();
  const uint32_t nd = kbits == 0 ? 1u : (kbits + RADIX_BITS - 1) / RADIX_BITS;
  const uint32_t idx_bits = n > 1 ? bit_width_u64(uint64_t(n) - 1) : 0u;
  const bool packed = kbits + idx_bits <= 64;
  const uint32_t shift0 = packed ? idx_bits : 0u;
  const uint32_t t = threadIdx.x, warp = t >> 5, lane = t & 31u;
  const bool owner = t < RADIX_BINS;  // this thread owns digit t in the per-digit steps

  // ---- phase 1: digit histograms ----------------------------------------
  for (uint32_t i = t; i < HIST_COPIES * MAX_DIGITS * RADIX_BINS; i += THREADS)
    (&sm.u.hist[0][0][0])[i] = 0;
  for (uint32_t i = t; i < WARPS * RADIX_BINS; i += THREADS) (&sm.match[0][0])[i] = 0;
  __syncthreads();
  {
    // The keys are computed once, here, and kept in the ping-pong buffer that
    // the first digit pass reads (keys[1]); the grid barrier below publishes
    // them like any pass's output.
    uint32_t(*h)[RADIX_BINS] = sm.u.hist[warp & (HIST_COPIES - 1)];
    uint64_t *kcache = buf.keys[1];
    for (uint32_t i = blockIdx.x * THREADS + t; i < n; i += gridDim.x * THREADS) {
      const uint64_t k = src.key(i);
      kcache[i] = k;
      for (uint32_t d = 0; d < nd; ++d) atomicAdd(&h[d][uint32_t(k >> (RADIX_BITS * d)) & 0xffu], 1u);
    }
  }
  __syncthreads();
  for (uint32_t i = t; i < nd * RADIX_BINS; i += THREADS) {
    uint32_t c = 0;
#pragma unroll
    for (int cp = 0; cp < HIST_COPIES; ++cp) c += (&sm.u.hist[cp][0][0])[i];
    if (c) atomicAdd(&hist[i], c);
  }
  __threadfence();  // the cached keys, before the barrier releases the first pass
  grid_barrier(st, &ctl->status);

  // ---- which digits need a pass ----------------------------------------
  if (t < MAX_DIGITS) sm.trivial[t] = 0;
  __syncthreads();
  if (owner)
    for (uint32_t d = 0; d < nd; ++d)
      if (ld_relaxed_u32(&hist[d * RADIX_BINS + t]) == n) sm.trivial[d] = 1;
  __syncthreads();
  if (t == 0) {
    uint32_t na = 0;
    for (uint32_t d = 0; d < nd; ++d)
      if (!sm.trivial[d]) sm.active[na++] = d;
    if (na == 0) sm.active[na++] = 0;  // one pass always materialises the items
    sm.num_active = na;
    if (blockIdx.x == 0) {
      st->final_buf = (na - 1) & 1u;
      st->passes = na;
      st->packed = packed ? 1u : 0u;
      st->idx_bits = idx_bits;
      st->key_bits = kbits;
    }
  }
  __syncthreads();
  const uint32_t num_active = sm.num_active;
  const uint32_t num_tiles = (n + TILE - 1) / TILE;
  const uint64_t idx_mask = (1ull << idx_bits) - 1;

  // ---- digit passes ------------------------------------------------------
  for (uint32_t p = 0; p < num_active; ++p) {
    const uint32_t shift = shift0 + sm.active[p] * RADIX_BITS;
    {
      uint32_t total;
      const uint32_t ds = block_exclusive_sum<THREADS>(
          owner ? ld_relaxed_u32(&hist[sm.active[p] * RADIX_BINS + t]) : 0u, sm.scratch, &total);
      if (owner) sm.digit_start[t] = ds;
    }
    const bool from_src = p == 0;
    const uint64_t *kin = buf.keys[(p + 1) & 1];
    const uint32_t *vin = buf.vals[(p + 1) & 1];
    uint64_t *kout = buf.keys[p & 1];
    uint32_t *vout = buf.vals[p & 1];
    const uint32_t epoch = ctl->epoch + epoch_off + p;
    uint32_t *ctr = &ctl->work[work_slot + p];

    for (;;) {
      if (t == 0) sm.tile = atomicAdd(ctr, 1u);
      for (uint32_t i = t; i < WARPS * RADIX_BINS; i += THREADS) (&sm.whist[0][0])[i] = 0;
      __syncthreads();
      const uint32_t tile = sm.tile;
      if (tile >= num_tiles) break;
      const uint32_t base = tile * TILE;
      const uint32_t wbase = base + warp * WARP_ITEMS;

      uint64_t k[ITEMS];
      uint32_t v[ITEMS];
      uint32_t rank[ITEMS];
#pragma unroll
      for (int i = 0; i < ITEMS; ++i) {
        const uint32_t idx = wbase + uint32_t(i) * 32u + lane;
        k[i] = 0;
        v[i] = 0;
        if (idx < n) {
          if (from_src) {  // the key stored by the histogram phase
            const uint64_t key = kin[idx];
            k[i] = packed ? ((key << idx_bits) | idx) : key;
            v[i] = idx;
          } else {
            k[i] = kin[idx];
            if (!packed) v[i] = vin[idx];
          }
        }
      }
      // Warp-private multi-split: rank each item among earlier items of the
      // warp with the same digit.  The lanes sharing a digit (its peers) come
      // from one shared-memory atomicOr per lane into the warp's mask for that
      // digit, or, when every valid lane holds the same digit (the high digits
      // of spatially coherent keys), from the valid mask alone.  One leader per
      // digit per step updates the warp's counter and clears the mask.
#pragma unroll
      for (int i = 0; i < ITEMS; ++i) {
        const bool valid = (wbase + uint32_t(i) * 32u + lane) < n;
        const uint32_t d = uint32_t(k[i] >> shift) & 0xffu;
        const uint32_t vmask = __ballot_sync(FULL_MASK, valid);
        const uint32_t d0 = __shfl_sync(FULL_MASK, d, 0);
        const bool uniform = __all_sync(FULL_MASK, !valid || d == d0);
        uint32_t peers = vmask;
        if (!uniform) {  // peers from shared-memory masks: one atomic per lane
          if (valid) atomicOr(&sm.match[warp][d], 1u << lane);
          __syncwarp();
          peers = valid ? sm.match[warp][d] : 0u;
          __syncwarp();
        }
        uint32_t prev = 0;
        uint32_t leader = 0;
        if (valid) {
          leader = 31u - __clz(peers);
          if (lane == leader) {
            prev = sm.whist[warp][d];
            sm.whist[warp][d] = prev + uint32_t(__popc(peers));
            if (!uniform) sm.match[warp][d] = 0u;
          }
        }
        prev = __shfl_sync(FULL_MASK, prev, leader);
        rank[i] = prev + uint32_t(__popc(peers & lanemask_lt()));
        __syncwarp();
      }
      __syncthreads();
      // Thread t owns digit t: exclusive prefix over warps, tile count.
      uint32_t cnt = 0;
      uint64_t *lb_mine = buf.lookback + size_t(tile) * RADIX_BINS + t;
      if (owner) {
#pragma unroll
        for (int w = 0; w < WARPS; ++w) {
          const uint32_t c = sm.whist[w][t];
          sm.whist[w][t] = cnt;
          cnt += c;
        }
        // Publish the tile aggregate as early as possible.
        st_relaxed(lb_mine, lb_pack(epoch, tile == 0 ? LB_INC : LB_AGG, cnt));
      }
      uint32_t tile_total;
      const uint32_t texcl = block_exclusive_sum<THREADS>(cnt, sm.scratch, &tile_total);
      if (owner) sm.tile_excl[t] = texcl;
      __syncthreads();
      // Scatter to shared memory in digit order.
#pragma unroll
      for (int i = 0; i < ITEMS; ++i) {
        if ((wbase + uint32_t(i) * 32u + lane) < n) {
          const uint32_t d = uint32_t(k[i] >> shift) & 0xffu;
          const uint32_t pos = sm.tile_excl[d] + sm.whist[warp][d] + rank[i];
          sm.u.tile.keys[pos] = k[i];
          if (!packed) sm.u.tile.vals[pos] = v[i];
        }
      }
      // Resolve the look-back for digit t, LB_WIDTH predecessors per step
      // (independent loads, one latency), stopping at the first inclusive.
      uint32_t excl = 0;
      if (owner && tile > 0) {
        int64_t j = int64_t(tile) - 1;
        uint32_t spins = 0;
        bool done = false;
        while (!done && j >= 0) {
          uint64_t w[LB_WIDTH];
#pragma unroll
          for (int q = 0; q < LB_WIDTH; ++q)
            w[q] = (j - q >= 0) ? ld_relaxed(buf.lookback + size_t(j - q) * RADIX_BINS + t)
                                : lb_pack(epoch, LB_INC, 0);
          uint32_t consumed = 0;
#pragma unroll
          for (int q = 0; q < LB_WIDTH; ++q) {
            if (done || consumed != uint32_t(q)) break;
            const uint64_t flag = w[q] & (3ull << 30);
            if (uint32_t(w[q] >> 32) != epoch || flag == 0) break;
            excl += uint32_t(w[q]) & LB_COUNT_MASK;
            ++consumed;
            if (flag == LB_INC) done = true;
          }
          j -= consumed;
          if (!done && consumed == 0) {
            if (++spins > SPIN_LIMIT) {
              atomicOr(&ctl->status, ST_TIMEOUT);
              break;
            }
            __nanosleep(20);
          }
        }
        st_relaxed(lb_mine, lb_pack(epoch, LB_INC, excl + cnt));
      }
      if (owner) sm.gbase[t] = sm.digit_start[t] + excl - texcl;
      __syncthreads();
      const uint32_t tile_n = min(uint32_t(TILE), n - base);
      for (uint32_t j = t; j < tile_n; j += THREADS) {
        const uint64_t kk = sm.u.tile.keys[j];
        const uint32_t pos = sm.gbase[uint32_t(kk >> shift) & 0xffu] + j;
        if (pos < n) {
          kout[pos] = kk;
          if (!packed) vout[pos] = sm.u.tile.vals[j];
        } else {
          atomicOr(&ctl->status, ST_INTERNAL);
        }
      }
      __syncthreads();
    }
    if (p + 1 < num_active) grid_barrier(st, &ctl->status);
  }
  (void)idx_mask;
}

}  // namespace srcu
