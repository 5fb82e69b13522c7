// radix.cuh -- onesweep LSD radix sort of keys with their point indices, as
// one persistent cooperative kernel per sort.
//
// Phase 1 computes every key once (kept for the first pass) and histograms
// its digits (shared-memory atomics, which B200 executes at full rate even
// when lanes collide).  Digits are 8 bits wide, or 9 bits in the shapes built
// for them (512 threads) when that takes fewer passes over the key width at
// hand -- 43-bit keys of a batch sort in 5 passes instead of 6.  After a grid
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

#include <type_traits>

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

// Shared memory of one sort block of WARPS warps for tiles of TILE keys and
// digits of up to DBITS bits.  The per-warp digit counters of the 9-bit shapes
// are 16-bit (a tile holds fewer than 2^16 keys), which keeps two blocks of
// 512 threads on an SM.
template <int TILE, int WARPS = OS_WARPS, int DBITS = RADIX_BITS>
struct OnesweepSmemT {
  static constexpr int BINS = 1 << DBITS;
  using WarpCount = typename std::conditional<(DBITS > RADIX_BITS), uint16_t, uint32_t>::type;
  static_assert(TILE < 65536, "16-bit per-warp digit counters");
  union {
    OnesweepTileSmem<TILE> tile;
    uint32_t hist[HIST_COPIES][MAX_DIGITS][BINS];
  } u;
  WarpCount whist[WARPS][BINS];
  uint32_t match[WARPS][BINS];  // per-warp peer masks, zero between uses
  uint32_t digit_start[BINS];
  uint32_t tile_excl[BINS];
  uint32_t gbase[BINS];
  uint32_t scratch[WARPS];
  uint32_t trivial[MAX_DIGITS];
  uint32_t active[MAX_DIGITS];
  uint32_t num_active;
  uint32_t tile;
};
using OnesweepSmem = OnesweepSmemT<OS_TILE>;

// The sort's launch shapes the library is built with: keys per thread, the
// blocks per SM the registers are capped for, threads per block, and the
// widest digit (a thread per digit bin: 256 threads for 8-bit digits, 512
// for 9-bit ones, which run 8-bit passes when 9 bits save none).  The
// autotuner picks among them per input size (srcu_set_sort_tuning).
constexpr int SORT_CONFIGS = 8;
constexpr int kSortItems[SORT_CONFIGS] = {16, 8, 12, 8, 8, 12, 8, 12};
constexpr int kSortMinBlocks[SORT_CONFIGS] = {2, 3, 3, 4, 2, 1, 2, 1};
constexpr int kSortThreads[SORT_CONFIGS] = {256, 256, 256, 256, 512, 512, 512, 512};
constexpr int kSortDigitBits[SORT_CONFIGS] = {8, 8, 8, 8, 8, 8, 9, 9};
constexpr int SORT_MIN_TILE = 2048;  // the smallest tile (keys) the look-back buffer is sized for
// Look-back words per key of a tile of TILE keys with BINS digit bins is
// BINS / TILE; the buffer holds RADIX_BINS / SORT_MIN_TILE per key.
constexpr bool lookback_fits(int tile, int bins) {
  return int64_t(bins) * SORT_MIN_TILE <= int64_t(RADIX_BINS) * tile;
}

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

template <class Src, int ITEMS = OS_ITEMS, int MINB = 2, int THREADS = OS_THREADS,
          int DBITS = RADIX_BITS>
__global__ void __launch_bounds__(THREADS, MINB) k_sort(Src src, Control *ctl, uint32_t *hist,
                                                     SortBuffers buf, uint32_t epoch_off,
                                                     int work_slot, SortState *st) {
  constexpr int WARPS = THREADS / 32;
  constexpr int TILE = THREADS * ITEMS;
  constexpr int WARP_ITEMS = ITEMS * 32;
  constexpr uint32_t BINS = 1u << DBITS;  // digit bins of the widest digit; `hist` stride
  static_assert(THREADS >= int(BINS) && THREADS % 32 == 0, "a thread per digit bin at least");
  static_assert(DBITS >= RADIX_BITS && DBITS <= WIDE_RADIX_BITS, "digit width");
  using Smem = OnesweepSmemT<TILE, WARPS, DBITS>;
  using WarpCount = typename Smem::WarpCount;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  Smem &sm = *reinterpret_cast<Smem *>(smem_raw);
  if (ld_relaxed_u32(&ctl->status)) return;  // before any barrier: every block agrees
  src.prepare(ctl);
  const uint32_t n = src.count(ctl);
  const uint32_t kbits = src.key_bits();
  // The digit width: DBITS where it takes fewer passes over kbits than 8-bit
  // digits, else 8 (every block computes the same).
  const uint32_t nd_narrow = kbits == 0 ? 1u : (kbits + RADIX_BITS - 1) / RADIX_BITS;
  const uint32_t nd_wide = kbits == 0 ? 1u : (kbits + DBITS - 1) / DBITS;
  const uint32_t dbits = nd_wide < nd_narrow ? uint32_t(DBITS) : uint32_t(RADIX_BITS);
  const uint32_t nd = nd_wide < nd_narrow ? nd_wide : nd_narrow;
  const uint32_t dmask = (1u << dbits) - 1u;
  const uint32_t idx_bits = n > 1 ? bit_width_u64(uint64_t(n) - 1) : 0u;
  const bool packed = kbits + idx_bits <= 64;
  const uint32_t shift0 = packed ? idx_bits : 0u;
  const uint32_t t = threadIdx.x, warp = t >> 5, lane = t & 31u;
  const bool owner = t <= dmask;  // this thread owns digit t in the per-digit steps

  // ---- phase 1: digit histograms ----------------------------------------
  for (uint32_t i = t; i < HIST_COPIES * MAX_DIGITS * BINS; i += THREADS)
    (&sm.u.hist[0][0][0])[i] = 0;
  for (uint32_t i = t; i < WARPS * BINS; i += THREADS) (&sm.match[0][0])[i] = 0;
  __syncthreads();
  {
    // The keys are computed once, here, and kept in the ping-pong buffer that
    // the first digit pass reads (keys[1]); the grid barrier below publishes
    // them like any pass's output.
    uint32_t(*h)[BINS] = sm.u.hist[warp & (HIST_COPIES - 1)];
    uint64_t *kcache = buf.keys[1];
    for (uint32_t i = blockIdx.x * THREADS + t; i < n; i += gridDim.x * THREADS) {
      const uint64_t k = src.key(i);
      kcache[i] = k;
      for (uint32_t d = 0; d < nd; ++d) atomicAdd(&h[d][uint32_t(k >> (dbits * d)) & dmask], 1u);
    }
  }
  __syncthreads();
  for (uint32_t i = t; i < nd * BINS; i += THREADS) {
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
      if (ld_relaxed_u32(&hist[d * BINS + t]) == n) sm.trivial[d] = 1;
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
    const uint32_t shift = shift0 + sm.active[p] * dbits;
    {
      uint32_t total;
      const uint32_t ds = block_exclusive_sum<THREADS>(
          owner ? ld_relaxed_u32(&hist[sm.active[p] * BINS + t]) : 0u, sm.scratch, &total);
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
      for (uint32_t i = t; i < WARPS * BINS; i += THREADS) (&sm.whist[0][0])[i] = 0;
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
        const uint32_t d = uint32_t(k[i] >> shift) & dmask;
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
            sm.whist[warp][d] = WarpCount(prev + uint32_t(__popc(peers)));
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
      uint64_t *lb_mine = buf.lookback + size_t(tile) * BINS + t;
      if (owner) {
#pragma unroll
        for (int w = 0; w < WARPS; ++w) {
          const uint32_t c = sm.whist[w][t];
          sm.whist[w][t] = WarpCount(cnt);
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
          const uint32_t d = uint32_t(k[i] >> shift) & dmask;
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
            w[q] = (j - q >= 0) ? ld_relaxed(buf.lookback + size_t(j - q) * BINS + t)
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
        const uint32_t pos = sm.gbase[uint32_t(kk >> shift) & dmask] + j;
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
