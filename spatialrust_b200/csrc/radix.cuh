// radix.cuh -- onesweep LSD radix sort of (u64 key, u32 index) pairs.
//
// One up-front kernel histograms every 8-bit digit of every key
// (k_digit_hist); each digit pass (k_onesweep) then ranks a 4096-key tile
// with warp-level multi-split (__match_any_sync), resolves the tile's global
// digit offsets by decoupled look-back over earlier tiles, and scatters
// through shared memory so global writes are coalesced runs (Adinets &
// Merrill, "Onesweep", 2022).  Passes whose digit is identical for every key
// are skipped on the device, so the host always launches MAX_DIGITS passes
// and never synchronises to learn how many bits the keys use.  Tiles are
// claimed through an atomic counter, so look-back only ever waits on tiles
// that are already running; every wait is bounded.
//
// The sort is stable: within a tile items are ranked in input order, and
// tiles are ordered by index.  Because the first pass reads indices 0..n-1
// in order, equal keys keep ascending point index -- the order in which the
// reference accumulates a voxel's points (voxel.rs:502-520).
#pragma once

#include "plans.cuh"

namespace srcu {

constexpr int OS_THREADS = 256;
constexpr int OS_WARPS = OS_THREADS / 32;
constexpr int OS_ITEMS = 16;
constexpr int OS_WARP_ITEMS = OS_ITEMS * 32;
constexpr int OS_TILE = OS_THREADS * OS_ITEMS;  // 4096 keys per tile
constexpr int HIST_THREADS = 256;

struct OnesweepSmem {
  uint64_t keys[OS_TILE];
  uint32_t vals[OS_TILE];
  uint32_t whist[OS_WARPS][RADIX_BINS];
  uint32_t digit_start[RADIX_BINS];
  uint32_t tile_excl[RADIX_BINS];
  uint32_t gbase[RADIX_BINS];
  uint32_t scratch[OS_WARPS];
  uint32_t trivial[MAX_DIGITS];
  uint32_t active[MAX_DIGITS];
  uint32_t num_active;
  uint32_t tile;
};

// Ping-pong buffers of one sort.
struct SortBuffers {
  uint64_t *keys[2];
  uint32_t *vals[2];
  uint64_t *lookback;  // >= num_tiles * 256 words, zeroed once at allocation
};

// Number of non-trivial digits and their list, from the digit histograms.
// At least one pass always runs so the (key, index) pairs are materialised.
__device__ __forceinline__ void onesweep_active_digits(const uint32_t *hist, uint32_t n,
                                                       uint32_t nd, OnesweepSmem &sm) {
  const uint32_t t = threadIdx.x;
  if (t < MAX_DIGITS) sm.trivial[t] = 0;
  __syncthreads();
  for (uint32_t d = 0; d < nd; ++d)
    if (hist[d * RADIX_BINS + t] == n) sm.trivial[d] = 1;
  __syncthreads();
  if (t == 0) {
    uint32_t na = 0;
    for (uint32_t d = 0; d < nd; ++d)
      if (!sm.trivial[d]) sm.active[na++] = d;
    if (na == 0) sm.active[na++] = 0;
    sm.num_active = na;
  }
  __syncthreads();
}

// Histograms all digits of all keys.  hist: MAX_DIGITS x 256, zeroed by k_begin.
template <class Src>
__global__ void __launch_bounds__(HIST_THREADS) k_digit_hist(Src src, Control *ctl, uint32_t *hist) {
  __shared__ uint32_t sh[MAX_DIGITS][RADIX_BINS];
  if (ld_relaxed_u32(&ctl->status)) return;
  src.prepare(ctl);
  const uint32_t n = src.count(ctl);
  const uint32_t nd = src.num_digits();
  for (uint32_t i = threadIdx.x; i < MAX_DIGITS * RADIX_BINS; i += HIST_THREADS)
    (&sh[0][0])[i] = 0;
  __syncthreads();
  const uint32_t lane = threadIdx.x & 31u;
  const uint32_t stride = gridDim.x * HIST_THREADS;
  for (uint32_t base = blockIdx.x * HIST_THREADS + (threadIdx.x & ~31u); base < n; base += stride) {
    const uint32_t i = base + lane;
    const bool valid = i < n;
    uint64_t k = 0;
    uint32_t v = 0;
    if (valid) src.load(i, k, v);
    for (uint32_t d = 0; d < nd; ++d) {
      const uint32_t b = valid ? (uint32_t(k >> (RADIX_BITS * d)) & 0xffu) : 0x100u;
      const uint32_t peers = __match_any_sync(FULL_MASK, b);
      if (valid && lane == uint32_t(__ffs(peers) - 1)) atomicAdd(&sh[d][b], uint32_t(__popc(peers)));
    }
  }
  __syncthreads();
  for (uint32_t i = threadIdx.x; i < nd * RADIX_BINS; i += HIST_THREADS) {
    const uint32_t c = (&sh[0][0])[i];
    if (c) atomicAdd(&hist[i], c);
  }
}

// One onesweep digit pass.  Launch `launch` (0..MAX_DIGITS-1) processes the
// launch-th non-trivial digit; launch 0 reads keys from `src`, later launches
// from buffer (launch-1)&1; output goes to buffer launch&1.  Launch 0 stores
// the index of the buffer holding the final result in final_buf[0] and the
// number of passes that run in final_buf[2] (Control::{v,c}sort_final/_passes).
template <class Src>
__global__ void __launch_bounds__(OS_THREADS, 2) k_onesweep(Src src, Control *ctl, const uint32_t *hist,
                                                         SortBuffers buf, int launch,
                                                         uint32_t epoch_off, int work_slot,
                                                         uint32_t *final_buf) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  OnesweepSmem &sm = *reinterpret_cast<OnesweepSmem *>(smem_raw);
  if (ld_relaxed_u32(&ctl->status)) return;
  src.prepare(ctl);
  const uint32_t n = src.count(ctl);
  const uint32_t nd = src.num_digits();
  const uint32_t t = threadIdx.x;
  onesweep_active_digits(hist, n, nd, sm);
  if (launch == 0 && blockIdx.x == 0 && t == 0) {
    final_buf[0] = (sm.num_active - 1) & 1u;
    final_buf[2] = sm.num_active;  // the passes counter sits two words after the buffer index
  }
  if (uint32_t(launch) >= sm.num_active) return;
  const uint32_t digit = sm.active[launch];
  const uint32_t shift = digit * RADIX_BITS;
  {
    uint32_t total;
    sm.digit_start[t] = block_exclusive_sum<OS_THREADS>(hist[digit * RADIX_BINS + t], sm.scratch, &total);
  }
  const bool from_src = launch == 0;
  const uint64_t *kin = buf.keys[(launch + 1) & 1];
  const uint32_t *vin = buf.vals[(launch + 1) & 1];
  uint64_t *kout = buf.keys[launch & 1];
  uint32_t *vout = buf.vals[launch & 1];
  const uint32_t epoch = ctl->epoch + epoch_off + uint32_t(launch);
  const uint32_t num_tiles = (n + OS_TILE - 1) / OS_TILE;
  uint32_t *ctr = &ctl->work[work_slot + launch];
  const uint32_t warp = t >> 5, lane = t & 31u;

  for (;;) {
    if (t == 0) sm.tile = atomicAdd(ctr, 1u);
    for (uint32_t i = t; i < OS_WARPS * RADIX_BINS; i += OS_THREADS) (&sm.whist[0][0])[i] = 0;
    __syncthreads();
    const uint32_t tile = sm.tile;
    if (tile >= num_tiles) break;
    const uint32_t base = tile * OS_TILE;
    const uint32_t wbase = base + warp * OS_WARP_ITEMS;

    uint64_t k[OS_ITEMS];
    uint32_t v[OS_ITEMS];
    uint32_t rank[OS_ITEMS];
#pragma unroll
    for (int i = 0; i < OS_ITEMS; ++i) {
      const uint32_t idx = wbase + uint32_t(i) * 32u + lane;
      k[i] = ~0ull;
      v[i] = 0;
      if (idx < n) {
        if (from_src) {
          src.load(idx, k[i], v[i]);
        } else {
          k[i] = kin[idx];
          v[i] = vin[idx];
        }
      }
    }
    // Warp-private multi-split: rank each key among earlier keys of the warp
    // with the same digit.  Exactly one leader per digit per step updates the
    // warp's counter, so no atomics are needed.
#pragma unroll
    for (int i = 0; i < OS_ITEMS; ++i) {
      const bool valid = (wbase + uint32_t(i) * 32u + lane) < n;
      const uint32_t d = valid ? (uint32_t(k[i] >> shift) & 0xffu) : 0x100u;
      const uint32_t peers = __match_any_sync(FULL_MASK, d);
      const uint32_t leader = 31u - __clz(peers);
      uint32_t prev = 0;
      if (valid && lane == leader) {
        prev = sm.whist[warp][d];
        sm.whist[warp][d] = prev + uint32_t(__popc(peers));
      }
      prev = __shfl_sync(FULL_MASK, prev, leader);
      rank[i] = prev + uint32_t(__popc(peers & lanemask_lt()));
      __syncwarp();
    }
    __syncthreads();
    // Thread t owns digit t: exclusive prefix over warps, tile count.
    uint32_t cnt = 0;
#pragma unroll
    for (int w = 0; w < OS_WARPS; ++w) {
      const uint32_t c = sm.whist[w][t];
      sm.whist[w][t] = cnt;
      cnt += c;
    }
    // Publish the tile aggregate as early as possible.
    uint64_t *lb_mine = buf.lookback + size_t(tile) * RADIX_BINS + t;
    st_relaxed(lb_mine, lb_pack(epoch, tile == 0 ? LB_INC : LB_AGG, cnt));
    uint32_t tile_total;
    const uint32_t texcl = block_exclusive_sum<OS_THREADS>(cnt, sm.scratch, &tile_total);
    sm.tile_excl[t] = texcl;
    __syncthreads();
    // Scatter to shared memory in digit order.
#pragma unroll
    for (int i = 0; i < OS_ITEMS; ++i) {
      const bool valid = (wbase + uint32_t(i) * 32u + lane) < n;
      if (valid) {
        const uint32_t d = uint32_t(k[i] >> shift) & 0xffu;
        const uint32_t pos = sm.tile_excl[d] + sm.whist[warp][d] + rank[i];
        sm.keys[pos] = k[i];
        sm.vals[pos] = v[i];
      }
    }
    // Resolve the look-back for digit t.
    uint32_t excl = 0;
    if (tile > 0) {
      int64_t j = int64_t(tile) - 1;
      uint32_t spins = 0;
      while (j >= 0) {
        const uint64_t w = ld_relaxed(buf.lookback + size_t(j) * RADIX_BINS + t);
        const uint64_t flag = w & (3ull << 30);
        if (uint32_t(w >> 32) == epoch && flag != 0) {
          excl += uint32_t(w) & LB_COUNT_MASK;
          if (flag == LB_INC) break;
          --j;
        } else {
          if (++spins > SPIN_LIMIT) {
            atomicOr(&ctl->status, ST_TIMEOUT);
            break;
          }
          __nanosleep(20);
        }
      }
      st_relaxed(lb_mine, lb_pack(epoch, LB_INC, excl + cnt));
    }
    sm.gbase[t] = sm.digit_start[t] + excl - texcl;
    __syncthreads();
    const uint32_t tile_n = min(uint32_t(OS_TILE), n - base);
    for (uint32_t j = t; j < tile_n; j += OS_THREADS) {
      const uint64_t kk = sm.keys[j];
      const uint32_t pos = sm.gbase[uint32_t(kk >> shift) & 0xffu] + j;
      if (pos < n) {
        kout[pos] = kk;
        vout[pos] = sm.vals[j];
      } else {
        atomicOr(&ctl->status, ST_INTERNAL);
      }
    }
    __syncthreads();
  }
}

}  // namespace srcu
