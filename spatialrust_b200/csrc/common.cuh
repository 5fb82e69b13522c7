// common.cuh -- shared device helpers for the sm_100a uniform-grid path.
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

namespace srcu {

constexpr uint32_t FULL_MASK = 0xffffffffu;

// Device status word bits (Control::status).  Any non-zero value makes the
// remaining kernels of a chain return immediately; the host maps the bits to
// an srcu_status after synchronising.
enum StatusBits : uint32_t {
  ST_TIMEOUT = 1u << 0,        // a bounded look-back / barrier / mbarrier wait gave up
  ST_KEY_OVERFLOW = 1u << 1,   // packed voxel key needs more than 64 bits
  ST_HASH_FULL = 1u << 2,      // cell hash probe sequence exhausted (cannot happen at load <= 1/2)
  ST_TOO_MANY_POINTS = 1u << 3,// more points than a 30-bit look-back count can hold
  ST_BAD_PARAMS = 1u << 4,     // NaN or negative radius reached the device
  ST_INTERNAL = 1u << 5,       // an output index failed its bounds check (write skipped)
};

// Upper bound on polls of any spin-wait.  With __nanosleep backoff this is
// well under a second; afterwards the waiter sets ST_TIMEOUT and moves on.
constexpr uint32_t SPIN_LIMIT = 1u << 21;

__device__ __forceinline__ uint32_t lane_id() {
  uint32_t l;
  asm("mov.u32 %0, %%laneid;" : "=r"(l));
  return l;
}

__device__ __forceinline__ uint32_t lanemask_lt() {
  uint32_t m;
  asm("mov.u32 %0, %%lanemask_lt;" : "=r"(m));
  return m;
}

// Order-preserving float <-> uint encoding for atomicMin/atomicMax.
__device__ __forceinline__ uint32_t f2ord(float f) {
  uint32_t u = __float_as_uint(f);
  return (u & 0x80000000u) ? ~u : (u | 0x80000000u);
}
__host__ __device__ __forceinline__ float ord2f(uint32_t u) {
  uint32_t b = (u & 0x80000000u) ? (u & 0x7fffffffu) : ~u;
#ifdef __CUDA_ARCH__
  return __uint_as_float(b);
#else
  float f;
  __builtin_memcpy(&f, &b, 4);
  return f;
#endif
}

__device__ __forceinline__ uint64_t ld_relaxed(const uint64_t *p) {
  uint64_t v;
  asm volatile("ld.relaxed.gpu.global.u64 %0, [%1];" : "=l"(v) : "l"(p) : "memory");
  return v;
}
__device__ __forceinline__ void st_relaxed(uint64_t *p, uint64_t v) {
  asm volatile("st.relaxed.gpu.global.u64 [%0], %1;" ::"l"(p), "l"(v) : "memory");
}
__device__ __forceinline__ uint32_t ld_relaxed_u32(const uint32_t *p) {
  uint32_t v;
  asm volatile("ld.relaxed.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
  return v;
}
__device__ __forceinline__ void st_relaxed_u32(uint32_t *p, uint32_t v) {
  asm volatile("st.relaxed.gpu.global.u32 [%0], %1;" ::"l"(p), "r"(v) : "memory");
}

// Decoupled look-back words: [epoch:32][flag:2][count:30].  The epoch makes
// words left over from earlier launches read as "not yet published", so the
// arrays are zeroed once at allocation and never again.
constexpr uint64_t LB_AGG = 1ull << 30;
constexpr uint64_t LB_INC = 2ull << 30;
constexpr uint32_t LB_COUNT_MASK = (1u << 30) - 1;
constexpr uint64_t LB_MAX_COUNT = (1ull << 30) - 1;

__device__ __forceinline__ uint64_t lb_pack(uint32_t epoch, uint64_t flag, uint32_t count) {
  return (uint64_t(epoch) << 32) | flag | uint64_t(count & LB_COUNT_MASK);
}

// Exclusive prefix of `value` over all tiles before `tile` (decoupled
// look-back, Merrill & Garland 2016).  Publishes this tile's aggregate
// first, then its inclusive prefix.  Bounded: on timeout sets ST_TIMEOUT
// in *status and returns what it has.
__device__ __forceinline__ uint32_t lookback_exclusive(uint64_t *words, size_t stride, uint32_t tile,
                                                       uint32_t value, uint32_t epoch,
                                                       uint32_t *status) {
  uint64_t *mine = words + size_t(tile) * stride;
  if (tile == 0) {
    st_relaxed(mine, lb_pack(epoch, LB_INC, value));
    return 0;
  }
  st_relaxed(mine, lb_pack(epoch, LB_AGG, value));
  uint32_t excl = 0;
  int64_t j = int64_t(tile) - 1;
  uint32_t spins = 0;
  while (j >= 0) {
    uint64_t w = ld_relaxed(words + size_t(j) * stride);
    uint32_t e = uint32_t(w >> 32);
    uint64_t flag = w & (3ull << 30);
    if (e == epoch && flag != 0) {
      excl += uint32_t(w) & LB_COUNT_MASK;
      if (flag == LB_INC) break;
      --j;
    } else {
      if (++spins > SPIN_LIMIT) {
        atomicOr(status, ST_TIMEOUT);
        break;
      }
      __nanosleep(32);
    }
  }
  st_relaxed(mine, lb_pack(epoch, LB_INC, excl + value));
  return excl;
}

// Warp-cooperative decoupled look-back for one counter per tile: the whole
// warp calls it with the same arguments; lane l inspects tile (j - l), so one
// step covers 32 predecessors and the walk is 32x shorter than a one-word
// walk.  Returns the exclusive prefix in every lane.  Bounded.
__device__ __forceinline__ uint32_t lookback_exclusive_warp(uint64_t *words, uint32_t tile,
                                                            uint32_t value, uint32_t epoch,
                                                            uint32_t *status) {
  const uint32_t lane = threadIdx.x & 31u;
  uint64_t *mine = words + tile;
  if (tile == 0) {
    if (lane == 0) st_relaxed(mine, lb_pack(epoch, LB_INC, value));
    return 0;
  }
  if (lane == 0) st_relaxed(mine, lb_pack(epoch, LB_AGG, value));
  uint32_t excl = 0;
  int64_t j = int64_t(tile) - 1;
  uint32_t spins = 0;
  while (j >= 0) {
    const int64_t idx = j - int64_t(lane);
    uint64_t w = lb_pack(epoch, LB_INC, 0);  // before tile 0: an inclusive zero
    if (idx >= 0) w = ld_relaxed(words + idx);
    const uint64_t flag = w & (3ull << 30);
    const bool ready = uint32_t(w >> 32) == epoch && flag != 0;
    const uint32_t not_ready = __ballot_sync(FULL_MASK, !ready);
    const uint32_t inc = __ballot_sync(FULL_MASK, ready && flag == LB_INC);
    // lanes [0, first not-ready) are usable; stop at the first inclusive among them
    const uint32_t usable = not_ready ? (1u << (__ffs(not_ready) - 1)) - 1u : FULL_MASK;
    const uint32_t inc_usable = inc & usable;
    uint32_t take;  // lanes whose counts are added this step
    if (inc_usable) {
      const uint32_t first_inc = __ffs(inc_usable) - 1;
      take = first_inc == 31 ? FULL_MASK : ((1u << (first_inc + 1)) - 1u);
    } else {
      take = usable;
    }
    uint32_t c = ((take >> lane) & 1u) ? (uint32_t(w) & LB_COUNT_MASK) : 0u;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) c += __shfl_xor_sync(FULL_MASK, c, o);
    excl += c;
    if (inc_usable) break;
    const uint32_t consumed = __popc(take);
    j -= consumed;
    if (consumed == 0) {
      if (++spins > SPIN_LIMIT) {
        if (lane == 0) atomicOr(status, ST_TIMEOUT);
        break;
      }
      __nanosleep(32);
    }
  }
  if (lane == 0) st_relaxed(mine, lb_pack(epoch, LB_INC, excl + value));
  return excl;
}

// Block-wide exclusive sum over 256 threads (8 warps).  `scratch` holds >= 8
// words of shared memory.  Returns the exclusive prefix; *total = block sum.
template <int THREADS>
__device__ __forceinline__ uint32_t block_exclusive_sum(uint32_t v, uint32_t *scratch,
                                                        uint32_t *total) {
  constexpr int WARPS = THREADS / 32;
  const uint32_t lane = threadIdx.x & 31u, warp = threadIdx.x >> 5;
  uint32_t x = v;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    uint32_t y = __shfl_up_sync(FULL_MASK, x, o);
    if (lane >= uint32_t(o)) x += y;
  }
  if (lane == 31) scratch[warp] = x;
  __syncthreads();
  uint32_t warp_off = 0, sum = 0;
#pragma unroll
  for (int w = 0; w < WARPS; ++w) {
    uint32_t s = scratch[w];
    if (w < int(warp)) warp_off += s;
    sum += s;
  }
  __syncthreads();
  *total = sum;
  return warp_off + x - v;
}

// Self-test of the failure path: waits for *flag to become non-zero, polling
// at most max_polls times about a microsecond apart, then gives up the way
// every wait in this library does (status bit ST_TIMEOUT) and returns.
template <class Ctl>
__global__ void k_selftest_wait(Ctl *ctl, const uint32_t *flag, uint32_t max_polls) {
  if (threadIdx.x != 0) return;
  uint32_t polls = 0;
  while (ld_relaxed_u32(flag) == 0) {
    if (++polls > max_polls) {
      atomicOr(&ctl->status, ST_TIMEOUT);
      return;
    }
    __nanosleep(1000);
  }
}

__device__ __forceinline__ uint32_t warp_exclusive_sum(uint32_t v, uint32_t *total) {
  const uint32_t lane = threadIdx.x & 31u;
  uint32_t x = v;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    uint32_t y = __shfl_up_sync(FULL_MASK, x, o);
    if (lane >= uint32_t(o)) x += y;
  }
  *total = __shfl_sync(FULL_MASK, x, 31);
  return x - v;
}

}  // namespace srcu
