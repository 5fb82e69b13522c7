// las.cuh -- LAS point-record decoding on the device.
//
// The reference reads LAS through the `las` crate (0.9, not vendored) and
// keeps x, y, z, intensity, classification, gps_time and RGB
// (crates/spatialrust-io/src/las/reader.rs:242-279, schema.rs:27-52): each
// coordinate is the f64 `scale * X + offset` of the record's i32 X (the
// published LAS transform), stored as `value as f32`.  Here the same fields
// are decoded from the raw records of the LAS 1.0-1.4 point data record
// formats 0-10 (ASPRS LAS specification 1.4 R15, tables 7-17), with one
// addition: an optional FP64 origin is subtracted before the f32 conversion,
// so georeferenced coordinates keep their precision in the f32 columns.
//
// Records move through shared memory in tiles, double-buffered: one thread
// issues a bulk asynchronous copy (cp.async.bulk, completion counted on an
// mbarrier) of the tile's 16-byte-aligned interior while the block parses the
// previous tile; the unaligned head and tail bytes of a tile are loaded by
// plain loads, so nothing outside the record array is read.  Global and shared
// addresses are congruent mod 16.  Each thread then parses whole records with
// funnel shifts over aligned 32-bit words.  Every mbarrier wait is bounded.
#pragma once

#include "common.cuh"

namespace srcu {

constexpr int LAS_THREADS = 256;
constexpr uint32_t LAS_TILE_RECORDS = 512;   // records per tile (at most)
constexpr uint32_t LAS_BUF_MAX = 48 * 1024;  // record bytes of one tile buffer (at most)

struct LasDecodeDev {
  uint64_t n;
  uint32_t record_len;
  uint32_t per_tile;   // records per tile
  uint32_t buf_bytes;  // bytes of one tile buffer: per_tile * record_len + 32, 16-aligned
  uint32_t class_off;  // classification byte
  uint32_t class_mask; // 0x1f for formats 0-5 (bits 5-7 are flags), 0xff for 6-10
  int32_t gps_off;     // -1: the format has no GPS time
  int32_t rgb_off;     // -1: the format has no colour
  int32_t has_origin;
  double scale[3], offset[3], origin[3];
};

struct LasOutDev {
  float *pos[3];
  float *intensity;
  uint8_t *cls;
  double *gps;
  uint16_t *rgb[3];
};

__device__ __forceinline__ uint32_t smem_addr(const void *p) {
  return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

__device__ __forceinline__ void mbar_init(uint64_t *bar, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_addr(bar)), "r"(count)
               : "memory");
}

// One arrival that also announces `bytes` of asynchronous copy into this phase.
__device__ __forceinline__ void mbar_arrive_expect_tx(uint64_t *bar, uint32_t bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_addr(bar)),
               "r"(bytes)
               : "memory");
}

__device__ __forceinline__ bool mbar_try_wait(uint64_t *bar, uint32_t parity) {
  uint32_t ok;
  asm volatile(
      "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n"
      " selp.u32 %0, 1, 0, p;\n}\n"
      : "=r"(ok)
      : "r"(smem_addr(bar)), "r"(parity)
      : "memory");
  return ok != 0;
}

// Bulk copy global -> this CTA's shared memory; dst, src and bytes 16-byte aligned.
__device__ __forceinline__ void bulk_copy_g2s(void *dst, const void *src, uint32_t bytes,
                                              uint64_t *bar) {
  asm volatile(
      "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
          smem_addr(dst)),
      "l"(src), "r"(bytes), "r"(smem_addr(bar))
      : "memory");
}

__device__ __forceinline__ uint32_t las_u32(const uint8_t *s, uint32_t off) {
  const uint32_t *w = reinterpret_cast<const uint32_t *>(s);
  const uint32_t i = off >> 2;
  return __funnelshift_r(w[i], w[i + 1], (off & 3u) * 8u);
}

__device__ __forceinline__ double las_coord(int32_t raw, double scale, double offset,
                                            int has_origin, double origin) {
  // scale * X + offset, each step rounded (no contraction), then - origin
  double v = __dadd_rn(__dmul_rn(scale, double(raw)), offset);
  if (has_origin) v = __dsub_rn(v, origin);
  return v;
}

// Byte range of one tile and its placement in a tile buffer.
struct LasTile {
  uintptr_t start, end, base, lo, hi;
  uint32_t count, shift;
  uint64_t first;
};

__device__ __forceinline__ LasTile las_tile(const uint8_t *records, const LasDecodeDev &d,
                                            uint64_t tile) {
  LasTile t;
  t.first = tile * d.per_tile;
  t.count = d.n - t.first < d.per_tile ? uint32_t(d.n - t.first) : d.per_tile;
  t.start = reinterpret_cast<uintptr_t>(records + t.first * d.record_len);
  t.end = t.start + uint64_t(t.count) * d.record_len;
  t.base = t.start & ~uintptr_t(15);
  t.shift = uint32_t(t.start - t.base);
  t.lo = (t.start + 15) & ~uintptr_t(15);
  t.hi = t.end & ~uintptr_t(15);
  if (t.lo > t.hi) t.lo = t.hi = t.end;  // the tile lies inside one 16-byte line
  return t;
}

__global__ void __launch_bounds__(LAS_THREADS) k_las_decode(const uint8_t *records, LasDecodeDev d,
                                                           LasOutDev o, uint32_t *status) {
  extern __shared__ __align__(128) uint8_t las_smem[];
  __shared__ __align__(8) uint64_t bars[2];
  const uint64_t tiles = (d.n + d.per_tile - 1) / d.per_tile;
  if (blockIdx.x >= tiles) return;  // whole block, before any barrier
  const uint64_t mine = (tiles - blockIdx.x + gridDim.x - 1) / gridDim.x;
  const uint32_t t = threadIdx.x;
  if (t == 0) {
    mbar_init(&bars[0], 1);
    mbar_init(&bars[1], 1);
  }
  __syncthreads();
  // Starts the copy of this block's k-th tile into buffer k & 1.
  auto stage = [&](uint64_t k) {
    const LasTile tl = las_tile(records, d, blockIdx.x + k * gridDim.x);
    uint8_t *buf = las_smem + (k & 1) * d.buf_bytes;
    if (t == 0) {
      // order this buffer's earlier generic accesses before the async copy
      asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
      const uint32_t bytes = uint32_t(tl.hi - tl.lo);
      mbar_arrive_expect_tx(&bars[k & 1], bytes);
      if (bytes) bulk_copy_g2s(buf + (tl.lo - tl.base), reinterpret_cast<const void *>(tl.lo), bytes,
                               &bars[k & 1]);
    }
    for (uintptr_t b = tl.start + t; b < tl.lo; b += LAS_THREADS)
      buf[b - tl.base] = *reinterpret_cast<const uint8_t *>(b);
    for (uintptr_t b = tl.hi + t; b < tl.end; b += LAS_THREADS)
      buf[b - tl.base] = *reinterpret_cast<const uint8_t *>(b);
  };
  auto wait = [&](uint64_t k) -> bool {
    uint32_t spins = 0;
    while (!mbar_try_wait(&bars[k & 1], uint32_t(k >> 1) & 1u))
      if (++spins > SPIN_LIMIT) return false;
    return true;
  };
  stage(0);
  for (uint64_t k = 0; k < mine; ++k) {
    if (k + 1 < mine) stage(k + 1);
    const bool ok = wait(k);
    // plain-loaded head/tail bytes of tile k are visible after this barrier
    if (__syncthreads_or(!ok)) {
      if (t == 0) atomicOr(status, ST_TIMEOUT);
      if (k + 1 < mine) wait(k + 1);  // the copy in flight, again bounded
      return;
    }
    const LasTile tl = las_tile(records, d, blockIdx.x + k * gridDim.x);
    const uint8_t *buf = las_smem + (k & 1) * d.buf_bytes;
    for (uint32_t j = t; j < tl.count; j += LAS_THREADS) {
      const uint32_t r = tl.shift + j * d.record_len;  // this record's first byte in the buffer
      const uint64_t i = tl.first + j;
#pragma unroll
      for (int a = 0; a < 3; ++a) {
        const int32_t raw = int32_t(las_u32(buf, r + 4 * a));
        o.pos[a][i] = __double2float_rn(las_coord(raw, d.scale[a], d.offset[a], d.has_origin,
                                                  d.origin[a]));
      }
      if (o.intensity) o.intensity[i] = float(las_u32(buf, r + 12) & 0xffffu);
      if (o.cls) o.cls[i] = uint8_t(buf[r + d.class_off] & d.class_mask);
      if (o.gps && d.gps_off >= 0) {
        const uint32_t w0 = las_u32(buf, r + d.gps_off);
        const uint32_t w1 = las_u32(buf, r + d.gps_off + 4);
        o.gps[i] = __hiloint2double(int(w1), int(w0));
      }
      if (d.rgb_off >= 0) {
#pragma unroll
        for (int c = 0; c < 3; ++c)
          if (o.rgb[c]) o.rgb[c][i] = uint16_t(las_u32(buf, r + d.rgb_off + 2 * c) & 0xffffu);
      }
    }
    __syncthreads();  // buffer k & 1 is free for tile k + 2
  }
}

}  // namespace srcu
