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
// Records are staged through shared memory with 16-byte loads (global and
// shared addresses congruent mod 16, head and tail bytes loaded singly, so
// nothing outside the record array is read), then each thread parses one
// record with funnel shifts over aligned 32-bit words.
#pragma once

#include "common.cuh"

namespace srcu {

constexpr int LAS_THREADS = 256;
constexpr uint32_t LAS_SMEM_MAX = 48 * 1024;  // record bytes staged per tile

struct LasDecodeDev {
  uint64_t n;
  uint32_t record_len;
  uint32_t per_tile;   // records per tile (<= LAS_THREADS)
  uint32_t class_off;  // classification byte
  uint32_t class_mask; // 0x1f for formats 0-5 (bits 5-7 are flags), 0xff for 6-10
  int32_t gps_off;     // -1: the format has no GPS time
  int32_t rgb_off;     // -1: the format has no colour
  int32_t has_origin;
  uint32_t pad;
  double scale[3], offset[3], origin[3];
};

struct LasOutDev {
  float *pos[3];
  float *intensity;
  uint8_t *cls;
  double *gps;
  uint16_t *rgb[3];
};

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

__global__ void __launch_bounds__(LAS_THREADS) k_las_decode(const uint8_t *records, LasDecodeDev d,
                                                           LasOutDev o) {
  extern __shared__ __align__(16) uint8_t las_smem[];
  const uint64_t tiles = (d.n + d.per_tile - 1) / d.per_tile;
  const uint32_t t = threadIdx.x;
  for (uint64_t tile = blockIdx.x; tile < tiles; tile += gridDim.x) {
    const uint64_t first = tile * d.per_tile;
    const uint32_t count = d.n - first < d.per_tile ? uint32_t(d.n - first) : d.per_tile;
    const uint8_t *start = records + first * d.record_len;
    const uint8_t *end = start + uint64_t(count) * d.record_len;
    const uintptr_t base = reinterpret_cast<uintptr_t>(start) & ~uintptr_t(15);
    const uint32_t shift = uint32_t(reinterpret_cast<uintptr_t>(start) - base);
    const uintptr_t lo = (reinterpret_cast<uintptr_t>(start) + 15) & ~uintptr_t(15);
    const uintptr_t hi = reinterpret_cast<uintptr_t>(end) & ~uintptr_t(15);
    if (lo < hi) {
      const uint32_t vecs = uint32_t((hi - lo) / 16);
      const uint4 *src = reinterpret_cast<const uint4 *>(lo);
      uint4 *dst = reinterpret_cast<uint4 *>(las_smem + (lo - base));
      for (uint32_t v = t; v < vecs; v += LAS_THREADS) dst[v] = __ldg(src + v);
      for (uintptr_t b = reinterpret_cast<uintptr_t>(start) + t; b < lo; b += LAS_THREADS)
        las_smem[b - base] = *reinterpret_cast<const uint8_t *>(b);
      for (uintptr_t b = hi + t; b < reinterpret_cast<uintptr_t>(end); b += LAS_THREADS)
        las_smem[b - base] = *reinterpret_cast<const uint8_t *>(b);
    } else {  // the tile lies inside one 16-byte line
      for (uintptr_t b = reinterpret_cast<uintptr_t>(start) + t; b < reinterpret_cast<uintptr_t>(end);
           b += LAS_THREADS)
        las_smem[b - base] = *reinterpret_cast<const uint8_t *>(b);
    }
    __syncthreads();
    if (t < count) {
      const uint32_t r = shift + t * d.record_len;  // this record's first byte in shared memory
      const uint64_t i = first + t;
#pragma unroll
      for (int a = 0; a < 3; ++a) {
        const int32_t raw = int32_t(las_u32(las_smem, r + 4 * a));
        const double v = las_coord(raw, d.scale[a], d.offset[a], d.has_origin, d.origin[a]);
        o.pos[a][i] = __double2float_rn(v);
      }
      if (o.intensity) o.intensity[i] = float(las_u32(las_smem, r + 12) & 0xffffu);
      if (o.cls) o.cls[i] = uint8_t(las_smem[r + d.class_off] & d.class_mask);
      if (o.gps && d.gps_off >= 0) {
        const uint32_t w0 = las_u32(las_smem, r + d.gps_off);
        const uint32_t w1 = las_u32(las_smem, r + d.gps_off + 4);
        o.gps[i] = __hiloint2double(int(w1), int(w0));
      }
      if (d.rgb_off >= 0) {
#pragma unroll
        for (int c = 0; c < 3; ++c)
          if (o.rgb[c]) o.rgb[c][i] = uint16_t(las_u32(las_smem, r + d.rgb_off + 2 * c) & 0xffffu);
      }
    }
    __syncthreads();
  }
}

}  // namespace srcu
