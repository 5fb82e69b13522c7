// ransac.cuh -- RANSAC plane hypothesis scoring on the device.
//
// The reference's CPU segmenter (crates/spatialrust-segmentation/src/
// plane.rs:266-301, plane_ransac.rs:54-94) builds each hypothesis plane from
// three points in f32 (plane_from_points: cross product, normalize, d =
// -n.p0) and counts the points with |n.p + d| <= threshold (distance_xyz,
// plane.rs:39-41).  The same f32 expressions are evaluated here in the same
// order with round-to-nearest and no contraction, so every count equals the
// reference's, and so do the best hypothesis and its inlier set.
//
// Scoring is compute-bound work of n x H predicate evaluations: each thread
// keeps RS_PTS points in registers, the block walks every plane held in
// shared memory, and counts go warp-reduced into shared then global counters.
#pragma once

#include "common.cuh"

namespace srcu {

constexpr int RS_THREADS = 256;
constexpr int RS_PTS = 8;                        // points per thread
constexpr int RS_TILE = RS_THREADS * RS_PTS;     // points per block
constexpr int RS_PLANES = 2048;                  // planes per shared-memory chunk

// plane_from_points (plane_ransac.rs:79-89) in f32: invalid when |n|^2 < 1e-12.
__global__ void k_ransac_planes(const float *x, const float *y, const float *z, uint64_t n,
                                const uint32_t *hyp, uint32_t count, float4 *planes,
                                uint32_t *valid, uint32_t *status) {
  const uint32_t h = blockIdx.x * blockDim.x + threadIdx.x;
  if (h >= count) return;
  const uint32_t i0 = hyp[3 * h], i1 = hyp[3 * h + 1], i2 = hyp[3 * h + 2];
  if (i0 >= n || i1 >= n || i2 >= n) {  // cannot happen: indices are drawn below n
    atomicOr(status, ST_INTERNAL);
    planes[h] = make_float4(0.f, 0.f, 0.f, 0.f);
    valid[h] = 0;
    return;
  }
  const float p0x = x[i0], p0y = y[i0], p0z = z[i0];
  const float v1x = __fsub_rn(x[i1], p0x), v1y = __fsub_rn(y[i1], p0y), v1z = __fsub_rn(z[i1], p0z);
  const float v2x = __fsub_rn(x[i2], p0x), v2y = __fsub_rn(y[i2], p0y), v2z = __fsub_rn(z[i2], p0z);
  // Vec3::cross (crates/spatialrust-math/src/vec.rs:71-78)
  float nx = __fsub_rn(__fmul_rn(v1y, v2z), __fmul_rn(v1z, v2y));
  float ny = __fsub_rn(__fmul_rn(v1z, v2x), __fmul_rn(v1x, v2z));
  float nz = __fsub_rn(__fmul_rn(v1x, v2y), __fmul_rn(v1y, v2x));
  const float ls = __fadd_rn(__fadd_rn(__fmul_rn(nx, nx), __fmul_rn(ny, ny)), __fmul_rn(nz, nz));
  if (ls < 1e-12f) {  // no plane (a NaN length goes on and counts no inlier)
    planes[h] = make_float4(0.f, 0.f, 0.f, 0.f);
    valid[h] = 0;
    return;
  }
  // Vec3::normalize (vec.rs:94-100): x / sqrt(x.x)
  const float len = __fsqrt_rn(ls);
  nx = __fdiv_rn(nx, len);
  ny = __fdiv_rn(ny, len);
  nz = __fdiv_rn(nz, len);
  const float dot = __fadd_rn(__fadd_rn(__fmul_rn(nx, p0x), __fmul_rn(ny, p0y)), __fmul_rn(nz, p0z));
  planes[h] = make_float4(nx, ny, nz, -dot);
  valid[h] = 1;
}

// PlaneModel::distance_xyz (plane.rs:39-41) <= threshold, in the reference's order.
__device__ __forceinline__ bool plane_inlier(float4 pl, float px, float py, float pz, float thr) {
  const float s = __fadd_rn(__fadd_rn(__fadd_rn(__fmul_rn(pl.x, px), __fmul_rn(pl.y, py)),
                                      __fmul_rn(pl.z, pz)),
                            pl.w);
  return fabsf(s) <= thr;
}

// counts[h] += inliers of plane h among this block's RS_TILE points, for the
// planes [blockIdx.y * per_chunk, +per_chunk): the second grid dimension
// splits the hypotheses so that small clouds still fill every SM.
__global__ void __launch_bounds__(RS_THREADS) k_ransac_score(const float *x, const float *y,
                                                             const float *z, uint64_t n,
                                                             const float4 *planes, uint32_t count,
                                                             uint32_t per_chunk, float thr,
                                                             uint32_t *counts) {
  __shared__ float4 sp[RS_PLANES];
  __shared__ uint32_t sc[RS_PLANES];
  float px[RS_PTS], py[RS_PTS], pz[RS_PTS];
  const uint64_t first = uint64_t(blockIdx.x) * RS_TILE;
#pragma unroll
  for (int k = 0; k < RS_PTS; ++k) {
    const uint64_t i = first + uint64_t(k) * RS_THREADS + threadIdx.x;  // coalesced
    const bool in = i < n;
    px[k] = in ? x[i] : __int_as_float(0x7fc00000);  // NaN: never an inlier
    py[k] = in ? y[i] : 0.f;
    pz[k] = in ? z[i] : 0.f;
  }
  const uint32_t lane = threadIdx.x & 31u;
  const uint32_t c_begin = blockIdx.y * per_chunk;
  const uint32_t c_end = min(count, c_begin + per_chunk);
  for (uint32_t c0 = c_begin; c0 < c_end; c0 += RS_PLANES) {
    const uint32_t m = min(uint32_t(RS_PLANES), c_end - c0);
    for (uint32_t j = threadIdx.x; j < m; j += RS_THREADS) {
      sp[j] = planes[c0 + j];
      sc[j] = 0;
    }
    __syncthreads();
    for (uint32_t j = 0; j < m; ++j) {
      const float4 pl = sp[j];
      uint32_t c = 0;
#pragma unroll
      for (int k = 0; k < RS_PTS; ++k) c += plane_inlier(pl, px[k], py[k], pz[k], thr) ? 1u : 0u;
      c = __reduce_add_sync(FULL_MASK, c);
      if (lane == 0 && c) atomicAdd(&sc[j], c);
    }
    __syncthreads();
    for (uint32_t j = threadIdx.x; j < m; j += RS_THREADS)
      if (sc[j]) atomicAdd(&counts[c0 + j], sc[j]);
    __syncthreads();
  }
}

// Inlier mask of one plane, and per-block FP64 partial sums over the inliers:
// pass 0: count, sum x, y, z; pass 1 (with the mean): the six centred second
// moments (refine_plane_from_inliers, plane_ransac.rs:96-150).  Blocks sum in
// a fixed order, so the result does not depend on scheduling.
constexpr int RM_THREADS = 256;

__global__ void __launch_bounds__(RM_THREADS) k_ransac_moments(const float *x, const float *y,
                                                               const float *z, uint64_t n,
                                                               const float4 *plane, float thr,
                                                               uint8_t *mask, int pass,
                                                               double3 mean, double *partials) {
  __shared__ double red[RM_THREADS];
  const float4 pl = *plane;
  double acc[6] = {0, 0, 0, 0, 0, 0};
  for (uint64_t i = blockIdx.x * uint64_t(RM_THREADS) + threadIdx.x; i < n;
       i += uint64_t(gridDim.x) * RM_THREADS) {
    const float px = x[i], py = y[i], pz = z[i];
    const bool in = plane_inlier(pl, px, py, pz, thr);
    if (pass == 0) {
      if (mask) mask[i] = in ? 1 : 0;
      if (in) {
        acc[0] += 1.0;
        acc[1] += double(px);
        acc[2] += double(py);
        acc[3] += double(pz);
      }
    } else if (in) {
      const double dx = double(px) - mean.x, dy = double(py) - mean.y, dz = double(pz) - mean.z;
      acc[0] += dx * dx;
      acc[1] += dy * dy;
      acc[2] += dz * dz;
      acc[3] += dx * dy;
      acc[4] += dx * dz;
      acc[5] += dy * dz;
    }
  }
  const int terms = pass == 0 ? 4 : 6;
  for (int k = 0; k < terms; ++k) {
    red[threadIdx.x] = acc[k];
    __syncthreads();
    for (int w = RM_THREADS / 2; w > 0; w >>= 1) {
      if (int(threadIdx.x) < w) red[threadIdx.x] += red[threadIdx.x + w];
      __syncthreads();
    }
    if (threadIdx.x == 0) partials[blockIdx.x * 6 + k] = red[0];
    __syncthreads();
  }
}

}  // namespace srcu
