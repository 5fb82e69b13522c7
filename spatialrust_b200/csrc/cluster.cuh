// cluster.cuh -- Euclidean cluster roots on the radius grid.
//
// The component structure of "dx*dx + dy*dy + dz*dz <= tol*tol" (f32, the
// predicate of uniform_grid.rs:440-520 and kdtree.rs:544-549) is unique, and
// so is the reference's answer for each point: the smallest point index of
// its component (union_min_root, uniform_grid.rs:410-418; compress_roots,
// :389-395).  Here the grid of the normal estimator (cell sort, cell table,
// column hash, 3x3 column ranges) supplies the candidates, and a lock-free
// union-find with minimum-index roots links the pairs: a root only ever
// hooks under a smaller root, by compare-and-swap on its own parent word, so
// every tree's root is its smallest member.
#pragma once

#include "normals.cuh"

namespace srcu {

constexpr int CL_THREADS = 256;

__global__ void k_cluster_init(const Control *ctl, uint32_t *parent,
                               const unsigned long long *count_dev) {
  if (ctl->status) return;
  const uint64_t n = count_dev ? *count_dev : ctl->n_points;
  for (uint64_t i = blockIdx.x * uint64_t(blockDim.x) + threadIdx.x; i < n;
       i += uint64_t(gridDim.x) * blockDim.x)
    parent[i] = uint32_t(i);
}

// Root of x with path halving.  Parents only ever move to ancestors, so the
// halving writes race benignly with other finds and with the hooks (a hook
// only rewrites the parent word of a root, which this never writes).
__device__ __forceinline__ uint32_t uf_find(uint32_t *parent, uint32_t x, uint32_t *status) {
  for (uint32_t it = 0; it < SPIN_LIMIT; ++it) {
    const uint32_t p = ld_relaxed_u32(parent + x);
    if (p == x) return x;
    const uint32_t gp = ld_relaxed_u32(parent + p);
    if (gp != p) st_relaxed_u32(parent + x, gp);
    x = gp;
  }
  atomicOr(status, ST_TIMEOUT);
  return x;
}

__device__ __forceinline__ void uf_union(uint32_t *parent, uint32_t a, uint32_t b,
                                         uint32_t *status) {
  for (uint32_t it = 0; it < SPIN_LIMIT; ++it) {
    uint32_t ra = uf_find(parent, a, status), rb = uf_find(parent, b, status);
    if (ra == rb) return;
    if (ra > rb) {
      const uint32_t t = ra;
      ra = rb;
      rb = t;
    }
    // hook the larger root under the smaller one; a failed swap means rb
    // stopped being a root meanwhile, so both roots are looked up again
    if (atomicCAS(parent + rb, rb, ra) == rb) return;
  }
  atomicOr(status, ST_TIMEOUT);
}

// One lane per cell-sorted point i: every candidate j > i of its 27-cell
// neighbourhood (each unordered pair once) that passes the predicate is
// unioned with it, by original point index.
__global__ void __launch_bounds__(CL_THREADS) k_cluster_union(Control *ctl, const float4 *pts,
                                                              const uint32_t *pt_cell,
                                                              const uint2 *ranges,
                                                              const unsigned long long *count_dev,
                                                              float r2, uint32_t *parent) {
  if (ld_relaxed_u32(&ctl->status)) return;
  const uint32_t n = uint32_t(count_dev ? *count_dev : ctl->n_points);
  const uint64_t u_count = ctl->n_cells;
  for (uint32_t i = blockIdx.x * CL_THREADS + threadIdx.x; i < n; i += gridDim.x * CL_THREADS) {
    const float4 q = pts[i];
    const uint32_t u = pt_cell[i];
    const uint32_t a = __float_as_uint(q.w);
    if (u >= u_count || a >= n) {  // cannot happen for a consistent cell table
      atomicOr(&ctl->status, ST_INTERNAL);
      continue;
    }
    const uint2 *rg = ranges + size_t(u) * 9;
#pragma unroll 1
    for (int r = 0; r < 9; ++r) {
      const uint2 range = rg[r];
      for (uint32_t j = range.x > i + 1 ? range.x : i + 1; j < range.y; ++j) {
        const float4 c = __ldg(pts + j);
        const float dx = __fsub_rn(c.x, q.x);
        const float dy = __fsub_rn(c.y, q.y);
        const float dz = __fsub_rn(c.z, q.z);
        const float d2 =
            __fadd_rn(__fadd_rn(__fmul_rn(dx, dx), __fmul_rn(dy, dy)), __fmul_rn(dz, dz));
        if (d2 <= r2) {
          const uint32_t b = __float_as_uint(c.w);
          if (b < n) uf_union(parent, a, b, &ctl->status);
          else atomicOr(&ctl->status, ST_INTERNAL);
        }
      }
    }
  }
}

// roots[i] = the (smallest-index) root of point i.
__global__ void k_cluster_roots(Control *ctl, uint32_t *parent, uint32_t *roots,
                                const unsigned long long *count_dev) {
  if (ld_relaxed_u32(&ctl->status)) return;
  const uint64_t n = count_dev ? *count_dev : ctl->n_points;
  for (uint64_t i = blockIdx.x * uint64_t(blockDim.x) + threadIdx.x; i < n;
       i += uint64_t(gridDim.x) * blockDim.x)
    roots[i] = uf_find(parent, uint32_t(i), &ctl->status);
}

}  // namespace srcu
