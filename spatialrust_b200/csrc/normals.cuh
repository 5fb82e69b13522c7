// normals.cuh -- uniform-grid radius normals: cell plan, cell table, hashed
// cell lookup, 3x3-column neighbour ranges, and the radius-neighbour
// covariance + eigensolve kernel.
//
// Semantics follow NormalEstimator's CPU radius mode
// (crates/spatialrust-features/src/normal.rs:102-164, 321-473): a neighbour
// of query q is any other point p with
//   (px-qx)^2 + (py-qy)^2 + (pz-qz)^2 <= r*r
// evaluated in f32 with round-to-nearest and no FMA, in exactly that order
// (kdtree.rs:544-549), so neighbour sets -- and counts -- are bit-identical
// to the reference's KD-tree search.  Points with fewer than min_neighbors
// neighbours get a NaN normal and curvature 0 (normal.rs:331-346).
#pragma once

#include "eig3.cuh"
#include "radix.cuh"

namespace srcu {

// Cell plan of each cloud from its bounds (any box that contains every
// finite point works).  h >= r (1 + 1e-5): points within r (f32 predicate)
// then differ by at most one cell per axis even after the FP64 cell
// arithmetic.  h is also kept >= extent / 2^19 so every axis fits in 20
// bits; larger cells only add candidates, never drop neighbours.
__global__ void k_cell_plans(Control *ctl, Batch bt) {
  if (ld_relaxed_u32(&ctl->status)) return;
  const uint32_t b = blockIdx.x * blockDim.x + threadIdx.x;
  if (b >= bt.clouds) return;
  const float radius = bt.nparams[b].radius;
  if (!(radius >= 0.0f) || isinf(radius)) {
    atomicOr(&ctl->status, ST_BAD_PARAMS);
    return;
  }
  CellPlan pl{};
  const Bounds bd = bt.bounds[b];
  double lo[3], ext[3], max_ext = 0.0;
  for (int a = 0; a < 3; ++a) {
    const bool any = bd.mn[a] != 0xffffffffu;
    lo[a] = any ? double(ord2f(bd.mn[a])) : 0.0;
    const double hi = any ? double(ord2f(bd.mx[a])) : 0.0;
    ext[a] = hi - lo[a];
    max_ext = fmax(max_ext, ext[a]);
  }
  double h = double(radius) * (1.0 + 1e-5);
  h = fmax(h, max_ext * (1.0 / 524288.0));
  h = fmax(h, 1e-30);
  uint32_t total = 0;
  for (int a = 0; a < 3; ++a) {
    const double d = floor(ext[a] / h) + 1.0;
    pl.dims[a] = d > 1048576.0 ? 1048576u : uint32_t(d);
    pl.bits[a] = bit_width_u64(pl.dims[a] - 1);
    total += pl.bits[a];
    pl.origin[a] = lo[a];
  }
  pl.h = h;
  pl.inv_h = 1.0 / h;
  pl.shift_y = pl.bits[2];
  pl.shift_x = pl.bits[1] + pl.bits[2];
  pl.total_bits = total;
  pl.num_digits = total == 0 ? 1u : (total + RADIX_BITS - 1) / RADIX_BITS;
  pl.r2 = __fmul_rn(radius, radius);
  pl.shell_tol = __fmul_rn(1e-6f, pl.r2);
  pl.valid = 1;
  bt.cplans[b] = pl;
  atomicMax(&ctl->ckey_bits, total);
  if (total + ctl->cloud_bits > 64) atomicOr(&ctl->status, ST_KEY_OVERFLOW);
}

// Places every cloud's (cx, cy) columns in one dense table when all of them
// fit its `capacity` slots: col_base per cloud by a block scan over clouds.
// Otherwise the chain keeps the column hash.  One block.
__global__ void k_column_base(Control *ctl, Batch bt, uint64_t capacity) {
  if (ld_relaxed_u32(&ctl->status)) return;
  __shared__ unsigned long long scratch[256];
  unsigned long long running = 0;
  for (uint32_t b0 = 0; b0 < bt.clouds; b0 += 256) {
    const uint32_t b = b0 + threadIdx.x;
    unsigned long long cols = 0;
    if (b < bt.clouds) cols = (unsigned long long)bt.cplans[b].dims[0] * bt.cplans[b].dims[1];
    scratch[threadIdx.x] = cols;
    __syncthreads();
    for (uint32_t off = 1; off < 256; off <<= 1) {  // inclusive Hillis-Steele scan
      const unsigned long long v = threadIdx.x >= off ? scratch[threadIdx.x - off] : 0ull;
      __syncthreads();
      scratch[threadIdx.x] += v;
      __syncthreads();
    }
    if (b < bt.clouds) bt.cplans[b].col_base = running + scratch[threadIdx.x] - cols;
    running += scratch[255];
    __syncthreads();
  }
  if (threadIdx.x == 0) {
    ctl->col_total = running;
    ctl->dense_cols = running <= capacity ? 1u : 0u;
  }
}

__device__ __forceinline__ uint64_t dense_column(const CellPlan &pl, uint64_t cx, uint64_t cy) {
  return pl.col_base + cx * pl.dims[1] + cy;
}

// Key source for the cell sort over `count_dev` points (V for the chained
// voxel -> normals path, n otherwise).  The cloud of point i comes from its
// packed voxel key (chained path) or from the batch offsets.
struct CellKeySrc {
  const float *x, *y, *z;
  const unsigned long long *count_dev;
  const uint64_t *voxel_keys;  // non-null: points are voxel centroids in key order
  Batch bt;
  CellPlan pl;  // the plan when there is one cloud
  uint32_t local_bits, cloud_bits, voxel_local_bits;
  __device__ __forceinline__ void prepare(const Control *ctl) {
    local_bits = ctl->ckey_bits;
    cloud_bits = ctl->cloud_bits;
    voxel_local_bits = ctl->vkey_bits;
    if (bt.clouds == 1) pl = bt.cplans[0];
  }
  __device__ __forceinline__ uint32_t count(const Control *ctl) const {
    return uint32_t(count_dev ? *count_dev : ctl->n_points);
  }
  __device__ __forceinline__ uint32_t key_bits() const { return local_bits + cloud_bits; }
  __device__ __forceinline__ uint32_t cloud(uint32_t i) const {
    if (voxel_keys) return voxel_local_bits >= 64 ? 0u : uint32_t(voxel_keys[i] >> voxel_local_bits);
    return cloud_of(bt, i);
  }
  __device__ __forceinline__ uint64_t key(uint32_t i) const {
    if (bt.clouds == 1) return cell_pack(pl, x[i], y[i], z[i]);
    const uint32_t b = cloud(i);
    return with_cloud(cell_pack(bt.cplans[b], x[i], y[i], z[i]), b, local_bits);
  }
};

constexpr int CELL_THREADS = 256;
// 1024-point tiles: at 417k points (C1's leaf-0.5 centroids) twice the tiles of
// 2048-point ones spread the look-back-bound tiles over every SM (45 -> 27 us),
// with no loss at 1.8M; 512-point tiles lose at 1.8M.
constexpr int CELL_ITEMS = 4;
constexpr int CELL_TILE = CELL_THREADS * CELL_ITEMS;

struct CellSmem {
  uint64_t keys[CELL_TILE + 1];
  uint32_t scratch[CELL_THREADS / 32];
  uint32_t tile;
};

// Cell table: gathers points into cell-sorted float4 records
// (x, y, z, bits of the original index), numbers the occupied cells (start
// offsets in the sorted order, cell keys; cell_start[U] = n) and records each
// sorted point's cell number.
__global__ void __launch_bounds__(CELL_THREADS) k_cells(Control *ctl, SortBuffers sort,
                                                        const SortState *sort_state,
                                                        const unsigned long long *count_dev,
                                                        const float4 *aos, float4 *pts,
                                                        uint32_t *pt_cell, uint64_t *cell_key,
                                                        uint32_t *cell_start, uint64_t *lookback) {
  __shared__ CellSmem sm;
  if (ld_relaxed_u32(&ctl->status)) return;
  const uint32_t n = uint32_t(count_dev ? *count_dev : ctl->n_points);
  if (n == 0) {
    if (blockIdx.x == 0 && threadIdx.x == 0) {
      ctl->n_cells = 0;
      cell_start[0] = 0;
    }
    return;
  }
  const SortedView sv = sorted_view(sort, *sort_state);
  const uint32_t epoch = ctl->epoch + EP_CELLS;
  const uint32_t num_tiles = (n + CELL_TILE - 1) / CELL_TILE;
  const uint32_t t = threadIdx.x;
  for (;;) {
    if (t == 0) sm.tile = atomicAdd(&ctl->work[WK_CELLS], 1u);
    __syncthreads();
    const uint32_t tile = sm.tile;
    if (tile >= num_tiles) break;
    const uint32_t base = tile * CELL_TILE;
    const uint32_t tile_n = min(uint32_t(CELL_TILE), n - base);
    for (uint32_t j = t; j < tile_n; j += CELL_THREADS) {
      sm.keys[1 + j] = sv.key(base + j);
      const uint32_t v = sv.val(base + j);
      if (v < n) {
        const float4 p = aos[v];
        pts[base + j] = make_float4(p.x, p.y, p.z, __uint_as_float(v));
      } else {  // a consistent sort never produces this; never read out of bounds
        pts[base + j] = make_float4(__int_as_float(0x7fc00000), 0.f, 0.f, __uint_as_float(0u));
        atomicOr(&ctl->status, ST_INTERNAL);
      }
    }
    if (t == 0) sm.keys[0] = base > 0 ? sv.key(base - 1) : ~sv.key(0);
    __syncthreads();
    const uint32_t j0 = t * CELL_ITEMS;
    uint32_t flags = 0;
#pragma unroll
    for (int i = 0; i < CELL_ITEMS; ++i) {
      const uint32_t j = j0 + i;
      if (j < tile_n && sm.keys[1 + j] != sm.keys[j]) flags |= 1u << i;
    }
    uint32_t tile_count;
    const uint32_t local = block_exclusive_sum<CELL_THREADS>(__popc(flags), sm.scratch, &tile_count);
    if (t < 32) {
      const uint32_t cb = lookback_exclusive_warp(lookback, tile, tile_count, epoch, &ctl->status);
      if (t == 0) sm.scratch[0] = cb;
    }
    __syncthreads();
    const uint32_t cbase = sm.scratch[0];
    uint32_t c = cbase + local;
#pragma unroll
    for (int i = 0; i < CELL_ITEMS; ++i) {
      const uint32_t j = j0 + i;
      if (flags & (1u << i)) {
        if (c < n) {
          cell_key[c] = sm.keys[1 + j];
          cell_start[c] = base + j;
        } else {
          atomicOr(&ctl->status, ST_INTERNAL);
        }
        ++c;
      }
      if (j < tile_n) pt_cell[base + j] = c - 1;  // the cell this point belongs to
    }
    if (t == 0 && tile == num_tiles - 1) {
      const uint32_t u_total = min(cbase + tile_count, n);
      ctl->n_cells = u_total;
      cell_start[u_total] = n;
    }
    __syncthreads();
  }
}

// Open-addressing table from cell key to cell number.  A slot holds
// [epoch:32][cell:32]; slots from earlier chains read as empty, so the table
// is cleared once at allocation only.  Keys are compared through cell_key[].
__device__ __forceinline__ uint32_t cell_hash(uint64_t key, uint32_t log2cap) {
  return uint32_t((key * 0x9E3779B97F4A7C15ull) >> (64 - log2cap));
}

// Column of a cell key: the key with its z field cleared, so the cloud id and
// the x, y fields name the column.  The cells of one column are consecutive
// in key order, sorted by z.
__device__ __forceinline__ uint64_t column_mask(const Batch &bt, uint32_t b) {
  return ~((1ull << bt.cplans[b < bt.clouds ? b : 0].bits[2]) - 1ull);
}

__device__ __forceinline__ uint32_t cloud_of_key(uint64_t full, const Batch &bt, uint32_t lb) {
  return (bt.clouds == 1 || lb >= 64) ? 0u : uint32_t(full >> lb);
}

// Hashes every occupied column to its first cell: one insert per column head
// (a cell whose predecessor lies in another column).  Slots hold
// [epoch:32][first cell:32]; the column key itself is read back from
// cell_key[first], so a slot is 8 bytes and the table never needs clearing.
__global__ void k_column_insert(Control *ctl, const uint64_t *cell_key, uint64_t *table,
                                uint32_t log2cap, Batch bt) {
  if (ld_relaxed_u32(&ctl->status)) return;
  const uint64_t u_count = ctl->n_cells;
  const uint32_t epoch = ctl->epoch + EP_CELLS;
  const uint32_t lb = ctl->ckey_bits;
  const uint32_t mask = (1u << log2cap) - 1u;
  const bool dense = ctl->dense_cols != 0;
  for (uint64_t u = blockIdx.x * uint64_t(blockDim.x) + threadIdx.x; u < u_count;
       u += uint64_t(gridDim.x) * blockDim.x) {
    const uint64_t full = cell_key[u];
    const uint32_t b = cloud_of_key(full, bt, lb);
    const uint64_t col = full & column_mask(bt, b);
    if (u > 0) {
      const uint64_t prev = cell_key[u - 1];
      if ((prev & column_mask(bt, cloud_of_key(prev, bt, lb))) == col) continue;
    }
    if (dense) {  // one slot per column: a plain store
      const CellPlan &pl = bt.cplans[b < bt.clouds ? b : 0];
      uint32_t cx, cy, cz;
      cell_unpack(pl, full & (lb >= 64 ? ~0ull : ((1ull << lb) - 1)), cx, cy, cz);
      const uint64_t idx = dense_column(pl, cx, cy);
      if (idx <= mask) table[idx] = (uint64_t(epoch) << 32) | u;
      else atomicOr(&ctl->status, ST_INTERNAL);
      continue;
    }
    uint32_t h = cell_hash(col, log2cap);
    const uint64_t mine = (uint64_t(epoch) << 32) | u;
    bool done = false;
    for (uint32_t probe = 0; probe <= mask && !done; ++probe) {
      unsigned long long *slot = reinterpret_cast<unsigned long long *>(table + h);
      unsigned long long old = *reinterpret_cast<volatile unsigned long long *>(slot);
      while (uint32_t(old >> 32) != epoch) {
        const unsigned long long seen = atomicCAS(slot, old, (unsigned long long)mine);
        if (seen == old) {
          done = true;
          break;
        }
        old = seen;
      }
      h = (h + 1) & mask;
    }
    if (!done) atomicOr(&ctl->status, ST_HASH_FULL);
  }
}

// First cell of column `col` (cloud b), or -1 when the column is empty.
__device__ __forceinline__ int64_t column_lookup(const uint64_t *table, const uint64_t *cell_key,
                                                 uint64_t col, uint64_t cmask, uint32_t log2cap,
                                                 uint32_t epoch) {
  const uint32_t mask = (1u << log2cap) - 1u;
  uint32_t h = cell_hash(col, log2cap);
  for (uint32_t probe = 0; probe <= mask; ++probe) {
    const uint64_t w = table[h];
    if (uint32_t(w >> 32) != epoch) return -1;
    const uint32_t f = uint32_t(w);
    // a head of another cloud differs in the cloud bits, which cmask keeps
    if ((cell_key[f] & cmask) == col) return f;
    h = (h + 1) & mask;
  }
  return -1;
}

// Key arithmetic of k_ranges in K (uint32_t where the chain's cell keys with
// their cloud bits fit 31 bits, uint64_t otherwise): a shift or a mask as wide
// as K is defined here, where C++ leaves it undefined.
template <class K>
__device__ __forceinline__ K shl_k(K v, uint32_t s) {
  return s >= 8 * sizeof(K) ? K(0) : K(v << s);
}
template <class K>
__device__ __forceinline__ K shr_k(K v, uint32_t s) {
  return s >= 8 * sizeof(K) ? K(0) : K(v >> s);
}
template <class K>
__device__ __forceinline__ K low_mask_k(uint32_t bits) {
  return bits >= 8 * sizeof(K) ? ~K(0) : K((K(1) << bits) - K(1));
}

// The 9 column ranges of cell u (see k_ranges), with cell keys held in K.
template <class K>
__device__ __forceinline__ void ranges_of_cell(uint32_t u, uint32_t u_count, const uint64_t *cell_key,
                                               const uint32_t *cell_start, const uint64_t *table,
                                               uint32_t log2cap, uint32_t tmask, bool dense,
                                               uint32_t epoch, uint32_t lb, const Batch &bt,
                                               uint2 *ranges) {
  const K none = ~K(0);  // no column: above every key (keys have at most 31 bits in uint32_t)
  const K full = K(cell_key[u]);
  const uint32_t b = (bt.clouds == 1 || lb >= 8 * sizeof(K)) ? 0u : uint32_t(shr_k<K>(full, lb));
  const CellPlan &pl = bt.cplans[b < bt.clouds ? b : 0];
  const int32_t dims0 = int32_t(pl.dims[0]), dims1 = int32_t(pl.dims[1]);
  const uint32_t dims2 = pl.dims[2];
  const uint32_t sx = pl.shift_x, sy = pl.shift_y;
  const K local = full & low_mask_k<K>(lb);
  const uint32_t cz = uint32_t(local & low_mask_k<K>(pl.bits[2]));
  const uint32_t cy = uint32_t(shr_k<K>(local, sy) & low_mask_k<K>(pl.bits[1]));
  const uint32_t cx = uint32_t(shr_k<K>(local, sx));
  const K cmask = ~low_mask_k<K>(pl.bits[2]);
  const K cloud_part = (bt.clouds == 1) ? K(0) : shl_k<K>(K(b), lb);
  const K zlo = cz > 0 ? K(cz - 1) : K(0);
  const K zhi = cz + 1 < dims2 ? K(cz + 1) : K(cz);
  uint2 *out = ranges + size_t(u) * 9;
  // centre column
  {
    uint32_t first = u, last = u;
    if (cz > 0 && u > 0 && K(cell_key[u - 1]) == full - K(1)) first = u - 1;
    if (cz + 1 < dims2 && u + 1 < u_count && K(cell_key[u + 1]) == full + K(1)) last = u + 1;
    out[4] = make_uint2(cell_start[first], cell_start[last + 1]);
  }
  // (1) column keys and first probes (a dense slot, or the first hash
  // slot), all loads issued together
  K ckey[8];
  uint32_t slot[8];
  uint64_t word[8];
#pragma unroll
  for (int k = 0; k < 8; ++k) {
    const int col = k < 4 ? k : k + 1;
    const int32_t nx = int32_t(cx) + col / 3 - 1;
    const int32_t ny = int32_t(cy) + col % 3 - 1;
    const bool inside = nx >= 0 && ny >= 0 && nx < dims0 && ny < dims1;
    ckey[k] = inside ? K(shl_k<K>(K(nx), sx) | shl_k<K>(K(ny), sy) | cloud_part) : none;
    uint64_t idx = cell_hash(uint64_t(ckey[k]), log2cap);
    if (dense) idx = inside ? dense_column(pl, uint64_t(nx), uint64_t(ny)) : 0;
    slot[k] = uint32_t(idx);
    word[k] = (inside && idx <= tmask) ? table[idx] : 0ull;
  }
  // first cell of each column (or -1), resolving hash probe chains
  int32_t f[8];
#pragma unroll
  for (int k = 0; k < 8; ++k) {
    f[k] = -1;
    if (dense) {
      if (ckey[k] != none && uint32_t(word[k] >> 32) == epoch) f[k] = int32_t(uint32_t(word[k]));
    } else if (ckey[k] != none) {
      uint32_t h = slot[k];
      uint64_t w = word[k];
      for (uint32_t probe = 0; probe <= tmask; ++probe) {
        if (uint32_t(w >> 32) != epoch) break;
        const uint32_t c = uint32_t(w);
        if ((K(cell_key[c]) & cmask) == ckey[k]) {
          f[k] = int32_t(c);
          break;
        }
        h = (h + 1) & tmask;
        w = table[h];
      }
    }
  }
  // steps (2) and (3) for four columns at a time (half the keys live at once)
#pragma unroll
  for (int g = 0; g < 2; ++g) {
    // (2) the keys of each column's first three cells
    K kk[4][3];
#pragma unroll
    for (int j = 0; j < 4; ++j)
#pragma unroll
      for (int q = 0; q < 3; ++q) {
        const int k = 4 * g + j;
        const uint32_t c = uint32_t(f[k]) + q;
        kk[j][q] = (f[k] >= 0 && c < u_count) ? K(cell_key[c]) : none;
      }
    // the cells [c, last] of each window
    uint32_t c0[4], c1[4];
    bool has[4];
#pragma unroll
    for (int j = 0; j < 4; ++j) {
      const int k = 4 * g + j;
      has[j] = false;
      c0[j] = c1[j] = 0;
      if (f[k] < 0) continue;
      const K lo_key = ckey[k] | zlo, hi_key = ckey[k] | zhi;
      uint32_t c = uint32_t(f[k]);
      K key0 = kk[j][0], key1 = kk[j][1], key2 = kk[j][2];
      if (key0 < lo_key) {  // the column reaches below the window: gallop to it
        uint32_t step = 1;
        while (c + step < u_count && K(cell_key[c + step]) < lo_key) {
          c += step;
          step <<= 1;
        }
        uint32_t hi = c + step < u_count ? c + step : u_count;
        while (hi - c > 1) {
          const uint32_t mid = c + ((hi - c) >> 1);
          if (K(cell_key[mid]) < lo_key) c = mid;
          else hi = mid;
        }
        c = hi;
        key0 = c < u_count ? K(cell_key[c]) : none;
        key1 = c + 1 < u_count ? K(cell_key[c + 1]) : none;
        key2 = c + 2 < u_count ? K(cell_key[c + 2]) : none;
      }
      if (c < u_count && key0 <= hi_key) {
        uint32_t last = c;
        if (c + 1 < u_count && key1 <= hi_key) {
          last = c + 1;
          if (c + 2 < u_count && key2 <= hi_key) last = c + 2;
        }
        has[j] = true;
        c0[j] = c;
        c1[j] = last + 1;
      }
    }
    // (3) the cell starts that bound each range
#pragma unroll
    for (int j = 0; j < 4; ++j) {
      const int k = 4 * g + j;
      const int col = k < 4 ? k : k + 1;
      out[col] = has[j] ? make_uint2(cell_start[c0[j]], cell_start[c1[j]]) : make_uint2(0, 0);
    }
  }
}

// For every occupied cell and each of the 3x3 neighbouring columns, the range
// of cell-sorted points in cells (cx+dx, cy+dy, cz-1 .. cz+1).  Those (at
// most three) cells are consecutive in key order, so each column is one
// contiguous range: 9 ranges cover the 27-cell neighbourhood.  One thread per
// cell: the key is unpacked once; the centre column holds the cell itself
// (its z neighbours are its key-order neighbours).  The other eight columns
// are resolved in rounds of independent loads, all eight columns at once:
// (1) their column-table slots, (2) the keys of each column's first three
// cells, (3) the two cell starts that bound each range.  A column whose first
// cell lies below the window (a column with cells under cz - 1) is searched
// by galloping from its first cell instead; a window holds at most three
// cells, so three keys from the first cell in the window decide its end.
// The kernel is bound by its integer arithmetic, so keys that fit 31 bits
// with their cloud bits (one scan at a 0.5 m radius: ~24 bits) are handled in
// 32-bit arithmetic, the rest in 64-bit.
__global__ void __launch_bounds__(256, 3) k_ranges(Control *ctl, const uint64_t *cell_key,
                                                const uint32_t *cell_start, const uint64_t *table,
                                                uint32_t log2cap, uint2 *ranges, Batch bt) {
  if (ld_relaxed_u32(&ctl->status)) return;
  const uint32_t u_count = uint32_t(ctl->n_cells);  // < 2^30 (the look-back counters)
  const uint32_t epoch = ctl->epoch + EP_CELLS;
  const uint32_t lb = ctl->ckey_bits;
  const uint32_t tmask = (1u << log2cap) - 1u;
  const bool dense = ctl->dense_cols != 0;
  const bool narrow = lb + ctl->cloud_bits <= 31;
  // Batches of 32 consecutive cells per warp: a fixed stride over the warps,
  // or, on large grids, claimed from the chain's counter, since cells differ in
  // cost (tall columns gallop) and a fixed share leaves warps idle at the end
  // (C3's 28.8M cells: 2.29 -> 2.16 ms; at 417k cells the claims cost 3%).
  const uint32_t lane = threadIdx.x & 31u;
  const uint32_t batches = (u_count + 31) / 32;
  const bool claimed = u_count > (1u << 22);
  const uint32_t warps = (gridDim.x * blockDim.x) >> 5;
  auto next = [&](uint32_t b) {
    if (!claimed) return b + warps;
    uint32_t c = 0;
    if (lane == 0) c = atomicAdd(&ctl->work[WK_RANGES], 1u);
    return __shfl_sync(FULL_MASK, c, 0);
  };
  const uint32_t first = claimed ? next(0) : (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  if (narrow) {
    for (uint32_t b = first; b < batches; b = next(b)) {
      const uint32_t u = b * 32 + lane;
      if (u < u_count)
        ranges_of_cell<uint32_t>(u, u_count, cell_key, cell_start, table, log2cap, tmask, dense,
                                 epoch, lb, bt, ranges);
    }
  } else {
    for (uint32_t b = first; b < batches; b = next(b)) {
      const uint32_t u = b * 32 + lane;
      if (u < u_count)
        ranges_of_cell<uint64_t>(u, u_count, cell_key, cell_start, table, log2cap, tmask, dense,
                                 epoch, lb, bt, ranges);
    }
  }
}

constexpr int NM_THREADS = 256;
constexpr int NM_FLUSH = 32;  // f32 partial moments are folded into FP64 every NM_FLUSH candidates
constexpr double NM_REFINE_GAP = 0.05;  // (l1 - l0) / trace below this -> FP64 moments
constexpr double NM_REFINE_MEAN = 0.875;  // |E[d]|^2 / E|d|^2 above this -> FP64 moments
constexpr uint32_t NM_STAGE = 256;  // candidate records staged per warp (4 KB), staged gather

// Staged gather: one mbarrier per warp, completed by the bulk copies' bytes.
__device__ __forceinline__ uint32_t nm_smem_addr(const void *p) {
  return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}
__device__ __forceinline__ void nm_bar_init(uint64_t *bar) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(nm_smem_addr(bar)) : "memory");
}
__device__ __forceinline__ void nm_bar_expect(uint64_t *bar, uint32_t bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(nm_smem_addr(bar)),
               "r"(bytes) : "memory");
}
__device__ __forceinline__ bool nm_bar_try(uint64_t *bar, uint32_t parity) {
  uint32_t ok;
  asm volatile("{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n"
               " selp.u32 %0, 1, 0, p;\n}\n" : "=r"(ok) : "r"(nm_smem_addr(bar)), "r"(parity) : "memory");
  return ok != 0;
}
// Non-multicast bulk copy global -> this CTA's shared memory (16-byte aligned
// addresses, a multiple of 16 bytes).
__device__ __forceinline__ void nm_bulk(void *dst, const void *src, uint32_t bytes, uint64_t *bar) {
  asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];"
               ::"r"(nm_smem_addr(dst)), "l"(src), "r"(bytes), "r"(nm_smem_addr(bar)) : "memory");
}
__device__ const uint2 nm_no_ranges[9] = {};  // the walk of a lane whose cell is out of range

// The neighbour walks of k_normals.
constexpr int WALK_L1 = 0;      // range by range through L1, two candidates per step
constexpr int WALK_STAGED = 1;  // range by range from shared memory filled by bulk copies
constexpr int WALK_PACKED = 2;  // range by range through L1, packed f32x2 arithmetic

// Packed f32x2 arithmetic (sm_100): two IEEE round-to-nearest f32 operations
// per instruction, component by component -- the same results as
// __fsub_rn / __fmul_rn / __fadd_rn / fmaf on each half.
__device__ __forceinline__ uint64_t f2_pack(float lo, float hi) {
  uint64_t r;
  asm("mov.b64 %0, {%1, %2};" : "=l"(r) : "f"(lo), "f"(hi));
  return r;
}
__device__ __forceinline__ void f2_unpack(uint64_t v, float &lo, float &hi) {
  asm("mov.b64 {%0, %1}, %2;" : "=f"(lo), "=f"(hi) : "l"(v));
}
__device__ __forceinline__ uint64_t f2_sub(uint64_t a, uint64_t b) {
  uint64_t r;
  asm("sub.rn.f32x2 %0, %1, %2;" : "=l"(r) : "l"(a), "l"(b));
  return r;
}
__device__ __forceinline__ uint64_t f2_mul(uint64_t a, uint64_t b) {
  uint64_t r;
  asm("mul.rn.f32x2 %0, %1, %2;" : "=l"(r) : "l"(a), "l"(b));
  return r;
}
__device__ __forceinline__ uint64_t f2_add(uint64_t a, uint64_t b) {
  uint64_t r;
  asm("add.rn.f32x2 %0, %1, %2;" : "=l"(r) : "l"(a), "l"(b));
  return r;
}
__device__ __forceinline__ uint64_t f2_fma(uint64_t a, uint64_t b, uint64_t c) {
  uint64_t r;
  asm("fma.rn.f32x2 %0, %1, %2, %3;" : "=l"(r) : "l"(a), "l"(b), "l"(c));
  return r;
}

// Covariance from moments about the query (S: sx sy sz sxx syy szz sxy sxz syz
// over n points) and its smallest eigenpair, FP64.
__device__ __forceinline__ Eig3 eig_from_moments(const double (&S)[9], uint32_t n) {
  const double inv = __drcp_rn(double(n));  // the correctly rounded 1 / n
  const double mx = S[0] * inv, my = S[1] * inv, mz = S[2] * inv;
  const double cxx = S[3] * inv - mx * mx, cyy = S[4] * inv - my * my;
  const double czz = S[5] * inv - mz * mz, cxy = S[6] * inv - mx * my;
  const double cxz = S[7] * inv - mx * mz, cyz = S[8] * inv - my * mz;
  return smallest_eigenpair(cxx, cyy, czz, cxy, cxz, cyz);
}

// The same covariance (assembled in FP64), solved in FP32: the closed form
// carries ~6e-8 of the trace in absolute error, so wherever the gap l1 - l0
// is at least NM_REFINE_GAP of the trace the eigenvector is within ~1e-6 rad.
// Smaller gaps go to the FP64 path.
__device__ __forceinline__ Eig3 eig_from_moments_f32(const double (&S)[9], uint32_t n) {
  const double inv = __drcp_rn(double(n));  // the correctly rounded 1 / n
  const double mx = S[0] * inv, my = S[1] * inv, mz = S[2] * inv;
  const double cxx = S[3] * inv - mx * mx, cyy = S[4] * inv - my * my;
  const double czz = S[5] * inv - mz * mz, cxy = S[6] * inv - mx * my;
  const double cxz = S[7] * inv - mx * mz, cyz = S[8] * inv - my * mz;
  return smallest_eigenpair_t<float>(float(cxx), float(cyy), float(czz), float(cxy), float(cxz),
                                     float(cyz));
}

// The same neighbour set (the f32 predicate), with every moment term formed
// and summed in FP64 -- used for near-degenerate covariances only.
__device__ __noinline__ void moments_fp64(const float4 *pts, const uint2 *rg, float4 qp, float r2,
                                          double (&S)[9]) {
#pragma unroll
  for (int k = 0; k < 9; ++k) S[k] = 0.0;
  for (int r = 0; r < 9; ++r) {
    const uint2 range = rg[r];
    for (uint32_t j = range.x; j < range.y; ++j) {
      const float4 c = __ldg(pts + j);
      const float fx = __fsub_rn(c.x, qp.x), fy = __fsub_rn(c.y, qp.y), fz = __fsub_rn(c.z, qp.z);
      const float d2 = __fadd_rn(__fadd_rn(__fmul_rn(fx, fx), __fmul_rn(fy, fy)), __fmul_rn(fz, fz));
      if (!(d2 <= r2)) continue;
      const double dx = double(c.x) - double(qp.x);
      const double dy = double(c.y) - double(qp.y);
      const double dz = double(c.z) - double(qp.z);
      S[0] += dx;
      S[1] += dy;
      S[2] += dz;
      S[3] += dx * dx;
      S[4] += dy * dy;
      S[5] += dz * dz;
      S[6] += dx * dy;
      S[7] += dx * dz;
      S[8] += dy * dz;
    }
  }
}

// Radius normals.  One warp per 32 consecutive cell-sorted points, one query
// per lane; the persistent warps claim these batches from a counter.  Each lane walks the 9 column ranges of its own cell (the 27-cell
// neighbourhood) and reads candidates through L1: lanes of the same cell read
// the same record at the same step, so loads are broadcasts, and the
// eigensolve runs on all 32 lanes.
//
// The query is a candidate of itself with d = p - q = 0 exactly, so it is
// counted and removed afterwards (hits - 1) instead of being compared by
// index in the loop; duplicates of the query stay neighbours, as in the
// reference (normal.rs:381-386).
//
// Moments are taken about the query point (d = p - q, the predicate's own
// differences): count, sum d, sum d d^T, accumulated in f32 for NM_FLUSH
// candidates and then folded into FP64.  C = S2/n - (S1/n)(S1/n)^T is
// assembled in FP64 and solved in FP32 (closed form); when the gap l1 - l0 is
// under NM_REFINE_GAP of the trace, the point's moments are recomputed with
// FP64 products over the same neighbour set and the solve is repeated in FP64.
// CountShell: the chain reports shell points (some cloud asked for it); the
// check costs a few instructions per candidate, so chains that do not want
// it run the variant without it.
// PlaneCov: instead of normal and curvature, write the GICP plane-regularised
// covariance of each point (crates/spatialrust-gpu/src/kernels/
// covariances_grid.rs:87-206): the neighbourhood covariance with its
// eigenvalues replaced by (eps, 1, 1).  With the orthonormal eigenbasis
// (n, a, b) that is eps n n^T + a a^T + b b^T = I + (eps - 1) n n^T, so only
// the smallest eigenvector is needed.  Six floats per point in cov
// ([c00, c11, c22, c01, c02, c12], the GpuCovariance layout); fewer than 3
// points in the (self-inclusive) neighbourhood give (eps, eps, eps, 0, 0, 0).
//
// Staged: the warp's candidate records are brought into shared memory by
// non-multicast bulk copies (cp.async.bulk on a per-warp mbarrier) before the
// walk, one copy per x-strip of the 3x3 column block -- for each x offset, the
// span over the warp's lanes of their three column ranges, which lie close
// together in the cell-sorted records.  A strip that does not fit the warp's
// NM_STAGE records is read from global memory as in the plain walk.  The plain
// walk reads through L1 instead; which one a context runs is a tuning choice
// (srcu_set_neighbor_staging).
template <bool CountShell, bool PlaneCov = false, int Walk = WALK_L1>
__global__ void __launch_bounds__(NM_THREADS, 4) k_normals(Control *ctl, const float4 *pts,
                                                           const uint32_t *pt_cell,
                                                           const uint2 *ranges,
                                                           const uint64_t *cell_key, Batch bt,
                                                           const unsigned long long *count_dev,
                                                           float *nx, float *ny, float *nz,
                                                           float *curv, uint32_t *counts,
                                                           float *cov, float cov_eps) {
  if (ld_relaxed_u32(&ctl->status)) return;
  const uint32_t lane = threadIdx.x & 31u;
  const uint32_t n = uint32_t(count_dev ? *count_dev : ctl->n_points);
  const uint64_t u_count = ctl->n_cells;
  const uint32_t lb = ctl->ckey_bits;
  const uint32_t batches = (n + 31) / 32;
  unsigned long long n_valid = 0, n_invalid = 0, n_shell = 0, n_fp64 = 0;
  float4 *sbuf = nullptr;  // this warp's staging buffer (Staged)
  uint64_t *sbar = nullptr;
  uint32_t phase = 0;
  bool timed_out = false;
  constexpr bool Staged = Walk == WALK_STAGED;
  if constexpr (Staged) {
    __shared__ float4 nm_stage[(NM_THREADS / 32) * NM_STAGE];
    __shared__ __align__(8) uint64_t nm_bar[NM_THREADS / 32];
    sbuf = nm_stage + (threadIdx.x >> 5) * NM_STAGE;
    sbar = &nm_bar[threadIdx.x >> 5];
    if (lane == 0) nm_bar_init(sbar);
    __syncwarp();
  }

  // Each warp claims its next batch of 32 queries from the chain's counter:
  // batches differ in cost (dense and sparse parts of a cloud), so claiming
  // keeps every warp busy to the end instead of a fixed share each.
  auto claim = [&]() {
    uint32_t c = 0;
    if (lane == 0) c = atomicAdd(&ctl->work[WK_NORMALS], 1u);
    return __shfl_sync(FULL_MASK, c, 0);
  };
  for (uint32_t b = claim(); b < batches; b = claim()) {
    const uint32_t i = b * 32 + lane;
    const bool active = i < n;
    const uint32_t ii = active ? i : n - 1;
    const float4 qp = pts[ii];
    const uint32_t u = pt_cell[ii];
    bool bad = false;
    if (u >= u_count) {  // cannot happen for a consistent cell table
      atomicOr(&ctl->status, ST_INTERNAL);
      if constexpr (Staged) {
        bad = true;  // the lane stays for the warp's collectives and walks nothing
      } else {
        continue;
      }
    }
    uint32_t cb = 0;  // the query's cloud
    if (!bad && bt.clouds > 1 && lb < 64) cb = uint32_t(cell_key[u] >> lb);
    if (cb >= bt.clouds) cb = 0;
    const NormalParamsDev prm = bt.nparams[cb];
    const float r2 = bt.cplans[cb].r2;
    const float shell_tol = bt.cplans[cb].shell_tol;
    const uint2 *rg = bad ? nm_no_ranges : ranges + size_t(u) * 9;
    float hits = 0.f;
    uint32_t shell = 0;
    double S[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0};  // sx sy sz sxx syy szz sxy sxz syz
    float F[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0};
    uint32_t since = 0;
    // One candidate: the reference's f32 predicate ((dx^2 + dy^2) + dz^2 <= r^2,
    // kdtree.rs:544-549) and the f32 partial moments of the hits.
    auto visit = [&](const float4 c) {
      const float dx = __fsub_rn(c.x, qp.x);
      const float dy = __fsub_rn(c.y, qp.y);
      const float dz = __fsub_rn(c.z, qp.z);
      const float xx = __fmul_rn(dx, dx), yy = __fmul_rn(dy, dy), zz = __fmul_rn(dz, dz);
      const float d2 = __fadd_rn(__fadd_rn(xx, yy), zz);
      if (d2 <= r2) {
        hits += 1.f;
        F[0] += dx;
        F[1] += dy;
        F[2] += dz;
        F[3] += xx;
        F[4] += yy;
        F[5] += zz;
        F[6] = fmaf(dx, dy, F[6]);
        F[7] = fmaf(dx, dz, F[7]);
        F[8] = fmaf(dy, dz, F[8]);
      }
      if (CountShell && prm.count_shell && d2 != 0.f && fabsf(__fsub_rn(d2, r2)) <= shell_tol)
        shell = 1;
    };
    auto flush = [&]() {
#pragma unroll
      for (int k = 0; k < 9; ++k) {
        S[k] += double(F[k]);
        F[k] = 0.f;
      }
    };
    if constexpr (Staged) {
      // Stage the warp's x-strips; shared index = record index + delta[d].
      int32_t delta[3];
      uint32_t staged = 0;
      {
        uint32_t lo[3], len[3], total = 0;
#pragma unroll
        for (int d = 0; d < 3; ++d) {
          uint32_t a = 0xffffffffu, z = 0;
#pragma unroll
          for (int k = 0; k < 3; ++k) {
            const uint2 g = rg[3 * d + k];
            if (g.y > g.x) {
              a = min(a, g.x);
              z = max(z, g.y);
            }
          }
          a = __reduce_min_sync(FULL_MASK, a);
          z = __reduce_max_sync(FULL_MASK, z);
          lo[d] = a;
          len[d] = z > a ? z - a : 0;
          delta[d] = int32_t(total) - int32_t(a);
          if (len[d] > 0 && total + len[d] <= NM_STAGE) {
            staged |= 1u << d;
            total += len[d];
          }
        }
        if (total > 0 && !timed_out) {
          __syncwarp();  // every lane is done with the buffer's previous contents
          if (lane == 0) {
            asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
            nm_bar_expect(sbar, total * 16u);
#pragma unroll
            for (int d = 0; d < 3; ++d)
              if ((staged >> d) & 1u)
                nm_bulk(sbuf + (int32_t(lo[d]) + delta[d]), pts + lo[d], len[d] * 16u, sbar);
          }
          uint32_t spins = 0;
          bool gave_up = false;
          while (!nm_bar_try(sbar, phase)) {
            if (++spins > SPIN_LIMIT) {
              gave_up = true;
              break;
            }
          }
          if (__any_sync(FULL_MASK, gave_up)) {
            timed_out = true;  // read everything from global memory from now on
            if (lane == 0) atomicOr(&ctl->status, ST_TIMEOUT);
          } else {
            phase ^= 1u;
          }
        }
        if (timed_out) staged = 0;
      }
      auto walk = [&](auto load, uint32_t a, uint32_t z) {
        uint32_t j = a;
        for (; j + 2 <= z; j += 2) {
          const float4 c0 = load(j);
          const float4 c1 = load(j + 1);
          visit(c0);
          visit(c1);
          since += 2;
          if (since >= NM_FLUSH) {
            since = 0;
            flush();
          }
        }
        if (j < z) {
          visit(load(j));
          if (++since >= NM_FLUSH) {
            since = 0;
            flush();
          }
        }
      };
      uint2 next = rg[0];
#pragma unroll 1
      for (int r = 0; r < 9; ++r) {
        const uint2 range = next;
        if (r < 8) next = rg[r + 1];
        const int d = r / 3;
        if ((staged >> d) & 1u) {
          const float4 *sp = sbuf + delta[d];
          walk([&](uint32_t j) { return sp[j]; }, range.x, range.y);
        } else {
          walk([&](uint32_t j) { return __ldg(pts + j); }, range.x, range.y);
        }
      }
    } else if constexpr (Walk == WALK_PACKED) {
      // The L1 walk's candidate order and flush points, with the predicate and
      // the moments in packed f32x2 arithmetic: the same IEEE operation on each
      // half, so every result is bit-identical to WALK_L1's.
      const uint64_t qxy = f2_pack(qp.x, qp.y);
      uint64_t a01 = 0, a34 = 0, a78 = 0;  // (sx, sy), (sxx, syy), (sxz, syz)
      float a2 = 0.f, a5 = 0.f, a6 = 0.f;  // sz, szz, sxy
      auto pvisit = [&](const float4 c) {
        // the reference predicate ((dx^2 + dy^2) + dz^2 <= r^2, kdtree.rs:544-549)
        const uint64_t dxy = f2_sub(f2_pack(c.x, c.y), qxy);
        const uint64_t pxy = f2_mul(dxy, dxy);
        float dx, dy, xx, yy;
        f2_unpack(dxy, dx, dy);
        f2_unpack(pxy, xx, yy);
        const float dz = __fsub_rn(c.z, qp.z);
        const float zz = __fmul_rn(dz, dz);
        const float d2 = __fadd_rn(__fadd_rn(xx, yy), zz);
        if (d2 <= r2) {
          hits += 1.f;
          a01 = f2_add(a01, dxy);
          a34 = f2_add(a34, pxy);
          a78 = f2_fma(dxy, f2_pack(dz, dz), a78);
          a2 += dz;
          a5 += zz;
          a6 = fmaf(dx, dy, a6);
        }
        if (CountShell && prm.count_shell && d2 != 0.f && fabsf(__fsub_rn(d2, r2)) <= shell_tol)
          shell = 1;
      };
      auto pflush = [&]() {
        float v0, v1, v3, v4, v7, v8;
        f2_unpack(a01, v0, v1);
        f2_unpack(a34, v3, v4);
        f2_unpack(a78, v7, v8);
        S[0] += double(v0);
        S[1] += double(v1);
        S[2] += double(a2);
        S[3] += double(v3);
        S[4] += double(v4);
        S[5] += double(a5);
        S[6] += double(a6);
        S[7] += double(v7);
        S[8] += double(v8);
        a01 = a34 = a78 = 0;
        a2 = a5 = a6 = 0.f;
      };
      uint2 next = rg[0];
#pragma unroll 1
      for (int r = 0; r < 9; ++r) {
        const uint2 range = next;
        if (r < 8) next = rg[r + 1];  // the next column's range loads under this one
        uint32_t j = range.x;
        for (; j + 2 <= range.y; j += 2) {  // two independent candidate loads per step
          const float4 c0 = __ldg(pts + j);
          const float4 c1 = __ldg(pts + j + 1);
          pvisit(c0);
          pvisit(c1);
          since += 2;
          if (since >= NM_FLUSH) {
            since = 0;
            pflush();
          }
        }
        if (j < range.y) {
          pvisit(__ldg(pts + j));
          if (++since >= NM_FLUSH) {
            since = 0;
            pflush();
          }
        }
      }
      pflush();
    } else {
      uint2 next = rg[0];
#pragma unroll 1
      for (int r = 0; r < 9; ++r) {
        const uint2 range = next;
        if (r < 8) next = rg[r + 1];  // the next column's range loads under this one
        uint32_t j = range.x;
        // two independent candidate loads in flight per step
        for (; j + 2 <= range.y; j += 2) {
          const float4 c0 = __ldg(pts + j);
          const float4 c1 = __ldg(pts + j + 1);
          visit(c0);
          visit(c1);
          since += 2;
          if (since >= NM_FLUSH) {
            since = 0;
            flush();
          }
        }
        if (j < range.y) {
          visit(__ldg(pts + j));
          if (++since >= NM_FLUSH) {
            since = 0;
            flush();
          }
        }
      }
    }
#pragma unroll
    for (int k = 0; k < 9; ++k) S[k] += double(F[k]);
    if (!active || bad) continue;
    // hits includes the query itself exactly once when it is finite.
    const bool finite = isfinite(qp.x) && isfinite(qp.y) && isfinite(qp.z);
    const uint32_t h = uint32_t(hits);
    const uint32_t cnt = (finite && h > 0) ? h - 1 : 0;
    const uint32_t n_eff = prm.include_self ? cnt + (finite ? 1 : 0) : cnt;
    const bool valid = prm.include_self ? (n_eff >= 3) : (cnt >= prm.min_neighbors && cnt > 0);
    float ox, oy, oz, oc;
    if (valid) {
      // The f32 moments carry ~1e-7 of E|d|^2 in rounding (d = p - q, about
      // the query), and the covariance E[d d^T] - E[d] E[d]^T inherits it
      // whole: where the neighbours' mean lies far from the query against
      // their spread (|E[d]|^2 > NM_REFINE_MEAN E|d|^2, so the trace is under
      // an eighth of E|d|^2) that is too much of the trace for the curvature
      // and, over a small gap, for the normal, so the moments are recomputed
      // with FP64 products (same neighbour set) and solved again in FP32.
      // The FP32 solve carries ~6e-8 of the trace; where the gap to the
      // second eigenvalue is under NM_REFINE_GAP of the trace the normal can
      // tilt by more than 1e-5 rad, and the point is solved in FP64 from FP64
      // moments.  One call site for the FP64 walk keeps the common path lean.
      const double inv_n = __drcp_rn(double(n_eff));
      const double e2 = (S[3] + S[4] + S[5]) * inv_n;
      const double m2 = (S[0] * S[0] + S[1] * S[1] + S[2] * S[2]) * (inv_n * inv_n);
      const bool exact_moments = !(m2 <= NM_REFINE_MEAN * e2);
      Eig3 e = eig_from_moments_f32(S, n_eff);
      const bool small_gap = !(e.l1 - e.l0 >= NM_REFINE_GAP * (e.l0 + e.l1 + e.l2));
      if (exact_moments || small_gap) {
        moments_fp64(pts, rg, qp, r2, S);
        if (small_gap) {
          e = eig_from_moments(S, n_eff);
          ++n_fp64;
        } else {
          e = eig_from_moments_f32(S, n_eff);
        }
      }
      // Orientation and normalisation in f32, as the reference computes them
      // (orient_normal_towards_viewpoint, normal.rs:408-421, with Vec3::dot
      // and Vec3::normalize, vec.rs:66-100): the unit eigenvector rounded to
      // f32 moves by ~1e-7 rad at most, and the sign test matches the
      // reference's own f32 test.
      float v0 = float(e.v[0]), v1 = float(e.v[1]), v2 = float(e.v[2]);
      if (!PlaneCov && prm.has_viewpoint) {
        const float wx = __fsub_rn(prm.vp[0], qp.x);
        const float wy = __fsub_rn(prm.vp[1], qp.y);
        const float wz = __fsub_rn(prm.vp[2], qp.z);
        const float dot = __fadd_rn(__fadd_rn(__fmul_rn(v0, wx), __fmul_rn(v1, wy)), __fmul_rn(v2, wz));
        if (dot < 0.0f) {
          v0 = -v0;
          v1 = -v1;
          v2 = -v2;
        }
      }
      const float len =
          sqrtf(__fadd_rn(__fadd_rn(__fmul_rn(v0, v0), __fmul_rn(v1, v1)), __fmul_rn(v2, v2)));
      ox = len != 0.0f ? v0 / len : v0;
      oy = len != 0.0f ? v1 / len : v1;
      oz = len != 0.0f ? v2 / len : v2;
      const float sum = float(e.l0 + e.l1 + e.l2);
      oc = sum > 0.0f ? float(e.l0) / sum : 0.0f;
      ++n_valid;
    } else {
      // include_self: (0, 0, 1) (normals_grid.rs:129-132), turned toward the
      // viewpoint as GpuNormalEstimator turns every normal (normal_gpu.rs:
      // 63-70): the f32 dot with vp - q is fl(vp.z - q.z), negative exactly
      // when vp.z < q.z.
      const float nanv = __int_as_float(0x7fc00000);
      ox = prm.include_self ? 0.0f : nanv;
      oy = prm.include_self ? 0.0f : nanv;
      oz = prm.include_self ? ((prm.has_viewpoint && prm.vp[2] < qp.z) ? -1.0f : 1.0f) : nanv;
      oc = 0.0f;
      ++n_invalid;
    }
    n_shell += shell;
    const uint32_t qidx = __float_as_uint(qp.w);
    if (qidx >= n) {  // cannot happen: records carry indices < n
      atomicOr(&ctl->status, ST_INTERNAL);
      continue;
    }
    if constexpr (PlaneCov) {
      float *o = cov + size_t(qidx) * 6;
      if (valid) {
        // (ox, oy, oz) is the unit normal; I + (eps - 1) n n^T
        const float s = cov_eps - 1.0f;
        o[0] = fmaf(s * ox, ox, 1.0f);
        o[1] = fmaf(s * oy, oy, 1.0f);
        o[2] = fmaf(s * oz, oz, 1.0f);
        o[3] = s * ox * oy;
        o[4] = s * ox * oz;
        o[5] = s * oy * oz;
      } else {
        o[0] = cov_eps;
        o[1] = cov_eps;
        o[2] = cov_eps;
        o[3] = 0.0f;
        o[4] = 0.0f;
        o[5] = 0.0f;
      }
      if (counts) counts[qidx] = n_eff;
      continue;
    }
    nx[qidx] = ox;
    ny[qidx] = oy;
    nz[qidx] = oz;
    curv[qidx] = oc;
    if (counts) counts[qidx] = prm.include_self ? n_eff : cnt;
  }
  if constexpr (Staged) {
    if (timed_out) {  // a copy that was given up on may still land: wait for it, bounded
      uint32_t spins = 0;
      while (!nm_bar_try(sbar, phase) && ++spins <= SPIN_LIMIT) {
      }
    }
  }
  // one atomic per warp for the counters
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    n_valid += __shfl_xor_sync(FULL_MASK, n_valid, o);
    n_invalid += __shfl_xor_sync(FULL_MASK, n_invalid, o);
    n_shell += __shfl_xor_sync(FULL_MASK, n_shell, o);
    n_fp64 += __shfl_xor_sync(FULL_MASK, n_fp64, o);
  }
  if (lane == 0) {
    if (n_valid) atomicAdd(&ctl->ncount.valid, n_valid);
    if (n_invalid) atomicAdd(&ctl->ncount.invalid, n_invalid);
    if (n_shell) atomicAdd(&ctl->ncount.shell, n_shell);
    if (n_fp64) atomicAdd(&ctl->ncount.fp64, n_fp64);
  }
}

}  // namespace srcu
