// plans.cuh -- device control block, voxel-key and cell-key plans.
//
// Voxel keys reproduce the reference's integer keys bit for bit:
//   explicit origin : ix = floor((x - ox) * inv_leaf) as i64  (voxel.rs:1088-1093)
//   origin = min    : ix = ((x - ox) * inv_leaf) as i64        (voxel.rs:1095-1107)
// computed with round-to-nearest f32 subtract and multiply (no FMA), with
// Rust's saturating cast (NaN -> 0).  The three per-axis keys are packed
// order-preservingly into one u64: (ix - kmin_x) in the high bits, then y,
// then z, so ascending u64 order is the reference's lexicographic
// (ix, iy, iz) order (voxel.rs:522-524).
#pragma once

#include <cstddef>

#include "common.cuh"

namespace srcu {

constexpr int RADIX_BITS = 8;        // the sort's narrow digit
constexpr int RADIX_BINS = 256;
constexpr int WIDE_RADIX_BITS = 9;   // the wide digit of the 512-thread sort shapes
constexpr int MAX_RADIX_BINS = 1 << WIDE_RADIX_BITS;
constexpr int MAX_DIGITS = 8;        // 64-bit keys, at either width
constexpr int MAX_COLS = 12;   // x, y, z + up to 9 attribute columns

// Bounds over finite coordinates (ordered-uint encoded), with flags for
// NaN / infinite values per axis.
struct Bounds {
  uint32_t mn[3];
  uint32_t mx[3];
  uint32_t flags;  // bit a: NaN seen on axis a; bit 3+a: +-inf seen on axis a
  uint32_t pad;
};

struct VoxelPlan {
  float origin[3];
  float inv_leaf;
  int32_t floor_mode;  // 1: explicit origin (floor), 0: min-corner origin (trunc)
  uint32_t bits[3];
  uint32_t shift_x, shift_y;
  uint32_t total_bits;
  uint32_t num_digits;
  int64_t kmin[3];
  uint32_t valid;
  uint32_t pad;
};

// Uniform grid for the radius search.  Cell size h >= r (1 + 1e-5) so any two
// points within r of each other (under the f32 predicate) lie in the same or
// adjacent cells; cells are computed in FP64 from the f32 coordinates.
struct CellPlan {
  double origin[3];
  double inv_h;
  double h;
  uint32_t dims[3];
  uint32_t bits[3];
  uint32_t shift_x, shift_y;
  uint32_t total_bits;
  uint32_t num_digits;
  float r2;          // fl(r * r), the reference predicate bound (kdtree.rs:350-357)
  float shell_tol;   // 1e-6 * r2
  uint32_t valid;
  uint32_t pad;
  uint64_t col_base; // first slot of this cloud's columns in the dense column table
};

// Per-cloud parameters on the device (srcu_voxel_params / srcu_normal_params).
// Per-voxel emission (srcu_voxel_params mode / attribute_policy).
constexpr int32_t AGG_FAST = 0;            // Centroid + Average: (sum * (1/count)) for every field
constexpr int32_t AGG_CENTROID_FIRST = 1;  // positions (sum / count), other fields first point
constexpr int32_t AGG_FIRST = 2;           // ApproximateFirst: every field from the first point

struct VoxelParamsDev {
  float leaf;
  int32_t has_origin;
  float origin[3];
  int32_t agg;  // AGG_*
};

struct NormalParamsDev {
  float radius;
  uint32_t min_neighbors;
  int32_t include_self;
  int32_t has_viewpoint;
  int32_t count_shell;  // report points with a candidate on the radius shell
  float vp[3];
};

// Many clouds in one chain.  Points of cloud b are [offsets[b], offsets[b+1])
// of the concatenated columns; its id sits above the per-cloud key bits of
// every voxel and cell key, so one sort orders all clouds at once.  A single
// cloud is the case clouds == 1.
struct Batch {
  uint32_t clouds;
  const uint32_t *offsets;         // clouds + 1 point offsets
  Bounds *bounds;                  // clouds
  VoxelPlan *vplans;               // clouds
  CellPlan *cplans;                // clouds
  const VoxelParamsDev *vparams;   // clouds
  const NormalParamsDev *nparams;  // clouds
  uint32_t *voxel_offsets;         // clouds + 1, voxel ranges of each cloud
};

// Cloud owning concatenated point i: the largest b with offsets[b] <= i.
__device__ __forceinline__ uint32_t cloud_of(const Batch &bt, uint32_t i) {
  uint32_t lo = 0, hi = bt.clouds;  // invariant: offsets[lo] <= i < offsets[hi]
  while (hi - lo > 1) {
    const uint32_t mid = (lo + hi) >> 1;
    if (__ldg(bt.offsets + mid) <= i) lo = mid;
    else hi = mid;
  }
  return lo;
}

__host__ __device__ __forceinline__ uint64_t with_cloud(uint64_t local_key, uint32_t cloud,
                                                        uint32_t local_bits) {
  return local_bits >= 64 ? local_key : (local_key | (uint64_t(cloud) << local_bits));
}

// State of one sort: where the result is and how it is encoded, plus the
// grid barrier of its persistent kernel.
struct SortState {
  uint32_t final_buf;  // ping-pong buffer holding the sorted items
  uint32_t passes;     // digit passes that ran (non-trivial digits)
  uint32_t packed;     // 1: items are (key << idx_bits) | index; 0: keys[] + vals[]
  uint32_t idx_bits;
  uint32_t key_bits;
  uint32_t bar_count;
  uint32_t bar_gen;
  uint32_t pad;
};

struct NormalCounters {
  unsigned long long valid;
  unsigned long long invalid;
  unsigned long long shell;
  unsigned long long fp64;
};

// One control block per context, zeroed (except the epoch) by k_begin at the
// start of every chain so the whole chain can be replayed from a CUDA graph.
struct Control {
  uint32_t epoch;   // bumped by EPOCHS_PER_RUN per chain; look-back words carry it
  uint32_t status;  // StatusBits
  unsigned long long n_points;  // input points of this chain
  unsigned long long n_voxels;  // V
  unsigned long long n_cells;   // U (occupied radius-grid cells)
  uint32_t work[64];            // per-kernel dynamic tile counters
  uint32_t clouds;              // B
  uint32_t cloud_bits;          // bits of the cloud id above the per-cloud key bits
  uint32_t vkey_bits;           // per-cloud voxel key bits (max over clouds)
  uint32_t ckey_bits;           // per-cloud cell key bits (max over clouds)
  NormalCounters ncount;
  SortState vsort;  // voxel-key sort
  SortState csort;  // cell-key sort
  uint32_t hist_v[MAX_DIGITS * MAX_RADIX_BINS];  // voxel-key digit histograms
  uint32_t hist_c[MAX_DIGITS * MAX_RADIX_BINS];  // cell-key digit histograms
  unsigned long long col_total;  // sum over clouds of dims_x * dims_y
  uint32_t dense_cols;           // 1: the column table is dense (it fits the table buffer)
  uint32_t pad2;
};

constexpr uint32_t EPOCHS_PER_RUN = 64;
// Epoch offsets (within a run) of each look-back user.
constexpr uint32_t EP_VSORT = 0;     // 8 passes
constexpr uint32_t EP_VSEG = 8;
constexpr uint32_t EP_CSORT = 16;    // 8 passes
constexpr uint32_t EP_CELLS = 24;
constexpr uint32_t EP_ORDER = 32;    // first-seen order sort of the plain-xyz path, 4 passes
// Work-counter slots.
constexpr int WK_VSORT = 0;   // 8 slots
constexpr int WK_VSEG = 8;
constexpr int WK_CSORT = 16;  // 8 slots
constexpr int WK_CELLS = 24;
constexpr int WK_NORMALS = 25;
constexpr int WK_RANGES = 26;
constexpr int WK_ORDER = 32;  // 4 slots

__device__ __forceinline__ int64_t rs_sat_i64(float t) {
  if (isnan(t)) return 0;
  if (t >= 9223372036854775808.0f) return INT64_MAX;
  if (t < -9223372036854775808.0f) return INT64_MIN;
  return static_cast<int64_t>(t);
}

__device__ __forceinline__ int64_t voxel_axis_key(float p, float o, float inv, int floor_mode) {
  float t = __fmul_rn(__fsub_rn(p, o), inv);
  if (floor_mode) t = floorf(t);
  return rs_sat_i64(t);
}

__device__ __forceinline__ uint64_t voxel_pack(const VoxelPlan &pl, float x, float y, float z) {
  const int64_t kx = voxel_axis_key(x, pl.origin[0], pl.inv_leaf, pl.floor_mode);
  const int64_t ky = voxel_axis_key(y, pl.origin[1], pl.inv_leaf, pl.floor_mode);
  const int64_t kz = voxel_axis_key(z, pl.origin[2], pl.inv_leaf, pl.floor_mode);
  const uint64_t ox = uint64_t(kx) - uint64_t(pl.kmin[0]);
  const uint64_t oy = uint64_t(ky) - uint64_t(pl.kmin[1]);
  const uint64_t oz = uint64_t(kz) - uint64_t(pl.kmin[2]);
  // shift by 64 is undefined; an axis with 0 bits always has offset 0.
  const uint64_t hx = pl.shift_x >= 64 ? 0 : (ox << pl.shift_x);
  const uint64_t hy = pl.shift_y >= 64 ? 0 : (oy << pl.shift_y);
  return hx | hy | oz;
}

__host__ __device__ __forceinline__ void voxel_unpack(const VoxelPlan &pl, uint64_t key,
                                                      int64_t out[3]) {
  const uint64_t mz = pl.bits[2] >= 64 ? ~0ull : ((1ull << pl.bits[2]) - 1);
  const uint64_t my = pl.bits[1] >= 64 ? ~0ull : ((1ull << pl.bits[1]) - 1);
  const uint64_t oz = key & mz;
  const uint64_t oy = pl.shift_y >= 64 ? 0 : ((key >> pl.shift_y) & my);
  const uint64_t ox = pl.shift_x >= 64 ? 0 : (key >> pl.shift_x);
  out[0] = int64_t(ox + uint64_t(pl.kmin[0]));
  out[1] = int64_t(oy + uint64_t(pl.kmin[1]));
  out[2] = int64_t(oz + uint64_t(pl.kmin[2]));
}

__device__ __forceinline__ uint32_t cell_axis(float p, double o, double inv_h, uint32_t dim) {
  if (!isfinite(p)) return 0;  // never a neighbour: the f32 predicate is false for it
  double u = (double(p) - o) * inv_h;
  double f = floor(u);
  if (!(f > 0.0)) return 0;
  if (f >= double(dim - 1)) return dim - 1;
  return uint32_t(f);
}

__device__ __forceinline__ uint64_t cell_pack(const CellPlan &pl, float x, float y, float z) {
  const uint64_t cx = cell_axis(x, pl.origin[0], pl.inv_h, pl.dims[0]);
  const uint64_t cy = cell_axis(y, pl.origin[1], pl.inv_h, pl.dims[1]);
  const uint64_t cz = cell_axis(z, pl.origin[2], pl.inv_h, pl.dims[2]);
  return (cx << pl.shift_x) | (cy << pl.shift_y) | cz;
}

__device__ __forceinline__ void cell_unpack(const CellPlan &pl, uint64_t key, uint32_t &cx,
                                            uint32_t &cy, uint32_t &cz) {
  cz = uint32_t(key & ((1ull << pl.bits[2]) - 1));
  cy = uint32_t((key >> pl.shift_y) & ((1ull << pl.bits[1]) - 1));
  cx = uint32_t(key >> pl.shift_x);
}

__host__ __device__ __forceinline__ uint32_t bit_width_u64(uint64_t v) {
  uint32_t b = 0;
  while (v) {
    ++b;
    v >>= 1;
  }
  return b;
}

}  // namespace srcu
