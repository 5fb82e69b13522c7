/*
 * srcu_oracle.c -- TEST INFRASTRUCTURE ONLY.
 *
 * CPU restatement of SpatialRust's CPU path for the uniform-grid hot path
 * (VoxelGrid centroid downsample + radius-mode normal estimation), plus an
 * FP64 oracle for normals.  Only tests/, __graft_entry__.smoke() and the
 * cpu_baseline / --impl reference legs of bench.py may load this library; the
 * product (spatialrust_b200) never links or calls it.
 *
 * The reference is a Rust workspace and cannot be compiled in this image (no
 * cargo/rustc), so this file restates its algorithms in C.  Every function
 * cites the reference file:line it follows.  Compile with
 * -O3 -ffp-contract=off and no fast-math so f32 arithmetic rounds exactly as
 * the Rust code does (Rust never contracts a*b+c into an FMA).
 *
 * Parity pins: the restatement is checked against every known-answer test the
 * reference holds for this path (tests/test_oracle_golden.py), e.g.
 * crates/spatialrust-filtering/src/voxel.rs:1271-1364,
 * crates/spatialrust-features/src/normal.rs:650-695,
 * crates/spatialrust/tests/mvp_pipeline.rs:1-26.
 */
#include <math.h>
#include <pthread.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>
#include <unistd.h>

#define OR_OK 0
#define OR_ERR_INVALID (-1)
#define OR_ERR_NOMEM (-2)

/* ------------------------------------------------------------------------ */
/* Rust numeric-cast semantics                                              */
/* ------------------------------------------------------------------------ */

/* `f as i64` in Rust: truncate toward zero, saturate, NaN -> 0. */
static int64_t sat_f32_to_i64(float v) {
  if (isnan(v)) return 0;
  if (v >= 9223372036854775808.0f) return INT64_MAX;
  if (v < -9223372036854775808.0f) return INT64_MIN;
  return (int64_t)v;
}

/* `f as u32` in Rust: truncate toward zero, saturate at 0 and u32::MAX, NaN -> 0. */
static uint32_t sat_f32_to_u32(float v) {
  if (isnan(v) || v <= 0.0f) return 0;
  if (v >= 4294967296.0f) return UINT32_MAX;
  return (uint32_t)v;
}

/* f32::min / f32::max: NaN operands are ignored (IEEE minNum / maxNum). */
static float rs_minf(float a, float b) { return fminf(a, b); }
static float rs_maxf(float a, float b) { return fmaxf(a, b); }

/* ------------------------------------------------------------------------ */
/* Voxel grid centroid downsample                                           */
/* ------------------------------------------------------------------------ */

/* compute_bounds: crates/spatialrust-filtering/src/voxel.rs:1067-1079 */
void oracle_compute_bounds(const float *x, const float *y, const float *z, size_t n,
                           float mn[3], float mx[3]) {
  mn[0] = mx[0] = x[0];
  mn[1] = mx[1] = y[0];
  mn[2] = mx[2] = z[0];
  for (size_t i = 1; i < n; ++i) {
    mn[0] = rs_minf(mn[0], x[i]);
    mn[1] = rs_minf(mn[1], y[i]);
    mn[2] = rs_minf(mn[2], z[i]);
    mx[0] = rs_maxf(mx[0], x[i]);
    mx[1] = rs_maxf(mx[1], y[i]);
    mx[2] = rs_maxf(mx[2], z[i]);
  }
}

/* fits_u32_voxel_key: voxel.rs:1081-1086 */
static int fits_u32_voxel_key(const float mn[3], const float mx[3], float inv_leaf) {
  const float limit = (float)UINT32_MAX;
  return ((mx[0] - mn[0]) * inv_leaf) <= limit && ((mx[1] - mn[1]) * inv_leaf) <= limit &&
         ((mx[2] - mn[2]) * inv_leaf) <= limit;
}

/* voxel_key (floor, explicit origin): voxel.rs:1088-1093 */
static void voxel_key_floor(float x, float y, float z, const float o[3], float inv, int64_t k[3]) {
  k[0] = sat_f32_to_i64(floorf((x - o[0]) * inv));
  k[1] = sat_f32_to_i64(floorf((y - o[1]) * inv));
  k[2] = sat_f32_to_i64(floorf((z - o[2]) * inv));
}

/* voxel_key_nonnegative (truncation, origin = min corner): voxel.rs:1095-1107 */
static void voxel_key_trunc(float x, float y, float z, const float o[3], float inv, int64_t k[3]) {
  k[0] = sat_f32_to_i64((x - o[0]) * inv);
  k[1] = sat_f32_to_i64((y - o[1]) * inv);
  k[2] = sat_f32_to_i64((z - o[2]) * inv);
}

/* voxel_key_nonnegative_u32: voxel.rs:1109-1121 */
static void voxel_key_u32(float x, float y, float z, const float o[3], float inv, int64_t k[3]) {
  k[0] = sat_f32_to_u32((x - o[0]) * inv);
  k[1] = sat_f32_to_u32((y - o[1]) * inv);
  k[2] = sat_f32_to_u32((z - o[2]) * inv);
}

/* VoxelKeyHasher::mix: voxel.rs:22-28 (FxHash-style multiply-rotate). */
static inline uint64_t fx_mix(uint64_t h, uint64_t v) {
  h = ((h << 5) | (h >> 59)) ^ v;
  return h * 0x517cc1b727220a95ULL;
}

/* Open-addressing map from (i64,i64,i64) to a sequential cell id.  Stands in
 * for the reference's HashMap<_, _, BuildHasherDefault<VoxelKeyHasher>>; any
 * exact map yields the same cells, so only timing depends on this choice. */
typedef struct {
  int64_t *keys; /* 3 per slot */
  uint32_t *ids; /* UINT32_MAX = empty */
  size_t cap;    /* power of two */
  size_t len;
} cell_map;

static int cell_map_init(cell_map *m, size_t expected) {
  size_t cap = 64;
  while (cap < expected * 2) cap <<= 1;
  m->keys = (int64_t *)malloc(cap * 3 * sizeof(int64_t));
  m->ids = (uint32_t *)malloc(cap * sizeof(uint32_t));
  if (!m->keys || !m->ids) return OR_ERR_NOMEM;
  memset(m->ids, 0xff, cap * sizeof(uint32_t));
  m->cap = cap;
  m->len = 0;
  return OR_OK;
}

static void cell_map_free(cell_map *m) {
  free(m->keys);
  free(m->ids);
}

static inline size_t cell_hash(const int64_t k[3]) {
  uint64_t h = 0;
  h = fx_mix(h, (uint64_t)k[0]);
  h = fx_mix(h, (uint64_t)k[1]);
  h = fx_mix(h, (uint64_t)k[2]);
  return (size_t)(h ^ (h >> 29));
}

static int cell_map_grow(cell_map *m) {
  cell_map bigger;
  if (cell_map_init(&bigger, m->cap) != OR_OK) return OR_ERR_NOMEM;
  for (size_t s = 0; s < m->cap; ++s) {
    if (m->ids[s] == UINT32_MAX) continue;
    size_t p = cell_hash(&m->keys[3 * s]) & (bigger.cap - 1);
    while (bigger.ids[p] != UINT32_MAX) p = (p + 1) & (bigger.cap - 1);
    memcpy(&bigger.keys[3 * p], &m->keys[3 * s], 3 * sizeof(int64_t));
    bigger.ids[p] = m->ids[s];
  }
  bigger.len = m->len;
  cell_map_free(m);
  *m = bigger;
  return OR_OK;
}

/* Returns the id for key, inserting next_id when absent (*inserted = 1). */
static int cell_map_get_or_insert(cell_map *m, const int64_t k[3], uint32_t next_id, uint32_t *id,
                                  int *inserted) {
  if ((m->len + 1) * 2 > m->cap) {
    if (cell_map_grow(m) != OR_OK) return OR_ERR_NOMEM;
  }
  size_t p = cell_hash(k) & (m->cap - 1);
  for (;;) {
    uint32_t cur = m->ids[p];
    if (cur == UINT32_MAX) {
      memcpy(&m->keys[3 * p], k, 3 * sizeof(int64_t));
      m->ids[p] = next_id;
      m->len++;
      *id = next_id;
      *inserted = 1;
      return OR_OK;
    }
    const int64_t *q = &m->keys[3 * p];
    if (q[0] == k[0] && q[1] == k[1] && q[2] == k[2]) {
      *id = cur;
      *inserted = 0;
      return OR_OK;
    }
    p = (p + 1) & (m->cap - 1);
  }
}

/* Id of key k, or UINT32_MAX when absent (read-only probe). */
static uint32_t cell_map_find(const cell_map *m, const int64_t k[3]) {
  size_t p = cell_hash(k) & (m->cap - 1);
  for (;;) {
    const uint32_t cur = m->ids[p];
    if (cur == UINT32_MAX) return UINT32_MAX;
    const int64_t *q = &m->keys[3 * p];
    if (q[0] == k[0] && q[1] == k[1] && q[2] == k[2]) return cur;
    p = (p + 1) & (m->cap - 1);
  }
}

static const int64_t *g_sort_keys; /* qsort context (single-threaded use) */

static int cmp_cell_ids(const void *a, const void *b) {
  const int64_t *ka = &g_sort_keys[3 * (size_t)(*(const uint32_t *)a)];
  const int64_t *kb = &g_sort_keys[3 * (size_t)(*(const uint32_t *)b)];
  for (int i = 0; i < 3; ++i) {
    if (ka[i] < kb[i]) return -1;
    if (ka[i] > kb[i]) return 1;
  }
  return 0;
}

/*
 * VoxelGridDownsample centroid/average on the CPU.
 *
 * Follows filter_internal (voxel.rs:251-275: empty input, leaf check,
 * inv_leaf = 1/leaf in f32, origin = explicit or compute_bounds min) and
 * filter_cpu_centroid_fast (voxel.rs:464-540): when plain_xyz == 0 (any
 * schema other than exactly x,y,z -- e.g. point_xyzi) every field is summed
 * in f64 per voxel and cells are emitted sorted by (ix,iy,iz), each value
 * (f32)(sum * (1.0 / count)).  When plain_xyz != 0 the plain-xyz variant
 * filter_cpu_xyz_centroid_fast (voxel.rs:550-636) is followed instead: f32
 * sums, first-occurrence output order, value sum * (1.0f / count).
 *
 * Fields: x, y, z then n_attrs attribute columns (all read as f32, voxel.rs:692-701).
 * Outputs are caller-allocated with capacity n: out_fields[3 + n_attrs]
 * (x, y, z, attrs...), out_keys (3 per voxel, nullable), out_counts
 * (nullable), and *out_v = number of voxels.  When n == 0 the reference
 * returns the input unchanged; this returns *out_v = 0.
 * Returns 0, or OR_ERR_INVALID for leaf <= 0 (voxel.rs:260-264).
 */
int oracle_voxel_centroid(const float *x, const float *y, const float *z, const float *const *attrs,
                          int n_attrs, size_t n, float leaf, int has_origin, const float *origin,
                          int plain_xyz, float *const *out_fields, int64_t *out_keys,
                          uint32_t *out_counts, size_t *out_v) {
  *out_v = 0;
  if (n == 0) return OR_OK;
  if (leaf <= 0.0f) return OR_ERR_INVALID; /* a NaN leaf passes, as in the reference */
  const float inv_leaf = 1.0f / leaf;
  float o[3];
  int u32_keys = 0;
  const int origin_is_min = !has_origin;
  if (has_origin) {
    o[0] = origin[0];
    o[1] = origin[1];
    o[2] = origin[2];
  } else {
    float mx[3];
    oracle_compute_bounds(x, y, z, n, o, mx);
    u32_keys = fits_u32_voxel_key(o, mx, inv_leaf);
  }
  const int nf = 3 + n_attrs;
  cell_map map;
  size_t expected = plain_xyz ? (n / 2 < 16 ? 16 : (n / 2 > 1048576 ? 1048576 : n / 2)) : 64;
  if (cell_map_init(&map, expected) != OR_OK) return OR_ERR_NOMEM;
  size_t cap_cells = 1024;
  int64_t *keys = (int64_t *)malloc(cap_cells * 3 * sizeof(int64_t));
  uint32_t *counts = (uint32_t *)malloc(cap_cells * sizeof(uint32_t));
  double *sums = plain_xyz ? NULL : (double *)malloc(cap_cells * nf * sizeof(double));
  float *fsums = plain_xyz ? (float *)malloc(cap_cells * 3 * sizeof(float)) : NULL;
  size_t ncells = 0;
  for (size_t i = 0; i < n; ++i) {
    int64_t k[3];
    if (plain_xyz && u32_keys)
      voxel_key_u32(x[i], y[i], z[i], o, inv_leaf, k);
    else if (origin_is_min)
      voxel_key_trunc(x[i], y[i], z[i], o, inv_leaf, k);
    else
      voxel_key_floor(x[i], y[i], z[i], o, inv_leaf, k);
    uint32_t id;
    int inserted;
    if (cell_map_get_or_insert(&map, k, (uint32_t)ncells, &id, &inserted) != OR_OK) goto nomem;
    if (inserted) {
      if (ncells == cap_cells) {
        cap_cells *= 2;
        keys = (int64_t *)realloc(keys, cap_cells * 3 * sizeof(int64_t));
        counts = (uint32_t *)realloc(counts, cap_cells * sizeof(uint32_t));
        if (sums) sums = (double *)realloc(sums, cap_cells * nf * sizeof(double));
        if (fsums) fsums = (float *)realloc(fsums, cap_cells * 3 * sizeof(float));
      }
      memcpy(&keys[3 * ncells], k, 3 * sizeof(int64_t));
      counts[ncells] = 0;
      if (sums)
        for (int f = 0; f < nf; ++f) sums[ncells * nf + f] = 0.0;
      if (fsums) fsums[3 * ncells] = fsums[3 * ncells + 1] = fsums[3 * ncells + 2] = 0.0f;
      ncells++;
    }
    counts[id] += 1;
    if (plain_xyz) {
      fsums[3 * id] += x[i];
      fsums[3 * id + 1] += y[i];
      fsums[3 * id + 2] += z[i];
    } else {
      double *s = &sums[(size_t)id * nf];
      s[0] += (double)x[i];
      s[1] += (double)y[i];
      s[2] += (double)z[i];
      for (int a = 0; a < n_attrs; ++a) s[3 + a] += (double)attrs[a][i];
    }
  }
  uint32_t *order = (uint32_t *)malloc(ncells * sizeof(uint32_t));
  for (size_t c = 0; c < ncells; ++c) order[c] = (uint32_t)c;
  if (!plain_xyz) {
    g_sort_keys = keys;
    qsort(order, ncells, sizeof(uint32_t), cmp_cell_ids);
  }
  for (size_t r = 0; r < ncells; ++r) {
    const uint32_t id = order[r];
    if (plain_xyz) {
      const float inv_count = 1.0f / (float)counts[id];
      out_fields[0][r] = fsums[3 * id] * inv_count;
      out_fields[1][r] = fsums[3 * id + 1] * inv_count;
      out_fields[2][r] = fsums[3 * id + 2] * inv_count;
    } else {
      const double inv_count = 1.0 / (double)counts[id];
      for (int f = 0; f < nf; ++f) out_fields[f][r] = (float)(sums[(size_t)id * nf + f] * inv_count);
    }
    if (out_keys) memcpy(&out_keys[3 * r], &keys[3 * (size_t)id], 3 * sizeof(int64_t));
    if (out_counts) out_counts[r] = counts[id];
  }
  *out_v = ncells;
  free(order);
  free(keys);
  free(counts);
  free(sums);
  free(fsums);
  cell_map_free(&map);
  return OR_OK;
nomem:
  free(keys);
  free(counts);
  free(sums);
  free(fsums);
  cell_map_free(&map);
  return OR_ERR_NOMEM;
}

/* General voxel path: build_voxel_cells_cpu (voxel.rs:703-716: floor keys,
 * point indices per cell in input order), cells sorted by key (voxel.rs:
 * 354), append_voxel_point (voxel.rs:1123-1154): with approximate != 0
 * every field is the cell's first point; otherwise positions are
 * average_field (voxel.rs:1156-1165: f64 sum over the indices in order,
 * divided by the count, cast to f32) and the other fields are the first
 * point's (attribute_first) or average_field (attribute average).  The
 * reference only reaches this path for modes other than Centroid + Average
 * on its CPU policies. */
int oracle_voxel_general(const float *x, const float *y, const float *z, const float *const *attrs,
                         int n_attrs, size_t n, float leaf, int has_origin, const float *origin,
                         int approximate, int attribute_first, float *const *out_fields,
                         int64_t *out_keys, uint32_t *out_counts, size_t *out_v) {
  *out_v = 0;
  if (n == 0) return OR_OK;
  if (leaf <= 0.0f) return OR_ERR_INVALID;
  const float inv_leaf = 1.0f / leaf;
  float o[3];
  if (has_origin) {
    o[0] = origin[0];
    o[1] = origin[1];
    o[2] = origin[2];
  } else {
    float mx[3];
    oracle_compute_bounds(x, y, z, n, o, mx);
  }
  const int nf = 3 + n_attrs;
  cell_map map;
  if (cell_map_init(&map, 64) != OR_OK) return OR_ERR_NOMEM;
  size_t cap_cells = 1024;
  int64_t *keys = (int64_t *)malloc(cap_cells * 3 * sizeof(int64_t));
  uint32_t *counts = (uint32_t *)malloc(cap_cells * sizeof(uint32_t));
  size_t *first = (size_t *)malloc(cap_cells * sizeof(size_t));
  double *sums = (double *)malloc(cap_cells * nf * sizeof(double));
  size_t ncells = 0;
  for (size_t i = 0; i < n; ++i) {
    int64_t k[3];
    voxel_key_floor(x[i], y[i], z[i], o, inv_leaf, k);
    uint32_t id;
    int inserted;
    if (cell_map_get_or_insert(&map, k, (uint32_t)ncells, &id, &inserted) != OR_OK) goto nomem;
    if (inserted) {
      if (ncells == cap_cells) {
        cap_cells *= 2;
        keys = (int64_t *)realloc(keys, cap_cells * 3 * sizeof(int64_t));
        counts = (uint32_t *)realloc(counts, cap_cells * sizeof(uint32_t));
        first = (size_t *)realloc(first, cap_cells * sizeof(size_t));
        sums = (double *)realloc(sums, cap_cells * nf * sizeof(double));
      }
      memcpy(&keys[3 * ncells], k, 3 * sizeof(int64_t));
      counts[ncells] = 0;
      first[ncells] = i;
      for (int f = 0; f < nf; ++f) sums[ncells * nf + f] = 0.0;
      ncells++;
    }
    counts[id] += 1;
    double *sm = &sums[(size_t)id * nf];
    sm[0] += (double)x[i];
    sm[1] += (double)y[i];
    sm[2] += (double)z[i];
    for (int a = 0; a < n_attrs; ++a) sm[3 + a] += (double)attrs[a][i];
  }
  uint32_t *order = (uint32_t *)malloc(ncells * sizeof(uint32_t));
  for (size_t c = 0; c < ncells; ++c) order[c] = (uint32_t)c;
  g_sort_keys = keys;
  qsort(order, ncells, sizeof(uint32_t), cmp_cell_ids);
  for (size_t r = 0; r < ncells; ++r) {
    const uint32_t id = order[r];
    const size_t rep = first[id];
    for (int f = 0; f < nf; ++f) {
      const float rep_value = f == 0 ? x[rep] : f == 1 ? y[rep] : f == 2 ? z[rep] : attrs[f - 3][rep];
      const int take_first = approximate || (f >= 3 && attribute_first);
      out_fields[f][r] =
          take_first ? rep_value : (float)(sums[(size_t)id * nf + f] / (double)counts[id]);
    }
    if (out_keys) memcpy(&out_keys[3 * r], &keys[3 * (size_t)id], 3 * sizeof(int64_t));
    if (out_counts) out_counts[r] = counts[id];
  }
  *out_v = ncells;
  free(order);
  free(keys);
  free(counts);
  free(first);
  free(sums);
  cell_map_free(&map);
  return OR_OK;
nomem:
  free(keys);
  free(counts);
  free(first);
  free(sums);
  cell_map_free(&map);
  return OR_ERR_NOMEM;
}

/* ------------------------------------------------------------------------ */
/* KD-tree (crates/spatialrust-search/src/kdtree.rs)                         */
/* ------------------------------------------------------------------------ */

#define KD_LEAF_SIZE 16     /* kdtree.rs:10 */
#define KD_AXIS_LEAF 255    /* kdtree.rs:12 */
#define KD_INVALID UINT32_MAX

typedef struct {
  float split;
  uint32_t left, right, start, end;
  uint8_t axis;
} kd_node;

typedef struct {
  const float *x, *y, *z;
  uint32_t *order;
  kd_node *nodes;
  size_t n_nodes, cap_nodes;
  uint32_t root;
} kd_tree;

static inline float kd_coord(const kd_tree *t, uint32_t p, uint8_t axis) {
  return axis == 0 ? t->x[p] : (axis == 1 ? t->y[p] : t->z[p]);
}

/* select_axis: kdtree.rs:458-490 (widest extent, ties keep the lower axis) */
static uint8_t kd_select_axis(const kd_tree *t, size_t start, size_t end) {
  float mn[3] = {INFINITY, INFINITY, INFINITY}, mx[3] = {-INFINITY, -INFINITY, -INFINITY};
  for (size_t i = start; i < end; ++i) {
    uint32_t p = t->order[i];
    mn[0] = rs_minf(mn[0], t->x[p]);
    mn[1] = rs_minf(mn[1], t->y[p]);
    mn[2] = rs_minf(mn[2], t->z[p]);
    mx[0] = rs_maxf(mx[0], t->x[p]);
    mx[1] = rs_maxf(mx[1], t->y[p]);
    mx[2] = rs_maxf(mx[2], t->z[p]);
  }
  uint8_t best = 0;
  float best_extent = mx[0] - mn[0];
  for (uint8_t a = 1; a < 3; ++a) {
    float e = mx[a] - mn[a];
    if (e > best_extent) {
      best_extent = e;
      best = a;
    }
  }
  return best;
}

static inline void swap_u32(uint32_t *a, size_t i, size_t j) {
  uint32_t t = a[i];
  a[i] = a[j];
  a[j] = t;
}

/* partition_by_axis: kdtree.rs:519-541 */
static size_t kd_partition(kd_tree *t, size_t start, size_t end, uint8_t axis) {
  size_t pivot_index = (start + end) / 2;
  swap_u32(t->order, start, pivot_index);
  float pv = kd_coord(t, t->order[start], axis);
  size_t store = start + 1;
  for (size_t i = start + 1; i < end; ++i) {
    if (kd_coord(t, t->order[i], axis) < pv) {
      swap_u32(t->order, i, store);
      store++;
    }
  }
  swap_u32(t->order, start, store - 1);
  return store - 1;
}

/* select_nth_by_axis: kdtree.rs:492-517 */
static void kd_select_nth(kd_tree *t, size_t start, size_t end, uint8_t axis, size_t nth) {
  size_t left = start, right = end;
  while (left < right) {
    size_t pivot = kd_partition(t, left, right, axis);
    if (nth < pivot)
      right = pivot;
    else if (nth > pivot)
      left = pivot + 1;
    else
      break;
  }
}

/* build_node: kdtree.rs:416-456 (median split, leaves of <= 16 points) */
static uint32_t kd_build_node(kd_tree *t, size_t start, size_t end) {
  if (t->n_nodes == t->cap_nodes) {
    t->cap_nodes *= 2;
    t->nodes = (kd_node *)realloc(t->nodes, t->cap_nodes * sizeof(kd_node));
  }
  uint32_t idx = (uint32_t)t->n_nodes++;
  kd_node nd = {0.0f, KD_INVALID, KD_INVALID, (uint32_t)start, (uint32_t)end, 0};
  t->nodes[idx] = nd;
  size_t count = end - start;
  if (count <= KD_LEAF_SIZE) {
    t->nodes[idx].axis = KD_AXIS_LEAF;
    return idx;
  }
  uint8_t axis = kd_select_axis(t, start, end);
  size_t mid = start + count / 2;
  kd_select_nth(t, start, end, axis, mid);
  float split = kd_coord(t, t->order[mid], axis);
  t->nodes[idx].axis = axis;
  t->nodes[idx].split = split;
  uint32_t l = kd_build_node(t, start, mid);
  uint32_t r = kd_build_node(t, mid, end);
  t->nodes[idx].left = l;
  t->nodes[idx].right = r;
  return idx;
}

/* KdTree::from_slices: kdtree.rs:39-55 */
static int kd_build(kd_tree *t, const float *x, const float *y, const float *z, size_t n) {
  t->x = x;
  t->y = y;
  t->z = z;
  t->order = (uint32_t *)malloc((n ? n : 1) * sizeof(uint32_t));
  t->cap_nodes = n ? ((n + KD_LEAF_SIZE - 1) / KD_LEAF_SIZE) * 2 + 8 : 8;
  t->nodes = (kd_node *)malloc(t->cap_nodes * sizeof(kd_node));
  t->n_nodes = 0;
  if (!t->order || !t->nodes) return OR_ERR_NOMEM;
  for (size_t i = 0; i < n; ++i) t->order[i] = (uint32_t)i;
  t->root = n ? kd_build_node(t, 0, n) : KD_INVALID;
  return OR_OK;
}

static void kd_free(kd_tree *t) {
  free(t->order);
  free(t->nodes);
}

/* squared_distance: kdtree.rs:544-549 (tree point minus query, x+y+z order) */
static inline float kd_sq_dist(float px, float py, float pz, float qx, float qy, float qz) {
  float dx = px - qx;
  float dy = py - qy;
  float dz = pz - qz;
  return dx * dx + dy * dy + dz * dz;
}

typedef struct {
  uint32_t *idx;
  size_t len, cap;
} u32_vec;

static inline void u32_push(u32_vec *v, uint32_t val) {
  if (v->len == v->cap) {
    v->cap = v->cap ? v->cap * 2 : 64;
    v->idx = (uint32_t *)realloc(v->idx, v->cap * sizeof(uint32_t));
  }
  v->idx[v->len++] = val;
}

/* radius_recursive: kdtree.rs:124-165 */
static void kd_radius(const kd_tree *t, uint32_t node, float qx, float qy, float qz, float r2,
                      u32_vec *out) {
  if (node == KD_INVALID) return;
  const kd_node nd = t->nodes[node];
  if (nd.axis == KD_AXIS_LEAF) {
    for (uint32_t i = nd.start; i < nd.end; ++i) {
      uint32_t p = t->order[i];
      float d2 = kd_sq_dist(t->x[p], t->y[p], t->z[p], qx, qy, qz);
      if (d2 <= r2) u32_push(out, p);
    }
    return;
  }
  float diff = nd.axis == 0 ? qx - nd.split : (nd.axis == 1 ? qy - nd.split : qz - nd.split);
  uint32_t near_n = diff <= 0.0f ? nd.left : nd.right;
  uint32_t far_n = diff <= 0.0f ? nd.right : nd.left;
  kd_radius(t, near_n, qx, qy, qz, r2, out);
  if (diff * diff <= r2) kd_radius(t, far_n, qx, qy, qz, r2, out);
}

/* ------------------------------------------------------------------------ */
/* Eigen solvers                                                            */
/* ------------------------------------------------------------------------ */

/* symmetric_eigen3 (FP64 cyclic-max Jacobi, 32 sweeps, stop at 1e-12):
 * crates/spatialrust-math/src/eigen.rs:16-84.  a is row-major 3x3, v returns
 * eigenvectors as columns sorted by ascending eigenvalue. */
static void rs_symmetric_eigen3(const double m[3][3], double vals[3], double vecs[3][3],
                                int max_iter, double tol) {
  double a[3][3], v[3][3] = {{1, 0, 0}, {0, 1, 0}, {0, 0, 1}};
  memcpy(a, m, sizeof(a));
  for (int it = 0; it < max_iter; ++it) {
    int p = 0, q = 1;
    double mx = fabs(a[0][1]);
    if (fabs(a[0][2]) > mx) {
      mx = fabs(a[0][2]);
      p = 0;
      q = 2;
    }
    if (fabs(a[1][2]) > mx) {
      mx = fabs(a[1][2]);
      p = 1;
      q = 2;
    }
    if (mx < tol) break;
    double app = a[p][p], aqq = a[q][q], apq = a[p][q];
    double phi = 0.5 * (aqq - app) / apq;
    double sgn = phi > 0.0 ? 1.0 : (phi < 0.0 ? -1.0 : (signbit(phi) ? -1.0 : 1.0));
    double t = sgn / (fabs(phi) + sqrt(1.0 + phi * phi));
    double c = 1.0 / sqrt(1.0 + t * t);
    double s = t * c;
    double app_new = c * c * app - 2.0 * s * c * apq + s * s * aqq;
    double aqq_new = s * s * app + 2.0 * s * c * apq + c * c * aqq;
    a[p][p] = app_new;
    a[q][q] = aqq_new;
    a[p][q] = 0.0;
    a[q][p] = 0.0;
    for (int r = 0; r < 3; ++r) {
      if (r != p && r != q) {
        double arp = a[r][p], arq = a[r][q];
        a[r][p] = c * arp - s * arq;
        a[p][r] = a[r][p];
        a[r][q] = s * arp + c * arq;
        a[q][r] = a[r][q];
      }
    }
    for (int r = 0; r < 3; ++r) {
      double vrp = v[r][p], vrq = v[r][q];
      v[r][p] = c * vrp - s * vrq;
      v[r][q] = s * vrp + c * vrq;
    }
  }
  double ev[3] = {a[0][0], a[1][1], a[2][2]};
  int order[3] = {0, 1, 2};
  for (int i = 0; i < 3; ++i) /* stable insertion sort, like sort_by */
    for (int j = i; j > 0 && ev[order[j]] < ev[order[j - 1]]; --j) {
      int tmp = order[j];
      order[j] = order[j - 1];
      order[j - 1] = tmp;
    }
  for (int i = 0; i < 3; ++i) {
    vals[i] = ev[order[i]];
    for (int r = 0; r < 3; ++r) vecs[r][i] = v[r][order[i]];
  }
}

static inline void f3_cross(const float a[3], const float b[3], float o[3]) {
  o[0] = a[1] * b[2] - a[2] * b[1];
  o[1] = a[2] * b[0] - a[0] * b[2];
  o[2] = a[0] * b[1] - a[1] * b[0];
}

static inline float f3_dot(const float a[3], const float b[3]) {
  return a[0] * b[0] + a[1] * b[1] + a[2] * b[2];
}

/* Vec3::normalize: crates/spatialrust-math/src/vec.rs:94-100 */
static inline void f3_normalize(float v[3]) {
  float len = sqrtf(f3_dot(v, v));
  if (len == 0.0f) return;
  v[0] = v[0] / len;
  v[1] = v[1] / len;
  v[2] = v[2] / len;
}

static int cmp_f32(const void *a, const void *b) {
  float x = *(const float *)a, y = *(const float *)b;
  return (x > y) - (x < y);
}

/* symmetric_eigenvalues3 (closed form, f32): normal.rs:506-542 */
static void rs_eigenvalues3(float c00, float c11, float c22, float c01, float c02, float c12,
                            float out[3]) {
  const float eps = 1.1920929e-07f; /* f32::EPSILON */
  float p1 = c01 * c01 + c02 * c02 + c12 * c12;
  if (p1 <= eps) {
    out[0] = c00;
    out[1] = c11;
    out[2] = c22;
    qsort(out, 3, sizeof(float), cmp_f32);
    return;
  }
  float q = (c00 + c11 + c22) / 3.0f;
  float b00 = c00 - q, b11 = c11 - q, b22 = c22 - q;
  float p2 = b00 * b00 + b11 * b11 + b22 * b22 + 2.0f * p1;
  float p = sqrtf(p2 / 6.0f);
  if (p <= eps) {
    out[0] = out[1] = out[2] = q;
    return;
  }
  float inv_p = 1.0f / p;
  float n00 = b00 * inv_p, n11 = b11 * inv_p, n22 = b22 * inv_p;
  float n01 = c01 * inv_p, n02 = c02 * inv_p, n12 = c12 * inv_p;
  float det = n00 * (n11 * n22 - n12 * n12) - n01 * (n01 * n22 - n12 * n02) +
              n02 * (n01 * n12 - n11 * n02);
  float r = det * 0.5f;
  r = r < -1.0f ? -1.0f : (r > 1.0f ? 1.0f : r);
  float phi = acosf(r) / 3.0f;
  float largest = q + 2.0f * p * cosf(phi);
  float smallest = q + 2.0f * p * cosf(phi + 2.0f * 3.14159265358979323846f / 3.0f);
  float middle = 3.0f * q - largest - smallest;
  out[0] = smallest;
  out[1] = middle;
  out[2] = largest;
  qsort(out, 3, sizeof(float), cmp_f32);
}

/* eigenvector_for_eigenvalue: normal.rs:544-573 (returns 0 when |best|^2 <= 1e-24) */
static int rs_eigenvector(float c00, float c11, float c22, float c01, float c02, float c12,
                          float lambda, float out[3]) {
  float r0[3] = {c00 - lambda, c01, c02};
  float r1[3] = {c01, c11 - lambda, c12};
  float r2[3] = {c02, c12, c22 - lambda};
  float cand[3][3];
  f3_cross(r0, r1, cand[0]);
  f3_cross(r0, r2, cand[1]);
  f3_cross(r1, r2, cand[2]);
  int best = 0;
  float best_norm = f3_dot(cand[0], cand[0]);
  for (int i = 1; i < 3; ++i) {
    float nrm = f3_dot(cand[i], cand[i]);
    if (nrm > best_norm) {
      best = i;
      best_norm = nrm;
    }
  }
  if (best_norm <= 1e-24f) return 0;
  memcpy(out, cand[best], sizeof(float) * 3);
  f3_normalize(out);
  return 1;
}

/* smallest_eigenpair_for_covariance: normal.rs:475-504 */
static void rs_smallest_eigenpair(float c00, float c11, float c22, float c01, float c02, float c12,
                                  float normal[3], float *curv) {
  float ev[3];
  rs_eigenvalues3(c00, c11, c22, c01, c02, c12, ev);
  if (!rs_eigenvector(c00, c11, c22, c01, c02, c12, ev[0], normal)) {
    double m[3][3] = {{c00, c01, c02}, {c01, c11, c12}, {c02, c12, c22}};
    double vals[3], vecs[3][3];
    rs_symmetric_eigen3(m, vals, vecs, 32, 1e-12);
    normal[0] = (float)vecs[0][0];
    normal[1] = (float)vecs[1][0];
    normal[2] = (float)vecs[2][0];
    f3_normalize(normal);
  }
  float sum = ev[0] + ev[1] + ev[2];
  *curv = sum > 0.0f ? ev[0] / sum : 0.0f;
  f3_normalize(normal);
}

/* ------------------------------------------------------------------------ */
/* Radius normals: reference restatement (f32, KD-tree, threads)            */
/* ------------------------------------------------------------------------ */

typedef struct {
  const kd_tree *tree;
  const float *x, *y, *z;
  size_t start, end;
  float radius;
  uint32_t min_neighbors;
  int has_vp;
  float vp[3];
  float *nx, *ny, *nz, *curv;
  uint32_t *counts;
  size_t valid, invalid;
} normal_job;

/* estimate_normal_range + query_neighbors_into (radius branch) +
 * estimate_normal_from_neighbors + orient_normal_towards_viewpoint:
 * normal.rs:321-368, 370-386, 427-473, 408-421 */
static void *normal_worker(void *arg) {
  normal_job *j = (normal_job *)arg;
  u32_vec found = {0}, nb = {0};
  const float r2 = j->radius * j->radius;
  for (size_t i = j->start; i < j->end; ++i) {
    found.len = 0;
    nb.len = 0;
    if (j->radius >= 0.0f && j->tree->root != KD_INVALID)
      kd_radius(j->tree, j->tree->root, j->x[i], j->y[i], j->z[i], r2, &found);
    for (size_t k = 0; k < found.len; ++k)
      if (found.idx[k] != (uint32_t)i) u32_push(&nb, found.idx[k]);
    if (j->counts) j->counts[i] = (uint32_t)nb.len;
    j->nx[i] = j->ny[i] = j->nz[i] = NAN;
    j->curv[i] = 0.0f;
    if (nb.len < j->min_neighbors) {
      j->invalid++;
      continue;
    }
    float mx = 0.0f, my = 0.0f, mz = 0.0f;
    for (size_t k = 0; k < nb.len; ++k) {
      mx += j->x[nb.idx[k]];
      my += j->y[nb.idx[k]];
      mz += j->z[nb.idx[k]];
    }
    float cnt = (float)nb.len;
    mx /= cnt;
    my /= cnt;
    mz /= cnt;
    float c00 = 0, c11 = 0, c22 = 0, c01 = 0, c02 = 0, c12 = 0;
    for (size_t k = 0; k < nb.len; ++k) {
      float dx = j->x[nb.idx[k]] - mx, dy = j->y[nb.idx[k]] - my, dz = j->z[nb.idx[k]] - mz;
      c00 += dx * dx;
      c11 += dy * dy;
      c22 += dz * dz;
      c01 += dx * dy;
      c02 += dx * dz;
      c12 += dy * dz;
    }
    float inv = 1.0f / cnt;
    float normal[3], curv;
    rs_smallest_eigenpair(c00 * inv, c11 * inv, c22 * inv, c01 * inv, c02 * inv, c12 * inv, normal,
                          &curv);
    if (j->has_vp) {
      float view[3] = {j->vp[0] - j->x[i], j->vp[1] - j->y[i], j->vp[2] - j->z[i]};
      if (f3_dot(normal, view) < 0.0f) {
        normal[0] = -normal[0];
        normal[1] = -normal[1];
        normal[2] = -normal[2];
      }
      f3_normalize(normal);
    }
    j->nx[i] = normal[0];
    j->ny[i] = normal[1];
    j->nz[i] = normal[2];
    j->curv[i] = curv;
    j->valid++;
  }
  free(found.idx);
  free(nb.idx);
  return NULL;
}

/* parallel_worker_count: crates/spatialrust-search/src/staging.rs:11-28
 * (min(available, n / 16384) when n >= 4096, else 1). */
size_t oracle_parallel_worker_count(size_t n, size_t available) {
  if (n < 4096) return 1;
  size_t useful = n / 16384;
  if (useful < 1) useful = 1;
  return available < useful ? available : useful;
}

/*
 * NormalEstimator::estimate_with_diagnostics in radius mode on the CPU
 * (normal.rs:102-164): KD-tree over the cloud, per-point radius neighbours
 * with the query itself excluded, invalid below min_neighbors (NaN normal,
 * curvature 0), f32 two-pass covariance, closed-form eigen with FP64 Jacobi
 * fallback, optional viewpoint orientation.  Threads follow
 * parallel_worker_count / parallel_index_ranges (staging.rs:11-41);
 * threads == 0 uses every online CPU.  Returns valid count via *valid.
 */
int oracle_radius_normals_ref(const float *x, const float *y, const float *z, size_t n,
                              float radius, uint32_t min_neighbors, int has_vp, const float *vp,
                              int threads, float *nx, float *ny, float *nz, float *curv,
                              uint32_t *counts, size_t *valid, size_t *invalid) {
  *valid = *invalid = 0;
  if (n == 0) return OR_OK;
  if (radius < 0.0f) return OR_ERR_INVALID; /* normal.rs:109-111 */
  kd_tree tree;
  if (kd_build(&tree, x, y, z, n) != OR_OK) return OR_ERR_NOMEM;
  size_t avail = threads > 0 ? (size_t)threads : (size_t)sysconf(_SC_NPROCESSORS_ONLN);
  size_t workers = oracle_parallel_worker_count(n, avail);
  size_t chunk = (n + workers - 1) / workers;
  size_t njobs = (n + chunk - 1) / chunk;
  normal_job *jobs = (normal_job *)calloc(njobs, sizeof(normal_job));
  pthread_t *tids = (pthread_t *)calloc(njobs, sizeof(pthread_t));
  for (size_t w = 0; w < njobs; ++w) {
    normal_job *j = &jobs[w];
    j->tree = &tree;
    j->x = x;
    j->y = y;
    j->z = z;
    j->start = w * chunk;
    j->end = j->start + chunk < n ? j->start + chunk : n;
    j->radius = radius;
    j->min_neighbors = min_neighbors;
    j->has_vp = has_vp;
    if (has_vp) memcpy(j->vp, vp, sizeof(float) * 3);
    j->nx = nx;
    j->ny = ny;
    j->nz = nz;
    j->curv = curv;
    j->counts = counts;
  }
  if (njobs == 1) {
    normal_worker(&jobs[0]);
  } else {
    for (size_t w = 0; w < njobs; ++w) pthread_create(&tids[w], NULL, normal_worker, &jobs[w]);
    for (size_t w = 0; w < njobs; ++w) pthread_join(tids[w], NULL);
  }
  for (size_t w = 0; w < njobs; ++w) {
    *valid += jobs[w].valid;
    *invalid += jobs[w].invalid;
  }
  free(jobs);
  free(tids);
  kd_free(&tree);
  return OR_OK;
}

/* ------------------------------------------------------------------------ */
/* FP64 oracle for radius normals                                           */
/* ------------------------------------------------------------------------ */

typedef struct {
  const kd_tree *tree;
  const float *x, *y, *z;
  size_t start, end;
  float radius;
  double shell_rel;
  uint32_t min_neighbors;
  int has_vp;
  float vp[3];
  int include_self;
  double *nx, *ny, *nz, *curv, *gap;
  uint32_t *counts;
  uint8_t *shell;
} fp64_job;

/*
 * Same neighbour set as the reference (f32 predicate of kdtree.rs:544-549,
 * query excluded, normal.rs:381-386); FP64 two-pass mean and covariance;
 * FP64 cyclic-max Jacobi run to convergence (1e-300 tolerance, 200 rotations);
 * smallest eigenvector, sign toward the viewpoint (normal.rs:408-421, in FP64).
 * gap = (l1 - l0) / max(l2, tiny) flags ill-conditioned normals.
 * shell[i] = 1 when some other point has |d2 - r2| <= shell_rel * r2.
 *
 * include_self: the semantics of the reference's wgpu grid estimator
 * (NORMALS_GRID_WGSL, crates/spatialrust-gpu/src/kernels/normals_grid.rs:
 * 86-197, behind GpuNormalEstimator::estimate, normal_gpu.rs:33-83): the query
 * belongs to its own neighbourhood (its d2 is 0 when it is finite), a
 * neighbourhood of fewer than 3 points gives the normal (0, 0, 1) and
 * curvature 0 (normals_grid.rs:129-132), min_neighbors plays no part, and
 * every normal -- the fallback included -- is turned toward the viewpoint
 * (normal_gpu.rs:63-70).  counts[i] then includes the query.
 */
static void *fp64_worker(void *arg) {
  fp64_job *j = (fp64_job *)arg;
  u32_vec found = {0};
  const float r2 = j->radius * j->radius;
  const float r2_wide = (float)((double)r2 * (1.0 + 4.0 * j->shell_rel)) + 1e-30f;
  for (size_t i = j->start; i < j->end; ++i) {
    found.len = 0;
    if (j->tree->root != KD_INVALID)
      kd_radius(j->tree, j->tree->root, j->x[i], j->y[i], j->z[i], r2_wide, &found);
    const float qx = j->x[i], qy = j->y[i], qz = j->z[i];
    uint32_t cnt = 0;
    int shell = 0;
    double sx = 0, sy = 0, sz = 0;
    for (size_t k = 0; k < found.len; ++k) {
      uint32_t p = found.idx[k];
      if (p == (uint32_t)i && !j->include_self) continue;
      float d2 = kd_sq_dist(j->x[p], j->y[p], j->z[p], qx, qy, qz);
      if (p != (uint32_t)i && fabs((double)d2 - (double)r2) <= j->shell_rel * (double)r2) shell = 1;
      if (d2 <= r2) {
        cnt++;
        sx += j->x[p];
        sy += j->y[p];
        sz += j->z[p];
      }
    }
    j->counts[i] = cnt;
    j->shell[i] = (uint8_t)shell;
    j->nx[i] = j->ny[i] = j->nz[i] = NAN;
    j->curv[i] = 0.0;
    j->gap[i] = 0.0;
    if (j->include_self ? cnt < 3 : (cnt < j->min_neighbors || cnt == 0)) {
      if (j->include_self) { /* normals_grid.rs:129-132, oriented as normal_gpu.rs:63-70 */
        j->nx[i] = 0.0;
        j->ny[i] = 0.0;
        j->nz[i] = (j->has_vp && j->vp[2] < qz) ? -1.0 : 1.0;
      }
      continue;
    }
    double mx = sx / cnt, my = sy / cnt, mz = sz / cnt;
    double c[3][3] = {{0}};
    for (size_t k = 0; k < found.len; ++k) {
      uint32_t p = found.idx[k];
      if (p == (uint32_t)i && !j->include_self) continue;
      float d2 = kd_sq_dist(j->x[p], j->y[p], j->z[p], qx, qy, qz);
      if (!(d2 <= r2)) continue;
      double dx = j->x[p] - mx, dy = j->y[p] - my, dz = j->z[p] - mz;
      c[0][0] += dx * dx;
      c[1][1] += dy * dy;
      c[2][2] += dz * dz;
      c[0][1] += dx * dy;
      c[0][2] += dx * dz;
      c[1][2] += dy * dz;
    }
    for (int a = 0; a < 3; ++a)
      for (int b = a; b < 3; ++b) {
        c[a][b] /= cnt;
        c[b][a] = c[a][b];
      }
    double vals[3], vecs[3][3];
    rs_symmetric_eigen3(c, vals, vecs, 200, 1e-300);
    double n0 = vecs[0][0], n1 = vecs[1][0], n2 = vecs[2][0];
    double len = sqrt(n0 * n0 + n1 * n1 + n2 * n2);
    if (len > 0) {
      n0 /= len;
      n1 /= len;
      n2 /= len;
    }
    if (j->has_vp) {
      double vx = (double)j->vp[0] - qx, vy = (double)j->vp[1] - qy, vz = (double)j->vp[2] - qz;
      if (n0 * vx + n1 * vy + n2 * vz < 0.0) {
        n0 = -n0;
        n1 = -n1;
        n2 = -n2;
      }
    }
    j->nx[i] = n0;
    j->ny[i] = n1;
    j->nz[i] = n2;
    double sum = vals[0] + vals[1] + vals[2];
    j->curv[i] = sum > 0.0 ? vals[0] / sum : 0.0;
    double top = fabs(vals[2]) > 1e-300 ? fabs(vals[2]) : 1e-300;
    j->gap[i] = (vals[1] - vals[0]) / top;
  }
  free(found.idx);
  return NULL;
}

int oracle_radius_normals_fp64(const float *x, const float *y, const float *z, size_t n,
                               float radius, uint32_t min_neighbors, int has_vp, const float *vp,
                               double shell_rel, int threads, double *nx, double *ny, double *nz,
                               double *curv, double *gap, uint32_t *counts, uint8_t *shell,
                               int include_self) {
  if (n == 0) return OR_OK;
  if (radius < 0.0f) return OR_ERR_INVALID;
  kd_tree tree;
  if (kd_build(&tree, x, y, z, n) != OR_OK) return OR_ERR_NOMEM;
  size_t avail = threads > 0 ? (size_t)threads : (size_t)sysconf(_SC_NPROCESSORS_ONLN);
  size_t workers = n < 4096 ? 1 : (avail < n / 1024 ? avail : (n / 1024 ? n / 1024 : 1));
  size_t chunk = (n + workers - 1) / workers;
  size_t njobs = (n + chunk - 1) / chunk;
  fp64_job *jobs = (fp64_job *)calloc(njobs, sizeof(fp64_job));
  pthread_t *tids = (pthread_t *)calloc(njobs, sizeof(pthread_t));
  for (size_t w = 0; w < njobs; ++w) {
    fp64_job *j = &jobs[w];
    j->tree = &tree;
    j->x = x;
    j->y = y;
    j->z = z;
    j->start = w * chunk;
    j->end = j->start + chunk < n ? j->start + chunk : n;
    j->radius = radius;
    j->shell_rel = shell_rel;
    j->min_neighbors = min_neighbors;
    j->has_vp = has_vp;
    if (has_vp) memcpy(j->vp, vp, sizeof(float) * 3);
    j->include_self = include_self;
    j->nx = nx;
    j->ny = ny;
    j->nz = nz;
    j->curv = curv;
    j->gap = gap;
    j->counts = counts;
    j->shell = shell;
  }
  if (njobs == 1) {
    fp64_worker(&jobs[0]);
  } else {
    for (size_t w = 0; w < njobs; ++w) pthread_create(&tids[w], NULL, fp64_worker, &jobs[w]);
    for (size_t w = 0; w < njobs; ++w) pthread_join(tids[w], NULL);
  }
  free(jobs);
  free(tids);
  kd_free(&tree);
  return OR_OK;
}

/* ------------------------------------------------------------------------ */
/* The wgpu grid estimator's arithmetic, in f32                              */
/* ------------------------------------------------------------------------ */

/* rotate() of NORMALS_GRID_WGSL (normals_grid.rs:46-80): one Jacobi rotation
 * zeroing a[p][q], applied to the rows and columns of a and the columns of v. */
static void wgsl_rotate(float a[3][3], float v[3][3], int p, int q) {
  const float apq = a[p][q];
  if (fabsf(apq) < 1e-20f) return;
  const float app = a[p][p], aqq = a[q][q];
  const float phi = 0.5f * (aqq - app) / apq;
  float t;
  if (phi >= 0.0f) t = 1.0f / (phi + sqrtf(1.0f + phi * phi));
  else t = -1.0f / (-phi + sqrtf(1.0f + phi * phi));
  const float c = 1.0f / sqrtf(1.0f + t * t);
  const float s = t * c;
  for (int r = 0; r < 3; ++r) {
    const float arp = a[r][p], arq = a[r][q];
    a[r][p] = c * arp - s * arq;
    a[r][q] = s * arp + c * arq;
  }
  for (int r = 0; r < 3; ++r) {
    const float apr = a[p][r], aqr = a[q][r];
    a[p][r] = c * apr - s * aqr;
    a[q][r] = s * apr + c * aqr;
  }
  for (int r = 0; r < 3; ++r) {
    const float vrp = v[r][p], vrq = v[r][q];
    v[r][p] = c * vrp - s * vrq;
    v[r][q] = s * vrp + c * vrq;
  }
}

typedef struct {
  const kd_tree *tree;
  const float *x, *y, *z;
  size_t start, end;
  float r2;
  int has_vp;
  float vp[3];
  float *nx, *ny, *nz, *curv;
  uint32_t *counts;
} wgsl_job;

/* main() of NORMALS_GRID_WGSL (normals_grid.rs:86-197) on the neighbour set
 * of the f32 predicate with the query included, then GpuNormalEstimator's
 * host-side orientation (normal_gpu.rs:63-70, orient_normal_towards_viewpoint
 * normal.rs:408-421 with Vec3::dot / normalize, vec.rs:66-100).  f32 mean and
 * covariance sums (undivided), 16 sweeps of (0,1), (0,2), (1,2) rotations,
 * the smallest diagonal entry's column.  The shader visits the 27 cells in
 * its own order; sums here run in KD-tree order, so results agree with the
 * shader to f32 rounding, not bit for bit. */
static void *wgsl_worker(void *arg) {
  wgsl_job *j = (wgsl_job *)arg;
  u32_vec found = {0};
  for (size_t i = j->start; i < j->end; ++i) {
    found.len = 0;
    const float px = j->x[i], py = j->y[i], pz = j->z[i];
    if (j->tree->root != KD_INVALID) kd_radius(j->tree, j->tree->root, px, py, pz, j->r2, &found);
    float mean[3] = {0, 0, 0}, count = 0.0f;
    for (size_t k = 0; k < found.len; ++k) {
      const uint32_t q = found.idx[k];
      mean[0] += j->x[q];
      mean[1] += j->y[q];
      mean[2] += j->z[q];
      count += 1.0f;
    }
    j->counts[i] = (uint32_t)found.len;
    float n[3] = {0.0f, 0.0f, 1.0f}, curvature = 0.0f;
    if (count >= 3.0f) {
      for (int a = 0; a < 3; ++a) mean[a] = mean[a] / count;
      float c00 = 0, c11 = 0, c22 = 0, c01 = 0, c02 = 0, c12 = 0;
      for (size_t k = 0; k < found.len; ++k) {
        const uint32_t q = found.idx[k];
        const float dx = j->x[q] - mean[0], dy = j->y[q] - mean[1], dz = j->z[q] - mean[2];
        c00 = c00 + dx * dx;
        c11 = c11 + dy * dy;
        c22 = c22 + dz * dz;
        c01 = c01 + dx * dy;
        c02 = c02 + dx * dz;
        c12 = c12 + dy * dz;
      }
      float a[3][3] = {{c00, c01, c02}, {c01, c11, c12}, {c02, c12, c22}};
      float v[3][3] = {{1, 0, 0}, {0, 1, 0}, {0, 0, 1}};
      for (int sweep = 0; sweep < 16; ++sweep) {
        wgsl_rotate(a, v, 0, 1);
        wgsl_rotate(a, v, 0, 2);
        wgsl_rotate(a, v, 1, 2);
      }
      const float eig[3] = {a[0][0], a[1][1], a[2][2]};
      int m = 0;
      if (eig[1] < eig[m]) m = 1;
      if (eig[2] < eig[m]) m = 2;
      float len = sqrtf(v[0][m] * v[0][m] + v[1][m] * v[1][m] + v[2][m] * v[2][m]);
      if (len < 1e-20f) len = 1e-20f;
      for (int a2 = 0; a2 < 3; ++a2) n[a2] = v[a2][m] / len;
      const float trace = eig[0] + eig[1] + eig[2];
      if (trace > 0.0f) curvature = eig[m] / trace;
    }
    if (j->has_vp) {
      const float wx = j->vp[0] - px, wy = j->vp[1] - py, wz = j->vp[2] - pz;
      if (n[0] * wx + n[1] * wy + n[2] * wz < 0.0f) {
        n[0] = -n[0];
        n[1] = -n[1];
        n[2] = -n[2];
      }
      const float l = sqrtf(n[0] * n[0] + n[1] * n[1] + n[2] * n[2]);
      if (l != 0.0f)
        for (int a2 = 0; a2 < 3; ++a2) n[a2] = n[a2] / l;
    }
    j->nx[i] = n[0];
    j->ny[i] = n[1];
    j->nz[i] = n[2];
    j->curv[i] = curvature;
  }
  free(found.idx);
  return NULL;
}

int oracle_grid_normals_wgsl(const float *x, const float *y, const float *z, size_t n,
                             float radius, int has_vp, const float *vp, int threads, float *nx,
                             float *ny, float *nz, float *curv, uint32_t *counts) {
  if (n == 0) return OR_OK;
  if (radius < 0.0f) return OR_ERR_INVALID;
  kd_tree tree;
  if (kd_build(&tree, x, y, z, n) != OR_OK) return OR_ERR_NOMEM;
  size_t avail = threads > 0 ? (size_t)threads : (size_t)sysconf(_SC_NPROCESSORS_ONLN);
  size_t workers = n < 4096 ? 1 : (avail < n / 1024 ? avail : (n / 1024 ? n / 1024 : 1));
  size_t chunk = (n + workers - 1) / workers;
  size_t njobs = (n + chunk - 1) / chunk;
  wgsl_job *jobs = (wgsl_job *)calloc(njobs, sizeof(wgsl_job));
  pthread_t *tids = (pthread_t *)calloc(njobs, sizeof(pthread_t));
  for (size_t w = 0; w < njobs; ++w) {
    wgsl_job *j = &jobs[w];
    j->tree = &tree;
    j->x = x;
    j->y = y;
    j->z = z;
    j->start = w * chunk;
    j->end = j->start + chunk < n ? j->start + chunk : n;
    j->r2 = radius * radius; /* GridUniform.radius_sq, normals_grid.rs:263 */
    j->has_vp = has_vp;
    if (has_vp) memcpy(j->vp, vp, sizeof(float) * 3);
    j->nx = nx;
    j->ny = ny;
    j->nz = nz;
    j->curv = curv;
    j->counts = counts;
  }
  if (njobs == 1) {
    wgsl_worker(&jobs[0]);
  } else {
    for (size_t w = 0; w < njobs; ++w) pthread_create(&tids[w], NULL, wgsl_worker, &jobs[w]);
    for (size_t w = 0; w < njobs; ++w) pthread_join(tids[w], NULL);
  }
  free(jobs);
  free(tids);
  kd_free(&tree);
  return OR_OK;
}

/* Brute-force neighbour counts with the reference predicate (self excluded);
 * used to check the KD-tree restatement, as kdtree.rs's own tests do. */
void oracle_brute_radius_counts(const float *x, const float *y, const float *z, size_t n,
                                float radius, uint32_t *counts) {
  const float r2 = radius * radius;
  for (size_t i = 0; i < n; ++i) {
    uint32_t c = 0;
    for (size_t p = 0; p < n; ++p) {
      if (p == i) continue;
      if (kd_sq_dist(x[p], y[p], z[p], x[i], y[i], z[i]) <= r2) c++;
    }
    counts[i] = c;
  }
}

/* ------------------------------------------------------------------------ */
/* Euclidean cluster roots (crates/spatialrust-search/src/uniform_grid.rs)   */
/* ------------------------------------------------------------------------ */

#define OR_ERR_GRID_TOO_LARGE (-3)
#define UG_MAX_CELLS 64000000ull /* MAX_UNIFORM_GRID_CELLS, uniform_grid.rs:6 */

/* find_root without compression (uniform_grid.rs:420-425) */
static uint32_t uf_find_readonly(const uint32_t *parent, uint32_t i) {
  while (parent[i] != i) i = parent[i];
  return i;
}

/* union_min_root (uniform_grid.rs:410-418): the larger root joins the smaller */
static void uf_union_min(uint32_t *parent, uint32_t a, uint32_t b) {
  const uint32_t ra = uf_find_readonly(parent, a), rb = uf_find_readonly(parent, b);
  if (ra == rb) return;
  if (ra < rb) parent[rb] = ra;
  else parent[ra] = rb;
}

/* euclidean_cluster_roots (uniform_grid.rs:90-139) on one thread:
 * grid_bounds (:9-36: f32 min/max, dims = floor(span / cell) + 1, at most
 * 64M dense cells), build_grid (:44-87: counting sort over dense cells,
 * clamped floor cells), cluster_roots_sequential (:262-289: every point
 * unioned with every point of the 27 surrounding cells that passes
 * dx*dx + dy*dy + dz*dz <= tol*tol, differences neighbour minus point) and
 * compress_roots (:389-395).  roots[i] is the smallest index of i's
 * component.  Returns OR_ERR_INVALID for tol <= 0 or NaN, and
 * OR_ERR_GRID_TOO_LARGE where the reference reports the grid cap. */
int oracle_euclidean_roots(const float *x, const float *y, const float *z, size_t n, float tol,
                           uint32_t *roots) {
  if (!(tol > 0.0f)) return OR_ERR_INVALID;
  if (n == 0) return OR_OK;
  float mn[3] = {INFINITY, INFINITY, INFINITY}, mx[3] = {-INFINITY, -INFINITY, -INFINITY};
  for (size_t i = 0; i < n; ++i) {
    const float v[3] = {x[i], y[i], z[i]};
    for (int a = 0; a < 3; ++a) {
      mn[a] = rs_minf(mn[a], v[a]);
      mx[a] = rs_maxf(mx[a], v[a]);
    }
  }
  const float inv = 1.0f / tol;
  uint64_t dims[3];
  for (int a = 0; a < 3; ++a) {
    const int64_t span = sat_f32_to_i64(floorf((mx[a] - mn[a]) * inv)) + 1;
    dims[a] = (uint64_t)(span < 1 ? 1 : (span > 0xFFFFFFFFll ? 0xFFFFFFFFll : span));
  }
  const uint64_t cells = dims[0] * dims[1] * dims[2];
  if (dims[0] > UG_MAX_CELLS || dims[1] > UG_MAX_CELLS || dims[2] > UG_MAX_CELLS ||
      cells > UG_MAX_CELLS)
    return OR_ERR_GRID_TOO_LARGE;
  uint32_t *cell = (uint32_t *)malloc(n * sizeof(uint32_t));
  uint32_t *start = (uint32_t *)calloc(cells + 1, sizeof(uint32_t));
  uint32_t *sorted = (uint32_t *)malloc(n * sizeof(uint32_t));
  uint32_t *parent = (uint32_t *)malloc(n * sizeof(uint32_t));
  int64_t (*ci)[3] = (int64_t(*)[3])malloc(n * sizeof(int64_t[3]));
  if (!cell || !start || !sorted || !parent || !ci) {
    free(cell); free(start); free(sorted); free(parent); free(ci);
    return OR_ERR_NOMEM;
  }
  for (size_t i = 0; i < n; ++i) {
    const float v[3] = {x[i], y[i], z[i]};
    for (int a = 0; a < 3; ++a) {
      int64_t c = sat_f32_to_i64(floorf((v[a] - mn[a]) * inv));
      if (c < 0) c = 0;
      if (c > (int64_t)dims[a] - 1) c = (int64_t)dims[a] - 1;
      ci[i][a] = c;
    }
    cell[i] = (uint32_t)(((uint64_t)ci[i][2] * dims[1] + (uint64_t)ci[i][1]) * dims[0] +
                         (uint64_t)ci[i][0]);
    start[cell[i]]++;
  }
  uint32_t acc = 0;
  for (uint64_t c = 0; c <= cells; ++c) {
    const uint32_t k = start[c];
    start[c] = acc;
    acc += k;
  }
  {
    uint32_t *cursor = (uint32_t *)malloc((cells + 1) * sizeof(uint32_t));
    memcpy(cursor, start, (cells + 1) * sizeof(uint32_t));
    for (size_t i = 0; i < n; ++i) sorted[cursor[cell[i]]++] = (uint32_t)i;
    free(cursor);
  }
  for (size_t i = 0; i < n; ++i) parent[i] = (uint32_t)i;
  const float r2 = tol * tol;
  for (size_t i = 0; i < n; ++i) {
    for (int dz = -1; dz <= 1; ++dz)
      for (int dy = -1; dy <= 1; ++dy)
        for (int dx = -1; dx <= 1; ++dx) {
          const int64_t cx = ci[i][0] + dx, cy = ci[i][1] + dy, cz = ci[i][2] + dz;
          if (cx < 0 || cy < 0 || cz < 0 || cx >= (int64_t)dims[0] || cy >= (int64_t)dims[1] ||
              cz >= (int64_t)dims[2])
            continue;
          const uint64_t c = ((uint64_t)cz * dims[1] + (uint64_t)cy) * dims[0] + (uint64_t)cx;
          for (uint32_t s = start[c]; s < start[c + 1]; ++s) {
            const uint32_t j = sorted[s];
            const float ddx = x[j] - x[i], ddy = y[j] - y[i], ddz = z[j] - z[i];
            if (ddx * ddx + ddy * ddy + ddz * ddz <= r2) uf_union_min(parent, (uint32_t)i, j);
          }
        }
  }
  for (size_t i = 0; i < n; ++i) roots[i] = uf_find_readonly(parent, (uint32_t)i);
  free(cell); free(start); free(sorted); free(parent); free(ci);
  return OR_OK;
}

/* The reference's sparse-cell path (euclidean_cluster_roots_gpu_with_receipt,
 * crates/spatialrust-gpu/src/kernels/euclidean_cluster.rs:9-58, then
 * euclidean_cluster_roots_from_segments, uniform_grid.rs:148-250): cells are
 * voxel keys floor((p - min) * (1 / tol)) with the origin the f32 minimum
 * starting from point 0, kept in a hash map (no dense cap); every point is
 * unioned with the points of the 27 neighbouring keys (saturating) that pass
 * the predicate.  Same roots as the dense grid wherever both run. */
int oracle_euclidean_roots_sparse(const float *x, const float *y, const float *z, size_t n,
                                  float tol, uint32_t *roots) {
  if (!(tol > 0.0f)) return OR_ERR_INVALID;
  if (n == 0) return OR_OK;
  float o[3] = {x[0], y[0], z[0]};
  for (size_t i = 1; i < n; ++i) {
    o[0] = rs_minf(o[0], x[i]);
    o[1] = rs_minf(o[1], y[i]);
    o[2] = rs_minf(o[2], z[i]);
  }
  const float inv = 1.0f / tol;
  cell_map map;
  if (cell_map_init(&map, n < 16 ? 16 : n) != OR_OK) return OR_ERR_NOMEM;
  int64_t (*key)[3] = (int64_t(*)[3])malloc(n * sizeof(int64_t[3]));
  uint32_t *cell = (uint32_t *)malloc(n * sizeof(uint32_t));
  uint32_t *count = (uint32_t *)calloc(n + 1, sizeof(uint32_t));
  uint32_t *start = (uint32_t *)malloc((n + 1) * sizeof(uint32_t));
  uint32_t *members = (uint32_t *)malloc(n * sizeof(uint32_t));
  uint32_t *parent = (uint32_t *)malloc(n * sizeof(uint32_t));
  int rc = OR_OK;
  if (!key || !cell || !count || !start || !members || !parent) {
    rc = OR_ERR_NOMEM;
    goto done;
  }
  uint32_t ncells = 0;
  for (size_t i = 0; i < n; ++i) {
    voxel_key_floor(x[i], y[i], z[i], o, inv, key[i]);
    uint32_t id;
    int inserted;
    if (cell_map_get_or_insert(&map, key[i], ncells, &id, &inserted) != OR_OK) {
      rc = OR_ERR_NOMEM;
      goto done;
    }
    if (inserted) ncells++;
    cell[i] = id;
    count[id]++;
  }
  {
    uint32_t acc = 0;
    for (uint32_t c = 0; c < ncells; ++c) {
      start[c] = acc;
      acc += count[c];
      count[c] = 0;
    }
    start[ncells] = acc;
    for (size_t i = 0; i < n; ++i) members[start[cell[i]] + count[cell[i]]++] = (uint32_t)i;
  }
  for (size_t i = 0; i < n; ++i) parent[i] = (uint32_t)i;
  {
    const float r2 = tol * tol;
    for (size_t i = 0; i < n; ++i)
      for (int dz = -1; dz <= 1; ++dz)
        for (int dy = -1; dy <= 1; ++dy)
          for (int dx = -1; dx <= 1; ++dx) {
            const int64_t d[3] = {dx, dy, dz};
            int64_t nk[3];
            for (int a = 0; a < 3; ++a) {
              const int64_t k = key[i][a];  /* saturating_add */
              nk[a] = (d[a] > 0 && k == INT64_MAX) ? INT64_MAX
                      : (d[a] < 0 && k == INT64_MIN) ? INT64_MIN : k + d[a];
            }
            const uint32_t id = cell_map_find(&map, nk);
            if (id == UINT32_MAX) continue;
            for (uint32_t s2 = start[id]; s2 < start[id + 1]; ++s2) {
              const uint32_t j = members[s2];
              const float ddx = x[j] - x[i], ddy = y[j] - y[i], ddz = z[j] - z[i];
              if (ddx * ddx + ddy * ddy + ddz * ddz <= r2) uf_union_min(parent, (uint32_t)i, j);
            }
          }
  }
  for (size_t i = 0; i < n; ++i) roots[i] = uf_find_readonly(parent, (uint32_t)i);
done:
  free(key); free(cell); free(count); free(start); free(members); free(parent);
  cell_map_free(&map);
  return rc;
}

/* ------------------------------------------------------------------------ */
/* GICP plane covariances on the radius grid                                */
/* (crates/spatialrust-gpu/src/kernels/covariances_grid.rs:87-206)          */
/* ------------------------------------------------------------------------ */

typedef struct {
  const kd_tree *tree;
  const float *x, *y, *z;
  size_t start, end;
  float radius;
  double eps;
  double *cov, *gap;
  uint32_t *counts;
} cov_job;

/*
 * Per point: every point within radius (the f32 predicate, the query itself
 * included, covariances_grid.rs:100-121); fewer than 3 -> (eps, eps, eps, 0,
 * 0, 0) (:127-131); else the FP64 two-pass covariance, its eigenvectors by
 * FP64 cyclic-max Jacobi run to convergence, and sum_col lambda v v^T with
 * lambda = eps for the smallest eigenvalue and 1 for the others
 * (:165-202, the same rebuild as gicp.rs:276-291).  Output order
 * [c00, c11, c22, c01, c02, c12].  gap = (l1 - l0) / max(l2, tiny) flags
 * neighbourhoods whose plane is ill-defined.
 */
static void *cov_worker(void *arg) {
  cov_job *j = (cov_job *)arg;
  u32_vec found = {0};
  const float r2 = j->radius * j->radius;
  for (size_t i = j->start; i < j->end; ++i) {
    found.len = 0;
    if (j->tree->root != KD_INVALID)
      kd_radius(j->tree, j->tree->root, j->x[i], j->y[i], j->z[i], r2, &found);
    double *o = j->cov + 6 * i;
    j->counts[i] = (uint32_t)found.len;
    j->gap[i] = 0.0;
    if (found.len < 3) {
      o[0] = o[1] = o[2] = j->eps;
      o[3] = o[4] = o[5] = 0.0;
      continue;
    }
    double mx = 0, my = 0, mz = 0;
    for (size_t k = 0; k < found.len; ++k) {
      uint32_t p = found.idx[k];
      mx += j->x[p];
      my += j->y[p];
      mz += j->z[p];
    }
    mx /= (double)found.len;
    my /= (double)found.len;
    mz /= (double)found.len;
    double c[3][3] = {{0}};
    for (size_t k = 0; k < found.len; ++k) {
      uint32_t p = found.idx[k];
      double dx = j->x[p] - mx, dy = j->y[p] - my, dz = j->z[p] - mz;
      c[0][0] += dx * dx;
      c[1][1] += dy * dy;
      c[2][2] += dz * dz;
      c[0][1] += dx * dy;
      c[0][2] += dx * dz;
      c[1][2] += dy * dz;
    }
    c[1][0] = c[0][1];
    c[2][0] = c[0][2];
    c[2][1] = c[1][2];
    double vals[3], vecs[3][3];
    rs_symmetric_eigen3(c, vals, vecs, 200, 1e-300);
    double reg[6] = {0, 0, 0, 0, 0, 0};
    for (int col = 0; col < 3; ++col) {
      const double lam = col == 0 ? j->eps : 1.0;
      const double ax = vecs[0][col], ay = vecs[1][col], az = vecs[2][col];
      reg[0] += lam * ax * ax;
      reg[1] += lam * ay * ay;
      reg[2] += lam * az * az;
      reg[3] += lam * ax * ay;
      reg[4] += lam * ax * az;
      reg[5] += lam * ay * az;
    }
    memcpy(o, reg, sizeof(reg));
    double top = fabs(vals[2]) > 1e-300 ? fabs(vals[2]) : 1e-300;
    j->gap[i] = (vals[1] - vals[0]) / top;
  }
  free(found.idx);
  return NULL;
}

int oracle_plane_covariances(const float *x, const float *y, const float *z, size_t n,
                             float radius, double eps, int threads, double *cov, double *gap,
                             uint32_t *counts) {
  if (n == 0) return OR_OK;
  if (!(radius > 0.0f)) return OR_ERR_INVALID; /* covariances_grid.rs:231-233 */
  kd_tree tree;
  if (kd_build(&tree, x, y, z, n) != OR_OK) return OR_ERR_NOMEM;
  size_t avail = threads > 0 ? (size_t)threads : (size_t)sysconf(_SC_NPROCESSORS_ONLN);
  size_t workers = n < 4096 ? 1 : (avail < n / 1024 ? avail : (n / 1024 ? n / 1024 : 1));
  size_t chunk = (n + workers - 1) / workers;
  size_t njobs = (n + chunk - 1) / chunk;
  cov_job *jobs = (cov_job *)calloc(njobs, sizeof(cov_job));
  pthread_t *tids = (pthread_t *)calloc(njobs, sizeof(pthread_t));
  for (size_t w = 0; w < njobs; ++w) {
    cov_job *j = &jobs[w];
    j->tree = &tree;
    j->x = x;
    j->y = y;
    j->z = z;
    j->start = w * chunk;
    j->end = j->start + chunk < n ? j->start + chunk : n;
    j->radius = radius;
    j->eps = eps;
    j->cov = cov;
    j->gap = gap;
    j->counts = counts;
  }
  if (njobs == 1) {
    cov_worker(&jobs[0]);
  } else {
    for (size_t w = 0; w < njobs; ++w) pthread_create(&tids[w], NULL, cov_worker, &jobs[w]);
    for (size_t w = 0; w < njobs; ++w) pthread_join(tids[w], NULL);
  }
  free(jobs);
  free(tids);
  kd_free(&tree);
  return OR_OK;
}

/* ------------------------------------------------------------------------ */
/* Bounded streaming voxel (crates/spatialrust-pipeline/src/streaming.rs)    */
/* ------------------------------------------------------------------------ */

#define OR_ERR_KEY_RANGE (-4)

typedef struct {
  int64_t k[3];
  uint64_t src; /* stream offset: ties keep stream order (:805-838) */
} sv_item;

static int cmp_sv_item(const void *a, const void *b) {
  const sv_item *x = (const sv_item *)a, *y = (const sv_item *)b;
  for (int i = 0; i < 3; ++i) {
    if (x->k[i] < y->k[i]) return -1;
    if (x->k[i] > y->k[i]) return 1;
  }
  return x->src < y->src ? -1 : (x->src > y->src ? 1 : 0);
}

/* voxel_coordinate (:986-994): floor(value / leaf) in f64; out of the i64
 * range is an error; 2^63 saturates like `as i64`. */
static int sv_coordinate(double value, double leaf, int64_t *out) {
  double c = floor(value / leaf);
  if (c < -9223372036854775808.0 || c > 9223372036854775808.0) return 0;
  *out = c >= 9223372036854775808.0 ? INT64_MAX : (int64_t)c;
  return 1;
}

/*
 * StreamingVoxelSource over the whole stream at once (the result does not
 * depend on the chunk or run sizes, :1099-1130): points with a non-finite
 * coordinate are skipped (:464-466), keys by voxel_coordinate, every field
 * summed per voxel in stream order with CompensatedSum (:240-262, 852-858),
 * value sum / count (:631-633), voxels in ascending key order.  Fields are
 * x, y, z (f32) and n_attrs FP64 attribute columns.  Outputs (capacity n):
 * keys (3 per voxel), counts, positions as f32, attribute means in FP64.
 * Returns the voxel count, or OR_ERR_KEY_RANGE.
 */
long long oracle_stream_voxel(const float *x, const float *y, const float *z,
                              const double *const *attrs, int n_attrs, size_t n, float leaf_f32,
                              int64_t *out_keys, uint64_t *out_counts, float *out_pos,
                              double *out_attrs) {
  const double leaf = (double)leaf_f32;
  sv_item *items = (sv_item *)malloc((n ? n : 1) * sizeof(sv_item));
  if (!items) return OR_ERR_NOMEM;
  size_t m = 0;
  for (size_t i = 0; i < n; ++i) {
    const double p[3] = {(double)x[i], (double)y[i], (double)z[i]};
    if (!isfinite(p[0]) || !isfinite(p[1]) || !isfinite(p[2])) continue;
    for (int a = 0; a < 3; ++a)
      if (!sv_coordinate(p[a], leaf, &items[m].k[a])) {
        free(items);
        return OR_ERR_KEY_RANGE;
      }
    items[m].src = i;
    m++;
  }
  qsort(items, m, sizeof(sv_item), cmp_sv_item);
  const int nf = 3 + n_attrs;
  long long v = 0;
  size_t s = 0;
  while (s < m) {
    size_t e = s + 1;
    while (e < m && memcmp(items[e].k, items[s].k, sizeof(items[s].k)) == 0) e++;
    for (int f = 0; f < nf; ++f) {
      double sum = 0.0, corr = 0.0; /* CompensatedSum */
      for (size_t t = s; t < e; ++t) {
        const size_t i = items[t].src;
        const double val = f == 0 ? (double)x[i] : f == 1 ? (double)y[i] : f == 2 ? (double)z[i]
                                                                               : attrs[f - 3][i];
        const double corrected = val - corr;
        const double next = sum + corrected;
        corr = (next - sum) - corrected;
        sum = next;
      }
      const double mean = sum / (double)(e - s);
      if (f < 3) out_pos[3 * v + f] = (float)mean;
      else out_attrs[(size_t)n_attrs * v + (f - 3)] = mean;
    }
    memcpy(&out_keys[3 * v], items[s].k, sizeof(items[s].k));
    out_counts[v] = e - s;
    v++;
    s = e;
  }
  free(items);
  return v;
}

/* ------------------------------------------------------------------------ */
/* LAS point records (crates/spatialrust-io/src/las/reader.rs:242-279)       */
/* ------------------------------------------------------------------------ */

static uint32_t le_u32(const uint8_t *p) {
  return (uint32_t)p[0] | ((uint32_t)p[1] << 8) | ((uint32_t)p[2] << 16) | ((uint32_t)p[3] << 24);
}
static uint16_t le_u16(const uint8_t *p) { return (uint16_t)(p[0] | (p[1] << 8)); }

/*
 * The fields read_las keeps, from uncompressed point records of formats 0-10
 * (ASPRS LAS 1.4 R15 tables 7-17; the reference delegates the byte layout to
 * the `las` crate 0.9): x = (f32)(scale * X + offset [- origin]) with the
 * f64 products and sums rounded step by step, intensity as f32,
 * classification (low 5 bits of byte 15 for formats 0-5, byte 16 for 6-10),
 * gps_time (f64 at byte 20, or 22 for formats 6-10), red/green/blue (u16 at
 * byte 20 for format 2, 28 for 3 and 5, 30 for 7, 8 and 10).  rgb holds 3
 * columns of n.  Returns 0, or OR_ERR_INVALID for an unknown format.
 */
int oracle_las_decode(const uint8_t *rec, size_t n, int format, int record_length,
                      const double *scale, const double *offset, int has_origin,
                      const double *origin, float *x, float *y, float *z, float *intensity,
                      uint8_t *cls, double *gps, uint16_t *rgb) {
  static const int gps_off[11] = {-1, 20, -1, 20, 20, 20, 22, 22, 22, 22, 22};
  static const int rgb_off[11] = {-1, -1, 20, 28, -1, 28, -1, 30, 30, -1, 30};
  if (format < 0 || format > 10) return OR_ERR_INVALID;
  float *pos[3] = {x, y, z};
  for (size_t i = 0; i < n; ++i) {
    const uint8_t *r = rec + i * (size_t)record_length;
    for (int a = 0; a < 3; ++a) {
      const int32_t raw = (int32_t)le_u32(r + 4 * a);
      double v = scale[a] * (double)raw;
      v = v + offset[a];
      if (has_origin) v = v - origin[a];
      pos[a][i] = (float)v;
    }
    intensity[i] = (float)le_u16(r + 12);
    cls[i] = format >= 6 ? r[16] : (uint8_t)(r[15] & 0x1f);
    if (gps_off[format] >= 0) {
      uint64_t bits = (uint64_t)le_u32(r + gps_off[format]) |
                      ((uint64_t)le_u32(r + gps_off[format] + 4) << 32);
      memcpy(&gps[i], &bits, 8);
    }
    if (rgb_off[format] >= 0)
      for (int c = 0; c < 3; ++c) rgb[c * n + i] = le_u16(r + rgb_off[format] + 2 * c);
  }
  return OR_OK;
}

/* ------------------------------------------------------------------------ */
/* RANSAC plane segmentation (crates/spatialrust-segmentation/src/plane.rs,  */
/* plane_ransac.rs)                                                          */
/* ------------------------------------------------------------------------ */

typedef struct {
  uint64_t state;
} or_rng;

/* Rng (plane_ransac.rs:7-25) */
static uint64_t or_rng_next(or_rng *r) {
  r->state = r->state * 6364136223846793005ull + 1ull;
  return r->state;
}
static uint64_t or_rng_index(or_rng *r, uint64_t upper) {
  return ((or_rng_next(r) >> 32) * upper) >> 32;
}

/* plane_from_points (plane_ransac.rs:79-89), f32; returns 0 for None. */
static int or_plane(const float *x, const float *y, const float *z, const uint32_t idx[3],
                    float plane[4]) {
  const float p0x = x[idx[0]], p0y = y[idx[0]], p0z = z[idx[0]];
  const float v1x = x[idx[1]] - p0x, v1y = y[idx[1]] - p0y, v1z = z[idx[1]] - p0z;
  const float v2x = x[idx[2]] - p0x, v2y = y[idx[2]] - p0y, v2z = z[idx[2]] - p0z;
  float nx = v1y * v2z - v1z * v2y;
  float ny = v1z * v2x - v1x * v2z;
  float nz = v1x * v2y - v1y * v2x;
  const float ls = nx * nx + ny * ny + nz * nz;
  if (ls < 1e-12f) return 0;
  const float len = sqrtf(ls);
  if (len != 0.0f) {
    nx = nx / len;
    ny = ny / len;
    nz = nz / len;
  }
  plane[0] = nx;
  plane[1] = ny;
  plane[2] = nz;
  plane[3] = -(nx * p0x + ny * p0y + nz * p0z);
  return 1;
}

/* distance_xyz (plane.rs:39-41) <= threshold */
static int or_inlier(const float p[4], float x, float y, float z, float thr) {
  return fabsf(p[0] * x + p[1] * y + p[2] * z + p[3]) <= thr;
}

/*
 * RansacPlaneSegmenter::segment_cpu + finalize_plane_segmentation
 * (plane.rs:266-345): hypotheses from the seeded LCG (sample_indices,
 * plane_ransac.rs:27-43), the first plane with the most inliers, then
 * refine_plane_from_inliers (plane_ransac.rs:96-150: FP64 sequential means and
 * covariance, symmetric_eigen3, f32 normal normalized, d = -n.c).  Returns the
 * inlier count (mask: n bytes) and writes the model, or -1 (empty), -2 (< 3
 * points), -5 (fewer than min_inliers), -6 (no model).
 */
long long oracle_ransac_plane(const float *x, const float *y, const float *z, size_t n, float thr,
                              uint32_t max_iterations, uint64_t min_inliers, uint64_t seed,
                              float model[4], float hyp_model[4], uint32_t *best_index,
                              uint8_t *mask) {
  if (n == 0) return -1;
  if (n < 3) return -2;
  or_rng rng = {seed ? seed : 1};
  long long best = 0;
  int have = 0;
  *best_index = UINT32_MAX;
  for (uint32_t it = 0; it < max_iterations; ++it) {
    uint32_t idx[3];
    idx[0] = (uint32_t)or_rng_index(&rng, n);
    idx[1] = (uint32_t)or_rng_index(&rng, n);
    while (idx[1] == idx[0]) idx[1] = (uint32_t)or_rng_index(&rng, n);
    idx[2] = (uint32_t)or_rng_index(&rng, n);
    while (idx[2] == idx[0] || idx[2] == idx[1]) idx[2] = (uint32_t)or_rng_index(&rng, n);
    float pl[4];
    if (!or_plane(x, y, z, idx, pl)) continue;
    long long c = 0;
    for (size_t i = 0; i < n; ++i) c += or_inlier(pl, x[i], y[i], z[i], thr);
    if (c > best) {
      best = c;
      have = 1;
      memcpy(hyp_model, pl, sizeof(pl));
      *best_index = it;
    }
  }
  if ((uint64_t)best < min_inliers) return -5;
  if (!have) return -6;
  double mx = 0, my = 0, mz = 0;
  for (size_t i = 0; i < n; ++i) {
    mask[i] = (uint8_t)or_inlier(hyp_model, x[i], y[i], z[i], thr);
    if (mask[i]) {
      mx += (double)x[i];
      my += (double)y[i];
      mz += (double)z[i];
    }
  }
  memcpy(model, hyp_model, 4 * sizeof(float));
  if (best < 3) return best;
  const double cnt = (double)best;
  mx /= cnt;
  my /= cnt;
  mz /= cnt;
  double c[6] = {0, 0, 0, 0, 0, 0};
  for (size_t i = 0; i < n; ++i) {
    if (!mask[i]) continue;
    const double dx = (double)x[i] - mx, dy = (double)y[i] - my, dz = (double)z[i] - mz;
    c[0] += dx * dx;
    c[1] += dy * dy;
    c[2] += dz * dz;
    c[3] += dx * dy;
    c[4] += dx * dz;
    c[5] += dy * dz;
  }
  const double inv = 1.0 / cnt;
  const double cov[3][3] = {{c[0] * inv, c[3] * inv, c[4] * inv},
                            {c[3] * inv, c[1] * inv, c[5] * inv},
                            {c[4] * inv, c[5] * inv, c[2] * inv}};
  double vals[3], vecs[3][3];
  rs_symmetric_eigen3(cov, vals, vecs, 32, 1e-12);
  float nx = (float)vecs[0][0], ny = (float)vecs[1][0], nz = (float)vecs[2][0];
  const float len = sqrtf(nx * nx + ny * ny + nz * nz);
  if (len != 0.0f) {
    nx = nx / len;
    ny = ny / len;
    nz = nz / len;
  }
  const float cx = (float)mx, cy = (float)my, cz = (float)mz;
  model[0] = nx;
  model[1] = ny;
  model[2] = nz;
  model[3] = -(nx * cx + ny * cy + nz * cz);
  return best;
}

/* Exposes the f32 closed-form smallest eigenpair for unit tests. */
void oracle_smallest_eigenpair_f32(const float c[6], float normal[3], float *curv) {
  rs_smallest_eigenpair(c[0], c[1], c[2], c[3], c[4], c[5], normal, curv);
}

int oracle_abi_version(void) { return 1; }
