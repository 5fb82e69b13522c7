// ransac.cu -- host side of the RANSAC plane entry points (include/srcuda.h).
// Included at the end of srcuda.cu.
//
// srcu_ransac_plane_segment follows RansacPlaneSegmenter::segment_cpu and
// finalize_plane_segmentation (crates/spatialrust-segmentation/src/
// plane.rs:266-345): hypotheses from the reference's LCG (plane_ransac.rs:
// 7-43), every hypothesis scored on the device, the first hypothesis with the
// largest count wins (the CPU loop keeps a candidate only when it has strictly
// more inliers), its inliers are the answer, and the model is refined from
// them in FP64 (refine_plane_from_inliers, plane_ransac.rs:96-150) with the
// reference's Jacobi eigensolver (crates/spatialrust-math/src/eigen.rs:16-84).
#include <cmath>

#include "ransac.cuh"

namespace {

// Rng (plane_ransac.rs:7-25): 64-bit LCG, state = max(seed, 1).
struct RansacRng {
  uint64_t state;
  explicit RansacRng(uint64_t seed) : state(seed ? seed : 1) {}
  uint64_t next_u64() {
    state = state * 6364136223846793005ull + 1ull;
    return state;
  }
  uint64_t next_index(uint64_t upper) { return ((next_u64() >> 32) * upper) >> 32; }
};

// sample_indices (plane_ransac.rs:27-43) for len >= 3.
void sample_indices(RansacRng &rng, uint64_t len, uint32_t *out) {
  const uint64_t a = rng.next_index(len);
  uint64_t b = rng.next_index(len);
  while (b == a) b = rng.next_index(len);
  uint64_t c = rng.next_index(len);
  while (c == a || c == b) c = rng.next_index(len);
  out[0] = uint32_t(a);
  out[1] = uint32_t(b);
  out[2] = uint32_t(c);
}

double rs_signum(double v) { return std::signbit(v) ? -1.0 : 1.0; }  // f64::signum (NaN aside)

// symmetric_eigen3 (eigen.rs:16-84): cyclic-max Jacobi, 32 rotations at most,
// stop when the largest off-diagonal is below 1e-12; eigenvectors as columns
// sorted by ascending eigenvalue (a stable sort).
void jacobi_eigen3(const double (&m)[3][3], double (&vals)[3], double (&vecs)[3][3]) {
  double a[3][3], v[3][3] = {{1, 0, 0}, {0, 1, 0}, {0, 0, 1}};
  memcpy(a, m, sizeof(a));
  for (int it = 0; it < 32; ++it) {
    int p = 0, q = 1;
    double mx = std::fabs(a[0][1]);
    if (std::fabs(a[0][2]) > mx) {
      mx = std::fabs(a[0][2]);
      p = 0;
      q = 2;
    }
    if (std::fabs(a[1][2]) > mx) {
      mx = std::fabs(a[1][2]);
      p = 1;
      q = 2;
    }
    if (mx < 1e-12) break;
    const double app = a[p][p], aqq = a[q][q], apq = a[p][q];
    const double phi = 0.5 * (aqq - app) / apq;
    const double t = rs_signum(phi) / (std::fabs(phi) + std::sqrt(1.0 + phi * phi));
    const double c = 1.0 / std::sqrt(1.0 + t * t);
    const double s = t * c;
    const double app_new = c * c * app - 2.0 * s * c * apq + s * s * aqq;
    const double aqq_new = s * s * app + 2.0 * s * c * apq + c * c * aqq;
    a[p][p] = app_new;
    a[q][q] = aqq_new;
    a[p][q] = 0.0;
    a[q][p] = 0.0;
    for (int r = 0; r < 3; ++r) {
      if (r != p && r != q) {
        const double arp = a[r][p], arq = a[r][q];
        a[r][p] = c * arp - s * arq;
        a[p][r] = a[r][p];
        a[r][q] = s * arp + c * arq;
        a[q][r] = a[r][q];
      }
    }
    for (int r = 0; r < 3; ++r) {
      const double vp = v[r][p], vq = v[r][q];
      v[r][p] = c * vp - s * vq;
      v[r][q] = s * vp + c * vq;
    }
  }
  const double ev[3] = {a[0][0], a[1][1], a[2][2]};
  int order[3] = {0, 1, 2};
  for (int i = 1; i < 3; ++i)  // stable insertion sort
    for (int j = i; j > 0 && ev[order[j]] < ev[order[j - 1]]; --j) std::swap(order[j], order[j - 1]);
  for (int i = 0; i < 3; ++i) {
    vals[i] = ev[order[i]];
    for (int r = 0; r < 3; ++r) vecs[r][i] = v[r][order[i]];
  }
}

srcu_status ransac_reserve(srcu_ctx *ctx, uint32_t count, uint32_t grid_m) {
  ST_TRY(ensure(ctx, ctx->rs_hyp, size_t(std::max<uint32_t>(count, 1)) * 12));
  ST_TRY(ensure(ctx, ctx->rs_planes, size_t(std::max<uint32_t>(count, 1)) * 16));
  ST_TRY(ensure(ctx, ctx->rs_valid, size_t(std::max<uint32_t>(count, 1)) * 4));
  ST_TRY(ensure(ctx, ctx->rs_counts, size_t(std::max<uint32_t>(count, 1)) * 4));
  ST_TRY(ensure(ctx, ctx->rs_partials, size_t(grid_m) * 6 * 8));
  return SRCU_OK;
}

// Stages the positions and scores `count` hypotheses (host triples); leaves
// planes, validity and counts on the device and copies them to the host.
srcu_status ransac_score(srcu_ctx *ctx, const srcu_cloud *cloud, const float **cols,
                         const uint32_t *hyp_host, uint32_t count, float thr,
                         std::vector<float4> &planes, std::vector<uint32_t> &valid,
                         std::vector<uint32_t> &counts) {
  const uint64_t n = cloud->n;
  CU_TRY(cudaMemcpyAsync(ctx->rs_hyp.p, hyp_host, size_t(count) * 12, cudaMemcpyHostToDevice,
                         ctx->stream));
  CU_TRY(cudaMemsetAsync(ctx->rs_counts.p, 0, size_t(count) * 4, ctx->stream));
  uint32_t *status = &ctx->ctl->status;
  CU_TRY(cudaMemsetAsync(status, 0, sizeof(uint32_t), ctx->stream));
  {
    Launch l(ctx, SRCU_K_RANSAC);
    k_ransac_planes<<<ceil_div(count, 256), 256, 0, ctx->stream>>>(
        cols[0], cols[1], cols[2], n, ptr<const uint32_t>(ctx->rs_hyp), count,
        ptr<float4>(ctx->rs_planes), ptr<uint32_t>(ctx->rs_valid), status);
    // enough blocks for every SM: point tiles x hypothesis chunks (>= 32 planes each)
    const uint32_t tiles = std::max<uint32_t>(1, ceil_div(n, RS_TILE));
    const uint32_t want = uint32_t(ctx->num_sms) * 8;
    const uint32_t chunks = std::max<uint32_t>(
        1, std::min<uint32_t>(ceil_div(count, 32), ceil_div(want, tiles)));
    const uint32_t per_chunk = ceil_div(count, chunks);
    k_ransac_score<<<dim3(tiles, ceil_div(count, per_chunk)), RS_THREADS, 0, ctx->stream>>>(
        cols[0], cols[1], cols[2], n, ptr<const float4>(ctx->rs_planes), count, per_chunk, thr,
        ptr<uint32_t>(ctx->rs_counts));
  }
  CU_TRY(cudaGetLastError());
  planes.resize(count);
  valid.resize(count);
  counts.resize(count);
  CU_TRY(cudaMemcpyAsync(planes.data(), ctx->rs_planes.p, size_t(count) * 16, cudaMemcpyDeviceToHost,
                         ctx->stream));
  CU_TRY(cudaMemcpyAsync(valid.data(), ctx->rs_valid.p, size_t(count) * 4, cudaMemcpyDeviceToHost,
                         ctx->stream));
  CU_TRY(cudaMemcpyAsync(counts.data(), ctx->rs_counts.p, size_t(count) * 4, cudaMemcpyDeviceToHost,
                         ctx->stream));
  CU_TRY(cudaMemcpyAsync(&ctx->ctl_host->status, status, sizeof(uint32_t), cudaMemcpyDeviceToHost,
                         ctx->stream));
  CU_TRY(cudaStreamSynchronize(ctx->stream));
  if (ctx->ctl_host->status)
    return fail(ctx, SRCU_ERR_CUDA, "internal consistency check failed on the device (status 0x%x)",
                ctx->ctl_host->status);
  return SRCU_OK;
}

srcu_status ransac_stage(srcu_ctx *ctx, const srcu_cloud *cloud, const float **cols) {
  ST_TRY(reserve(ctx, cloud->n, 3, needs_staging(cloud), false, false));
  srcu_cloud xyz = *cloud;
  xyz.n_attrs = 0;
  return stage_input(ctx, &xyz, cols);
}

}  // namespace

extern "C" {

srcu_status srcu_ransac_plane_scores(srcu_ctx *ctx, const srcu_cloud *cloud,
                                     const uint32_t *hypotheses, uint32_t count,
                                     float distance_threshold, srcu_plane_score *scores) {
  if (!ctx) return SRCU_ERR_INVALID_ARGUMENT;
  ST_TRY(check_cloud(ctx, cloud));
  if (count == 0) return SRCU_OK;  // ransac_plane.rs:124-126
  if (!hypotheses || !scores) return fail(ctx, SRCU_ERR_MISSING_FIELD, "hypotheses or scores are NULL");
  for (uint64_t k = 0; k < uint64_t(count) * 3; ++k)
    if (hypotheses[k] >= cloud->n)
      return fail(ctx, SRCU_ERR_INVALID_ARGUMENT, "hypothesis index %u is out of range (%llu points)",
                  hypotheses[k], (unsigned long long)cloud->n);
  CU_TRY(cudaSetDevice(ctx->device));
  const float *cols[MAX_COLS];
  ST_TRY(ransac_stage(ctx, cloud, cols));
  ST_TRY(ransac_reserve(ctx, count, 1));
  std::vector<float4> planes;
  std::vector<uint32_t> valid, counts;
  ST_TRY(ransac_score(ctx, cloud, cols, hypotheses, count, distance_threshold, planes, valid,
                      counts));
  for (uint32_t h = 0; h < count; ++h) {
    scores[h].inlier_count = valid[h] ? counts[h] : 0;
    scores[h].normal[0] = planes[h].x;
    scores[h].normal[1] = planes[h].y;
    scores[h].normal[2] = planes[h].z;
    scores[h].d = planes[h].w;
  }
  return SRCU_OK;
}

srcu_status srcu_ransac_plane_segment(srcu_ctx *ctx, const srcu_cloud *cloud,
                                      const srcu_ransac_params *params, srcu_ransac_result *result,
                                      uint8_t *inlier_mask) {
  if (!ctx) return SRCU_ERR_INVALID_ARGUMENT;
  if (result) memset(result, 0, sizeof(*result));
  ST_TRY(check_cloud(ctx, cloud));
  if (!params || !result) return fail(ctx, SRCU_ERR_INVALID_ARGUMENT, "params or result is NULL");
  const uint64_t n = cloud->n;
  if (n == 0)  // plane.rs:267-271
    return fail(ctx, SRCU_ERR_INVALID_ARGUMENT, "cannot segment plane from empty point cloud");
  if (n < 3)  // plane.rs:274-278
    return fail(ctx, SRCU_ERR_INVALID_ARGUMENT, "plane segmentation requires at least three points");
  if (params->max_iterations > (1u << 26))
    return fail(ctx, SRCU_ERR_INVALID_ARGUMENT, "max_iterations %u exceeds 2^26",
                params->max_iterations);
  CU_TRY(cudaSetDevice(ctx->device));
  const uint32_t count = params->max_iterations;
  std::vector<uint32_t> hyp(size_t(std::max<uint32_t>(count, 1)) * 3);
  RansacRng rng(params->seed);
  for (uint32_t h = 0; h < count; ++h) sample_indices(rng, n, &hyp[3 * size_t(h)]);
  const float *cols[MAX_COLS];
  ST_TRY(ransac_stage(ctx, cloud, cols));
  const uint32_t grid_m = std::max<uint32_t>(1, std::min<uint32_t>(ceil_div(n, RM_THREADS),
                                                                    uint32_t(ctx->num_sms) * 2));
  ST_TRY(ransac_reserve(ctx, count, grid_m));
  std::vector<float4> planes;
  std::vector<uint32_t> valid, counts;
  if (count) ST_TRY(ransac_score(ctx, cloud, cols, hyp.data(), count, params->distance_threshold,
                                 planes, valid, counts));
  // the CPU loop: a candidate replaces the best only with strictly more inliers
  int64_t best = -1;
  uint32_t best_count = 0;
  for (uint32_t h = 0; h < count; ++h)
    if (valid[h] && counts[h] > best_count) {
      best = h;
      best_count = counts[h];
    }
  result->hypotheses = count;
  result->best_hypothesis = best < 0 ? UINT32_MAX : uint32_t(best);
  result->inlier_count = best_count;
  if (best_count < params->min_inliers)  // plane.rs:318-324
    return fail(ctx, SRCU_ERR_INVALID_ARGUMENT, "RANSAC found only %u inliers, minimum is %llu",
                best_count, (unsigned long long)params->min_inliers);
  if (best < 0)  // min_inliers == 0 and no plane with an inlier: no model to refine (:326-328)
    return fail(ctx, SRCU_ERR_INVALID_ARGUMENT, "failed to refine plane model");
  const float4 bp = planes[size_t(best)];
  result->hypothesis_normal[0] = bp.x;
  result->hypothesis_normal[1] = bp.y;
  result->hypothesis_normal[2] = bp.z;
  result->hypothesis_d = bp.w;
  // inlier mask + FP64 sums (pass 0), centred moments (pass 1)
  uint8_t *mask_dev = nullptr;
  if (inlier_mask && cloud->on_device) {
    mask_dev = inlier_mask;
  } else if (inlier_mask) {
    ST_TRY(ensure(ctx, ctx->rs_mask, n));
    mask_dev = ptr<uint8_t>(ctx->rs_mask);
  }
  const float4 *plane_dev = ptr<const float4>(ctx->rs_planes) + best;
  std::vector<double> part(size_t(grid_m) * 6);
  {
    Launch l(ctx, SRCU_K_RANSAC);
    k_ransac_moments<<<grid_m, RM_THREADS, 0, ctx->stream>>>(
        cols[0], cols[1], cols[2], n, plane_dev, params->distance_threshold, mask_dev, 0,
        make_double3(0, 0, 0), ptr<double>(ctx->rs_partials));
  }
  CU_TRY(cudaGetLastError());
  CU_TRY(cudaMemcpyAsync(part.data(), ctx->rs_partials.p, part.size() * 8, cudaMemcpyDeviceToHost,
                         ctx->stream));
  CU_TRY(cudaStreamSynchronize(ctx->stream));
  double cnt = 0, sx = 0, sy = 0, sz = 0;
  for (uint32_t b = 0; b < grid_m; ++b) {
    cnt += part[6 * b];
    sx += part[6 * b + 1];
    sy += part[6 * b + 2];
    sz += part[6 * b + 3];
  }
  if (uint64_t(cnt) != best_count)
    return fail(ctx, SRCU_ERR_CUDA, "inlier recount %llu differs from the score %u",
                (unsigned long long)cnt, best_count);
  float model[4] = {bp.x, bp.y, bp.z, bp.w};
  if (best_count >= 3) {  // refine_plane_from_inliers (plane_ransac.rs:96-150)
    const double mean[3] = {sx / cnt, sy / cnt, sz / cnt};
    {
      Launch l(ctx, SRCU_K_RANSAC);
      k_ransac_moments<<<grid_m, RM_THREADS, 0, ctx->stream>>>(
          cols[0], cols[1], cols[2], n, plane_dev, params->distance_threshold, nullptr, 1,
          make_double3(mean[0], mean[1], mean[2]), ptr<double>(ctx->rs_partials));
    }
    CU_TRY(cudaGetLastError());
    CU_TRY(cudaMemcpyAsync(part.data(), ctx->rs_partials.p, part.size() * 8,
                           cudaMemcpyDeviceToHost, ctx->stream));
    CU_TRY(cudaStreamSynchronize(ctx->stream));
    double c6[6] = {0, 0, 0, 0, 0, 0};  // c00 c11 c22 c01 c02 c12
    for (uint32_t b = 0; b < grid_m; ++b)
      for (int k = 0; k < 6; ++k) c6[k] += part[6 * b + k];
    const double inv = 1.0 / cnt;
    const double cov[3][3] = {{c6[0] * inv, c6[3] * inv, c6[4] * inv},
                              {c6[3] * inv, c6[1] * inv, c6[5] * inv},
                              {c6[4] * inv, c6[5] * inv, c6[2] * inv}};
    double vals[3], vecs[3][3];
    jacobi_eigen3(cov, vals, vecs);
    // the f32 normal, normalized in f32; centroid as f32; d = -n.c (Vec3<f32>)
    float nx = float(vecs[0][0]), ny = float(vecs[1][0]), nz = float(vecs[2][0]);
    const float len = std::sqrt(nx * nx + ny * ny + nz * nz);
    if (len != 0.0f) {
      nx /= len;
      ny /= len;
      nz /= len;
    }
    const float cx = float(mean[0]), cy = float(mean[1]), cz = float(mean[2]);
    model[0] = nx;
    model[1] = ny;
    model[2] = nz;
    model[3] = -(nx * cx + ny * cy + nz * cz);
  }
  for (int a = 0; a < 3; ++a) result->normal[a] = model[a];
  result->d = model[3];
  if (inlier_mask && !cloud->on_device) ST_TRY(copy_out(ctx, inlier_mask, mask_dev, n, 0));
  CU_TRY(cudaStreamSynchronize(ctx->stream));
  return SRCU_OK;
}

}  // extern "C"
