// stream.cu -- host side of the bounded streaming voxel (srcu_stream_voxel_*,
// include/srcuda.h).  Included at the end of srcuda.cu: it drives the
// context's sort buffers and control block like the other chains.
//
// Mirrors StreamingVoxelSource::try_build / next_chunk
// (crates/spatialrust-pipeline/src/streaming.rs:414-535, 594-676):
//   push()    appends a chunk to the device run buffer; a full buffer is a run:
//             bounds -> plan -> onesweep sort -> segment reduction into partial
//             records (key, count, compensated FP64 column sums);
//   finish()  reduces the last run, checks the reference's run and spool
//             limits, sorts every partial record by key and reduces again;
//   fetch()   copies a window of the final voxels (next_chunk's chunks).
#include "stream.cuh"

struct srcu_stream_voxel {
  srcu_ctx *ctx = nullptr;
  srcu_stream_voxel_params prm{};
  uint32_t nc = 3;
  double leaf = 0.0;
  uint64_t dev_run = 0;   // points per device run
  uint64_t fill = 0;      // points in the run buffer
  uint64_t points = 0;    // points pushed
  uint64_t device_runs = 0;
  uint64_t records = 0;   // partial records stored
  uint64_t rec_cap = 0;
  uint64_t voxels = 0;
  bool finished = false;
  int occ_point = 1, occ_record = 1;
  DevBuf run[MAX_COLS];                       // run buffer, 4 or 8 bytes per element
  DevBuf rk[3], rcnt, rsum[MAX_COLS];          // partial records
  DevBuf fk[3], fcnt, fsum[MAX_COLS];          // final records
  DevBuf opos[3], oattr[MAX_COLS], okeys;      // finished outputs
  DevBuf tile_heads, tile_off, long_list, plan, state;
  StreamState *state_host = nullptr;           // pinned
};

namespace {

uint32_t sv_elem(const srcu_stream_voxel *sv, uint32_t c) {
  return (c >= 3 && ((sv->prm.attr_f64_mask >> (c - 3)) & 1u)) ? 8u : 4u;
}

// Grows a device buffer to `bytes`, keeping its first `keep` bytes.
srcu_status grow_keep(srcu_ctx *ctx, DevBuf &b, size_t bytes, size_t keep) {
  if (b.bytes >= bytes) return SRCU_OK;
  DevBuf nb;
  ST_TRY(ensure(ctx, nb, bytes));
  if (keep && b.p) CU_TRY(cudaMemcpyAsync(nb.p, b.p, keep, cudaMemcpyDeviceToDevice, ctx->stream));
  if (b.p) {
    CU_TRY(cudaStreamSynchronize(ctx->stream));
    release(ctx, b);
  }
  b = nb;
  return SRCU_OK;
}

srcu_status sv_reserve_records(srcu_stream_voxel *sv, uint64_t need) {
  if (need <= sv->rec_cap) return SRCU_OK;
  srcu_ctx *ctx = sv->ctx;
  const uint64_t cap = std::max<uint64_t>({need, 2 * sv->rec_cap, 4 * sv->dev_run});
  const size_t keep = size_t(sv->records) * 8;
  for (int a = 0; a < 3; ++a) ST_TRY(grow_keep(ctx, sv->rk[a], cap * 8, keep));
  ST_TRY(grow_keep(ctx, sv->rcnt, cap * 8, keep));
  for (uint32_t c = 0; c < sv->nc; ++c) ST_TRY(grow_keep(ctx, sv->rsum[c], cap * 8, keep));
  sv->rec_cap = cap;
  return SRCU_OK;
}

StreamOut sv_out(DevBuf (&k)[3], DevBuf &cnt, DevBuf *sum, uint32_t nc, uint64_t base, uint64_t cap) {
  StreamOut o{};
  o.kx = ptr<long long>(k[0]);
  o.ky = ptr<long long>(k[1]);
  o.kz = ptr<long long>(k[2]);
  o.cnt = ptr<unsigned long long>(cnt);
  for (uint32_t c = 0; c < nc; ++c) o.sum[c] = ptr<double>(sum[c]);
  o.base = base;
  o.cap = cap;
  return o;
}

// Segment reduction of the current sort (ctl->n_points = n sorted items).
template <bool Records>
srcu_status sv_reduce(srcu_stream_voxel *sv, uint64_t n, const StreamIn &in, const StreamOut &out,
                      int count_finite) {
  srcu_ctx *ctx = sv->ctx;
  const uint64_t tiles = std::max<uint64_t>(1, ceil_div(n, SV_TILE));
  const uint64_t long_cap = n / (SV_SHORT + 1) + 1;
  ST_TRY(ensure(ctx, sv->tile_heads, tiles * 4));
  ST_TRY(ensure(ctx, sv->tile_off, tiles * 4));
  ST_TRY(ensure(ctx, sv->long_list, long_cap * sizeof(ulonglong2)));
  const uint32_t grid = std::max<uint32_t>(
      1, std::min<uint32_t>(uint32_t(tiles), uint32_t(ctx->num_sms) * 8));
  StreamState *st = ptr<StreamState>(sv->state);
  const StreamPlan *pl = ptr<const StreamPlan>(sv->plan);
  Launch l(ctx, SRCU_K_VOXEL_SEGMENTS);
  k_stream_flags<<<grid, SV_THREADS, 0, ctx->stream>>>(ctx->ctl, sort_buffers(ctx), &ctx->ctl->vsort,
                                                       pl, ptr<uint32_t>(sv->tile_heads), st,
                                                       count_finite);
  k_stream_scan<<<1, 1024, 0, ctx->stream>>>(ctx->ctl, ptr<const uint32_t>(sv->tile_heads),
                                             ptr<uint32_t>(sv->tile_off), st);
  k_stream_emit<Records><<<grid, SV_THREADS, 0, ctx->stream>>>(
      ctx->ctl, sort_buffers(ctx), &ctx->ctl->vsort, pl, ptr<const uint32_t>(sv->tile_off), in, out,
      st, ptr<ulonglong2>(sv->long_list), uint32_t(std::min<uint64_t>(long_cap, 0xffffffffu)));
  k_stream_long<Records><<<uint32_t(ctx->num_sms) * 2, SV_THREADS, 0, ctx->stream>>>(
      ctx->ctl, sort_buffers(ctx), &ctx->ctl->vsort, pl, in, out, st,
      ptr<const ulonglong2>(sv->long_list));
  CU_TRY(cudaGetLastError());
  return SRCU_OK;
}

// Reads the stream state and the control block; maps a key overflow to the
// reference's error text when the key left the i64 range.
srcu_status sv_sync(srcu_stream_voxel *sv) {
  srcu_ctx *ctx = sv->ctx;
  CU_TRY(cudaMemcpyAsync(sv->state_host, sv->state.p, sizeof(StreamState), cudaMemcpyDeviceToHost,
                         ctx->stream));
  srcu_status s = read_control(ctx);
  if (s == SRCU_ERR_KEY_OVERFLOW) {
    if (sv->state_host->overflow == 1)
      return fail(ctx, SRCU_ERR_INVALID_ARGUMENT, "voxel coordinate exceeds signed 64-bit range");
    return fail(ctx, SRCU_ERR_KEY_OVERFLOW,
                "the stream's voxel keys span more than 63 bits when packed");
  }
  return s;
}

// Sorts and reduces the run buffer into partial records.
srcu_status sv_flush(srcu_stream_voxel *sv) {
  const uint64_t n = sv->fill;
  if (n == 0) return SRCU_OK;
  srcu_ctx *ctx = sv->ctx;
  ST_TRY(sv_reserve_records(sv, sv->records + n));
  ST_TRY(reserve(ctx, n, 0, false, false, false));
  ST_TRY(reserve_batch(ctx, 1));
  const Batch bt = make_batch(ctx, 1);
  ST_TRY(begin_chain(ctx, n, bt, 1, nullptr, nullptr));
  const float *x = ptr<const float>(sv->run[0]);
  const float *y = ptr<const float>(sv->run[1]);
  const float *z = ptr<const float>(sv->run[2]);
  {
    Launch l(ctx, SRCU_K_BOUNDS);
    const uint32_t grid = std::max<uint32_t>(1, std::min<uint32_t>(ceil_div(n, 256),
                                                                    uint32_t(ctx->num_sms) * 2));
    k_stream_bounds<<<grid, 256, 0, ctx->stream>>>(ctx->ctl, x, y, z, bt.bounds);
  }
  {
    Launch l(ctx, SRCU_K_VOXEL_PLAN);
    k_stream_plan<<<1, 32, 0, ctx->stream>>>(ctx->ctl, bt.bounds, sv->leaf,
                                             ptr<StreamPlan>(sv->plan), ptr<StreamState>(sv->state));
  }
  StreamPointSrc src{};
  src.x = x;
  src.y = y;
  src.z = z;
  src.plan_ptr = ptr<const StreamPlan>(sv->plan);
  src.leaf = sv->leaf;
  ST_TRY(launch_sort(ctx, src, n, ctx->ctl->hist_v, EP_VSORT, WK_VSORT, &ctx->ctl->vsort,
                     sv->occ_point, SRCU_K_VOXEL_SORT));
  StreamIn in{};
  in.nc = sv->nc;
  in.f64_mask = sv->prm.attr_f64_mask << 3;
  for (uint32_t c = 0; c < sv->nc; ++c) in.col[c] = sv->run[c].p;
  ST_TRY(sv_reduce<false>(sv, n, in,
                          sv_out(sv->rk, sv->rcnt, sv->rsum, sv->nc, sv->records, sv->rec_cap), 1));
  ST_TRY(sv_sync(sv));
  sv->records += sv->state_host->segments;
  sv->device_runs += 1;
  sv->fill = 0;
  return SRCU_OK;
}

srcu_status sv_finish(srcu_stream_voxel *sv) {
  srcu_ctx *ctx = sv->ctx;
  ST_TRY(sv_flush(sv));
  // The reference spills every finite point into runs of run_points
  // (streaming.rs:458-485): its run count and spool extent follow from the
  // finite-point count alone, and so do its two fail-closed limits.
  CU_TRY(cudaMemcpyAsync(sv->state_host, sv->state.p, sizeof(StreamState), cudaMemcpyDeviceToHost,
                         ctx->stream));
  CU_TRY(cudaStreamSynchronize(ctx->stream));
  const uint64_t finite = sv->state_host->finite;
  const uint64_t runs = (finite + sv->prm.run_points - 1) / sv->prm.run_points;
  if (runs > sv->prm.max_runs)
    return fail(ctx, SRCU_ERR_INVALID_ARGUMENT, "streaming voxel run limit %llu exceeded",
                (unsigned long long)sv->prm.max_runs);
  const uint64_t spool = runs * 8 + finite * (32 + 8 * uint64_t(sv->nc));
  if (sv->prm.spool_limit_bytes && spool > sv->prm.spool_limit_bytes)
    return fail(ctx, SRCU_ERR_INVALID_ARGUMENT, "spool limit exceeded: requested extent %llu, limit %llu",
                (unsigned long long)spool, (unsigned long long)sv->prm.spool_limit_bytes);
  const uint64_t r = sv->records;
  sv->voxels = 0;
  if (r == 0) return SRCU_OK;
  if (r > LB_MAX_COUNT)
    return fail(ctx, SRCU_ERR_INVALID_ARGUMENT, "%llu partial voxel records exceed the merge limit %llu",
                (unsigned long long)r, (unsigned long long)LB_MAX_COUNT);
  // final records and outputs, r at most
  for (int a = 0; a < 3; ++a) ST_TRY(ensure(ctx, sv->fk[a], r * 8));
  ST_TRY(ensure(ctx, sv->fcnt, r * 8));
  for (uint32_t c = 0; c < sv->nc; ++c) ST_TRY(ensure(ctx, sv->fsum[c], r * 8));
  for (int a = 0; a < 3; ++a) ST_TRY(ensure(ctx, sv->opos[a], r * 4));
  for (uint32_t c = 3; c < sv->nc; ++c) ST_TRY(ensure(ctx, sv->oattr[c], r * 8));
  ST_TRY(ensure(ctx, sv->okeys, r * 24));
  ST_TRY(reserve(ctx, r, 0, false, false, false));
  ST_TRY(reserve_batch(ctx, 1));
  ST_TRY(begin_chain(ctx, r, make_batch(ctx, 1), 1, nullptr, nullptr));
  {
    Launch l(ctx, SRCU_K_VOXEL_PLAN);
    k_stream_merge_plan<<<1, 32, 0, ctx->stream>>>(ctx->ctl, ptr<StreamPlan>(sv->plan),
                                                   ptr<StreamState>(sv->state));
  }
  StreamRecordSrc src{};
  src.kx = ptr<const long long>(sv->rk[0]);
  src.ky = ptr<const long long>(sv->rk[1]);
  src.kz = ptr<const long long>(sv->rk[2]);
  src.plan_ptr = ptr<const StreamPlan>(sv->plan);
  ST_TRY(launch_sort(ctx, src, r, ctx->ctl->hist_v, EP_VSORT, WK_VSORT, &ctx->ctl->vsort,
                     sv->occ_record, SRCU_K_VOXEL_SORT));
  StreamIn in{};
  in.nc = sv->nc;
  in.f64_mask = ~0u;
  in.cnt = ptr<const unsigned long long>(sv->rcnt);
  for (uint32_t c = 0; c < sv->nc; ++c) in.col[c] = sv->rsum[c].p;
  const StreamOut fin = sv_out(sv->fk, sv->fcnt, sv->fsum, sv->nc, 0, r);
  ST_TRY(sv_reduce<true>(sv, r, in, fin, 0));
  StreamFinal o{};
  for (int a = 0; a < 3; ++a) o.pos[a] = ptr<float>(sv->opos[a]);
  for (uint32_t c = 3; c < sv->nc; ++c) o.attr[c - 3] = ptr<double>(sv->oattr[c]);
  o.keys3 = ptr<long long>(sv->okeys);
  {
    Launch l(ctx, SRCU_K_UNPACK_KEYS);
    const uint32_t grid = std::max<uint32_t>(1, std::min<uint32_t>(ceil_div(r, 256),
                                                                    uint32_t(ctx->num_sms) * 8));
    k_stream_finalize<<<grid, 256, 0, ctx->stream>>>(ctx->ctl, fin, sv->nc, o);
  }
  CU_TRY(cudaGetLastError());
  ST_TRY(sv_sync(sv));
  sv->voxels = sv->state_host->segments;
  return SRCU_OK;
}

void sv_release(srcu_stream_voxel *sv) {
  srcu_ctx *ctx = sv->ctx;
  for (auto &b : sv->run) release(ctx, b);
  for (auto &b : sv->rk) release(ctx, b);
  for (auto &b : sv->rsum) release(ctx, b);
  for (auto &b : sv->fk) release(ctx, b);
  for (auto &b : sv->fsum) release(ctx, b);
  for (auto &b : sv->opos) release(ctx, b);
  for (auto &b : sv->oattr) release(ctx, b);
  DevBuf *rest[] = {&sv->rcnt, &sv->fcnt, &sv->okeys, &sv->tile_heads, &sv->tile_off,
                    &sv->long_list, &sv->plan, &sv->state};
  for (DevBuf *b : rest) release(ctx, *b);
}

}  // namespace

extern "C" {

srcu_status srcu_stream_voxel_create(srcu_ctx *ctx, const srcu_stream_voxel_params *params,
                                     srcu_stream_voxel **out) {
  if (!ctx || !out) return SRCU_ERR_INVALID_ARGUMENT;
  *out = nullptr;
  if (!params) return fail(ctx, SRCU_ERR_INVALID_ARGUMENT, "stream params are NULL");
  // StreamingVoxelConfig::new (streaming.rs:345-363)
  if (!(params->leaf_size > 0.0f) || params->leaf_size == INFINITY)
    return fail(ctx, SRCU_ERR_INVALID_ARGUMENT, "streaming voxel leaf size must be positive and finite");
  if (params->run_points == 0 || params->max_runs == 0)
    return fail(ctx, SRCU_ERR_INVALID_ARGUMENT,
                "streaming voxel run_points and max_runs must be positive");
  if (params->n_attrs > MAX_COLS - 3)
    return fail(ctx, SRCU_ERR_INVALID_ARGUMENT, "at most %d attribute columns are supported",
                MAX_COLS - 3);
  CU_TRY(cudaSetDevice(ctx->device));
  // Reuse the buffers of the context's last stream: a new stream then
  // allocates nothing until it outgrows them.
  srcu_stream_voxel *sv = ctx->parked_stream;
  ctx->parked_stream = nullptr;
  if (!sv) sv = new srcu_stream_voxel();
  sv->ctx = ctx;
  sv->prm = *params;
  sv->nc = 3 + params->n_attrs;
  sv->leaf = double(params->leaf_size);
  sv->fill = sv->points = sv->device_runs = sv->records = sv->voxels = 0;
  sv->rec_cap = 0;  // re-derived from the kept buffers' sizes as records arrive
  sv->finished = false;
  // By default a device run holds at least 2^22 points whatever run_points
  // is: the run size only partitions the sums, the voxels do not depend on it,
  // and larger runs sort more efficiently and synchronise less often.
  sv->dev_run = params->device_run_points
                    ? uint64_t(params->device_run_points)
                    : std::max<uint64_t>(params->run_points, uint64_t(1) << 22);
  sv->dev_run = std::min<uint64_t>(sv->dev_run, uint64_t(1) << 26);
  auto bail = [&](srcu_status st) {
    stream_voxel_free(sv);
    return st;
  };
  if (cudaFuncSetAttribute(k_sort<StreamPointSrc>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                           sizeof(OnesweepSmem)) != cudaSuccess ||
      cudaFuncSetAttribute(k_sort<StreamRecordSrc>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                           sizeof(OnesweepSmem)) != cudaSuccess)
    return bail(fail(ctx, SRCU_ERR_CUDA, "cannot configure the streaming sort kernels"));
  cudaOccupancyMaxActiveBlocksPerMultiprocessor(&sv->occ_point, k_sort<StreamPointSrc>, OS_THREADS,
                                                sizeof(OnesweepSmem));
  cudaOccupancyMaxActiveBlocksPerMultiprocessor(&sv->occ_record, k_sort<StreamRecordSrc>,
                                                OS_THREADS, sizeof(OnesweepSmem));
  sv->occ_point = std::max(1, sv->occ_point);
  sv->occ_record = std::max(1, sv->occ_record);
  srcu_status s = SRCU_OK;
  for (uint32_t c = 0; c < sv->nc && s == SRCU_OK; ++c)
    s = ensure(ctx, sv->run[c], sv->dev_run * sv_elem(sv, c));
  if (s == SRCU_OK) s = ensure(ctx, sv->plan, sizeof(StreamPlan));
  if (s == SRCU_OK) s = ensure(ctx, sv->state, sizeof(StreamState));
  if (s != SRCU_OK) return bail(s);
  if (!sv->state_host &&
      cudaMallocHost(reinterpret_cast<void **>(&sv->state_host), sizeof(StreamState)) != cudaSuccess)
    return bail(fail(ctx, SRCU_ERR_CUDA, "cannot allocate pinned stream state"));
  StreamState init{};
  for (int a = 0; a < 3; ++a) {
    init.gmin[a] = LLONG_MAX;
    init.gmax[a] = LLONG_MIN;
  }
  *sv->state_host = init;
  if (cudaMemcpyAsync(sv->state.p, sv->state_host, sizeof(StreamState), cudaMemcpyHostToDevice,
                      ctx->stream) != cudaSuccess ||
      cudaStreamSynchronize(ctx->stream) != cudaSuccess)
    return bail(fail(ctx, SRCU_ERR_CUDA, "cannot initialise the stream state"));
  *out = sv;
  return SRCU_OK;
}

srcu_status srcu_stream_voxel_push(srcu_stream_voxel *sv, const srcu_cloud *chunk) {
  if (!sv) return SRCU_ERR_INVALID_ARGUMENT;
  srcu_ctx *ctx = sv->ctx;
  ST_TRY(check_cloud(ctx, chunk));
  if (sv->finished) return fail(ctx, SRCU_ERR_INVALID_ARGUMENT, "the stream is already finished");
  if (chunk->n_attrs != sv->prm.n_attrs)
    return fail(ctx, SRCU_ERR_INVALID_ARGUMENT, "chunk has %u attribute columns, the stream %u",
                chunk->n_attrs, sv->prm.n_attrs);
  if (strided(chunk))
    return fail(ctx, SRCU_ERR_INVALID_ARGUMENT, "streaming voxel chunks must be packed columns");
  CU_TRY(cudaSetDevice(ctx->device));
  const void *src[MAX_COLS] = {chunk->x, chunk->y, chunk->z};
  for (uint32_t a = 0; a < chunk->n_attrs; ++a) src[3 + a] = chunk->attrs[a];
  const cudaMemcpyKind kind = chunk->on_device ? cudaMemcpyDeviceToDevice : cudaMemcpyHostToDevice;
  uint64_t done = 0;
  while (done < chunk->n) {
    const uint64_t take = std::min<uint64_t>(chunk->n - done, sv->dev_run - sv->fill);
    for (uint32_t c = 0; c < sv->nc; ++c) {
      const uint32_t e = sv_elem(sv, c);
      CU_TRY(cudaMemcpyAsync(static_cast<char *>(sv->run[c].p) + sv->fill * e,
                             static_cast<const char *>(src[c]) + done * e, take * e, kind,
                             ctx->stream));
    }
    sv->fill += take;
    done += take;
    if (sv->fill == sv->dev_run) ST_TRY(sv_flush(sv));
  }
  sv->points += chunk->n;
  CU_TRY(cudaStreamSynchronize(ctx->stream));  // the chunk's memory may be reused on return
  return SRCU_OK;
}

srcu_status srcu_stream_voxel_finish(srcu_stream_voxel *sv, srcu_stream_voxel_info *info) {
  if (!sv) return SRCU_ERR_INVALID_ARGUMENT;
  srcu_ctx *ctx = sv->ctx;
  if (info) memset(info, 0, sizeof(*info));
  if (sv->finished) return fail(ctx, SRCU_ERR_INVALID_ARGUMENT, "the stream is already finished");
  CU_TRY(cudaSetDevice(ctx->device));
  sv->finished = true;
  ST_TRY(sv_finish(sv));
  if (info) {
    const uint64_t finite = sv->state_host->finite;
    info->points = sv->points;
    info->finite_points = finite;
    info->runs = (finite + sv->prm.run_points - 1) / sv->prm.run_points;
    info->spool_bytes = info->runs * 8 + finite * (32 + 8 * uint64_t(sv->nc));
    info->device_runs = sv->device_runs;
    info->partial_records = sv->records;
    info->voxels = sv->voxels;
  }
  return SRCU_OK;
}

srcu_status srcu_stream_voxel_fetch(srcu_stream_voxel *sv, uint64_t first, uint64_t count,
                                    const srcu_stream_voxel_out *out) {
  if (!sv) return SRCU_ERR_INVALID_ARGUMENT;
  srcu_ctx *ctx = sv->ctx;
  if (!sv->finished) return fail(ctx, SRCU_ERR_INVALID_ARGUMENT, "the stream is not finished");
  if (!out) return fail(ctx, SRCU_ERR_INVALID_ARGUMENT, "output is NULL");
  if (first > sv->voxels || count > sv->voxels - first)
    return fail(ctx, SRCU_ERR_INVALID_ARGUMENT, "voxels [%llu, %llu) are out of range (%llu voxels)",
                (unsigned long long)first, (unsigned long long)(first + count),
                (unsigned long long)sv->voxels);
  if (count == 0) return SRCU_OK;
  CU_TRY(cudaSetDevice(ctx->device));
  float *pos[3] = {out->x, out->y, out->z};
  for (int a = 0; a < 3; ++a)
    ST_TRY(copy_out(ctx, pos[a], ptr<float>(sv->opos[a]) + first, count * 4, out->on_device));
  for (uint32_t c = 3; c < sv->nc; ++c)
    if (out->attrs && out->attrs[c - 3])
      ST_TRY(copy_out(ctx, out->attrs[c - 3], ptr<double>(sv->oattr[c]) + first, count * 8,
                      out->on_device));
  ST_TRY(copy_out(ctx, out->keys, ptr<long long>(sv->okeys) + 3 * first, count * 24, out->on_device));
  ST_TRY(copy_out(ctx, out->counts, ptr<unsigned long long>(sv->fcnt) + first, count * 8,
                  out->on_device));
  CU_TRY(cudaStreamSynchronize(ctx->stream));
  return SRCU_OK;
}

void srcu_stream_voxel_destroy(srcu_stream_voxel *sv) {
  if (!sv) return;
  srcu_ctx *ctx = sv->ctx;
  cudaSetDevice(ctx->device);
  cudaStreamSynchronize(ctx->stream);
  if (!ctx->parked_stream) {  // kept for the context's next stream
    ctx->parked_stream = sv;
    return;
  }
  stream_voxel_free(sv);
}

}  // extern "C"

void stream_voxel_free(srcu_stream_voxel *sv) {
  if (!sv) return;
  sv_release(sv);
  if (sv->state_host) cudaFreeHost(sv->state_host);
  delete sv;
}
