// las.cu -- host side of srcu_las_decode (include/srcuda.h).  Included at the
// end of srcuda.cu.
#include "las.cuh"

namespace {

// Standard record length, GPS-time and RGB offsets of LAS point data record
// formats 0-10 (ASPRS LAS 1.4 R15, tables 7-17).
struct LasLayout {
  uint32_t len;
  int32_t gps, rgb;
};
constexpr LasLayout kLasLayouts[11] = {
    {20, -1, -1}, {28, 20, -1}, {26, -1, 20}, {34, 20, 28}, {57, 20, -1}, {63, 20, 28},
    {30, 22, -1}, {36, 22, 30}, {38, 22, 30}, {59, 22, -1}, {67, 22, 30}};

}  // namespace

extern "C" {

srcu_status srcu_las_decode(srcu_ctx *ctx, const void *records, uint64_t n, int32_t records_on_device,
                            const srcu_las_format *fmt, const srcu_las_out *out) {
  if (!ctx) return SRCU_ERR_INVALID_ARGUMENT;
  if (!fmt || !out) return fail(ctx, SRCU_ERR_INVALID_ARGUMENT, "LAS format or output is NULL");
  if (fmt->point_format > 10)
    return fail(ctx, SRCU_ERR_UNSUPPORTED_DTYPE, "LAS point data record format %u is not 0-10",
                fmt->point_format);
  const LasLayout lay = kLasLayouts[fmt->point_format];
  if (fmt->record_length < lay.len || fmt->record_length > 4096)
    return fail(ctx, SRCU_ERR_INVALID_ARGUMENT,
                "record length %u is outside [%u, 4096] for point format %u", fmt->record_length,
                lay.len, fmt->point_format);
  if (n == 0) return SRCU_OK;
  if (!records || !out->x || !out->y || !out->z)
    return fail(ctx, SRCU_ERR_MISSING_FIELD, "LAS records or position outputs are NULL");
  if (n > (uint64_t(1) << 40) / fmt->record_length)
    return fail(ctx, SRCU_ERR_INVALID_ARGUMENT, "too many LAS records in one call");
  if ((out->gps_time && lay.gps < 0) || ((out->red || out->green || out->blue) && lay.rgb < 0))
    return fail(ctx, SRCU_ERR_MISSING_FIELD, "point format %u has no %s", fmt->point_format,
                out->gps_time && lay.gps < 0 ? "gps_time" : "color");
  CU_TRY(cudaSetDevice(ctx->device));
  const uint32_t rl = fmt->record_length;
  const uint8_t *src = static_cast<const uint8_t *>(records);
  if (!records_on_device) {
    ST_TRY(ensure(ctx, ctx->stage_block, n * rl));
    CU_TRY(cudaMemcpyAsync(ctx->stage_block.p, records, n * rl, cudaMemcpyHostToDevice, ctx->stream));
    src = ptr<const uint8_t>(ctx->stage_block);
  }
  LasDecodeDev d{};
  d.n = n;
  d.record_len = rl;
  d.per_tile = std::min<uint32_t>(LAS_TILE_RECORDS, LAS_BUF_MAX / rl);
  d.buf_bytes = (d.per_tile * rl + 32 + 15) & ~15u;
  const bool extended = fmt->point_format >= 6;
  d.class_off = extended ? 16 : 15;
  d.class_mask = extended ? 0xffu : 0x1fu;
  d.gps_off = lay.gps;
  d.rgb_off = lay.rgb;
  d.has_origin = fmt->has_origin;
  for (int a = 0; a < 3; ++a) {
    d.scale[a] = fmt->scale[a];
    d.offset[a] = fmt->offset[a];
    d.origin[a] = fmt->origin[a];
  }
  // Outputs: the caller's device buffers, or device staging copied back.
  void *dst[9] = {out->x, out->y, out->z, out->intensity, out->classification, out->gps_time,
                  out->red, out->green, out->blue};
  const uint32_t elem[9] = {4, 4, 4, 4, 1, 8, 2, 2, 2};
  void *dev[9] = {};
  for (int c = 0; c < 9; ++c) {
    if (!dst[c]) continue;
    if (out->on_device) {
      dev[c] = dst[c];
    } else {
      ST_TRY(ensure(ctx, ctx->in[c], n * elem[c]));
      dev[c] = ctx->in[c].p;
    }
  }
  LasOutDev o{};
  for (int a = 0; a < 3; ++a) o.pos[a] = static_cast<float *>(dev[a]);
  o.intensity = static_cast<float *>(dev[3]);
  o.cls = static_cast<uint8_t *>(dev[4]);
  o.gps = static_cast<double *>(dev[5]);
  for (int c = 0; c < 3; ++c) o.rgb[c] = static_cast<uint16_t *>(dev[6 + c]);
  const uint64_t tiles = (n + d.per_tile - 1) / d.per_tile;
  const size_t smem = 2 * size_t(d.buf_bytes);  // two tile buffers
  CU_TRY(cudaFuncSetAttribute(k_las_decode, cudaFuncAttributeMaxDynamicSharedMemorySize,
                              int(2 * (LAS_BUF_MAX + 48))));
  int per_sm = 1;
  cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_las_decode, LAS_THREADS, smem);
  const uint32_t grid = uint32_t(std::min<uint64_t>(
      tiles, uint64_t(ctx->num_sms) * uint64_t(std::max(per_sm, 1))));
  uint32_t *status = &ctx->ctl->status;
  CU_TRY(cudaMemsetAsync(status, 0, sizeof(uint32_t), ctx->stream));
  {
    Launch l(ctx, SRCU_K_LAS_DECODE);
    k_las_decode<<<grid, LAS_THREADS, smem, ctx->stream>>>(src, d, o, status);
  }
  CU_TRY(cudaGetLastError());
  CU_TRY(cudaMemcpyAsync(&ctx->ctl_host->status, status, sizeof(uint32_t), cudaMemcpyDeviceToHost,
                         ctx->stream));
  CU_TRY(cudaStreamSynchronize(ctx->stream));
  if (ctx->ctl_host->status & ST_TIMEOUT)
    return fail(ctx, SRCU_ERR_TIMEOUT, "a bounded wait for a LAS record copy gave up");
  if (!out->on_device)
    for (int c = 0; c < 9; ++c)
      if (dst[c]) ST_TRY(copy_out(ctx, dst[c], dev[c], n * elem[c], 0));
  CU_TRY(cudaStreamSynchronize(ctx->stream));
  return SRCU_OK;
}

}  // extern "C"
