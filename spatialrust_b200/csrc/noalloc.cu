// noalloc.cu -- allocation-free voxel centroid downsample (srcu_voxel_centroid_noalloc).
//
// Some callers cannot call cudaMalloc: a real-time loop (for example a ROS 2
// executor thread handling each LiDAR frame) that must not allocate after
// start-up, or a host application whose device memory belongs to another
// allocator that forbids raw allocations.  This entry point runs the same
// voxel chain as srcu_voxel_centroid, but its scratch -- control block, sort
// ping-pong buffers, look-back words, packed keys -- lives in one file-scope
// __device__ array of fixed size, so no call allocates device memory.  The
// caller passes device-resident input and output columns.
//
// Included at the end of srcuda.cu, so it shares that translation unit's
// kernels; the scratch array and the code that takes its address are here.

#include <mutex>

namespace {

constexpr uint64_t NA_MAX_POINTS = SRCU_NOALLOC_MAX_POINTS;
constexpr size_t na_align(size_t b) { return (b + 255) & ~size_t(255); }
constexpr size_t NA_CTL = 0;
constexpr size_t NA_KEYS0 = NA_CTL + na_align(sizeof(Control));
constexpr size_t NA_KEYS1 = NA_KEYS0 + na_align(NA_MAX_POINTS * 8);
constexpr size_t NA_VALS0 = NA_KEYS1 + na_align(NA_MAX_POINTS * 8);
constexpr size_t NA_VALS1 = NA_VALS0 + na_align(NA_MAX_POINTS * 4);
constexpr size_t NA_LB_SORT = NA_VALS1 + na_align(NA_MAX_POINTS * 4);
constexpr size_t NA_LB_SEG =
    NA_LB_SORT + na_align(((NA_MAX_POINTS + OS_TILE - 1) / OS_TILE) * RADIX_BINS * 8);
constexpr size_t NA_VKEYS = NA_LB_SEG + na_align(((NA_MAX_POINTS + SEG_TILE - 1) / SEG_TILE) * 8);
constexpr size_t NA_VCOUNTS = NA_VKEYS + na_align(NA_MAX_POINTS * 8);
constexpr size_t NA_BATCH = NA_VCOUNTS + na_align(NA_MAX_POINTS * 4);
// one-cloud batch arrays: offsets[2], bounds, plan, parameters, voxel offsets[2]
constexpr size_t NA_B_OFFSETS = NA_BATCH;
constexpr size_t NA_B_BOUNDS = NA_B_OFFSETS + 256;
constexpr size_t NA_B_VPLAN = NA_B_BOUNDS + na_align(sizeof(Bounds));
constexpr size_t NA_B_VPARAMS = NA_B_VPLAN + na_align(sizeof(VoxelPlan));
constexpr size_t NA_B_VOFF = NA_B_VPARAMS + na_align(sizeof(VoxelParamsDev));
constexpr size_t NA_BYTES = NA_B_VOFF + 256;
constexpr int NA_MAX_DEVICES = 64;

}  // namespace

// The scratch.  Zero at module load on each device (look-back words then
// carry epoch 0, which no chain uses); every call reuses it and leaves its
// contents behind.  In host code this name is only a stand-in for the device
// symbol: its device address comes from cudaGetSymbolAddress below.
static __device__ __align__(256) unsigned char g_noalloc_scratch[NA_BYTES];

namespace {

struct NoallocDevice {
  bool ready = false;
  unsigned char *base = nullptr;  // device address of g_noalloc_scratch on this device
  int num_sms = 0;
  int occ_sort = 1;
  int occ_seg = 1;
  // Host mirror of the scratch control block's epoch: each call's k_begin
  // advances it by EPOCHS_PER_RUN.  Before it would wrap, the look-back words
  // are cleared and it restarts at 0, as epoch_guard does for a context.
  uint32_t epoch_host = 0;
  uint64_t epoch_restarts = 0;
};

NoallocDevice g_noalloc_dev[NA_MAX_DEVICES];
std::mutex g_noalloc_mu;

// One-time set-up per device, with that device current: the scratch's device
// address and the launch attributes.  Runs inside the first call on a device.
srcu_status noalloc_setup(int device, NoallocDevice **out) {
  std::lock_guard<std::mutex> lock(g_noalloc_mu);
  NoallocDevice &d = g_noalloc_dev[device];
  if (!d.ready) {
    void *p = nullptr;
    if (cudaGetSymbolAddress(&p, g_noalloc_scratch) != cudaSuccess) {
      cudaGetLastError();
      return SRCU_ERR_CUDA;
    }
    if (cudaDeviceGetAttribute(&d.num_sms, cudaDevAttrMultiProcessorCount, device) != cudaSuccess ||
        cudaFuncSetAttribute(k_sort<VoxelKeySrc>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             sizeof(OnesweepSmem)) != cudaSuccess ||
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&d.occ_sort, k_sort<VoxelKeySrc>,
                                                      OS_THREADS, sizeof(OnesweepSmem)) != cudaSuccess ||
        configure_segment_kernels() != cudaSuccess ||
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&d.occ_seg, k_voxel_segments<4>, SEG_THREADS,
                                                      segment_smem_bytes(4)) != cudaSuccess) {
      cudaGetLastError();
      return SRCU_ERR_CUDA;
    }
    d.occ_sort = std::max(1, d.occ_sort);
    d.occ_seg = std::max(1, d.occ_seg);
    d.base = static_cast<unsigned char *>(p);
    d.ready = true;
  }
  *out = &d;
  return SRCU_OK;
}

template <int NC>
void noalloc_segments(cudaStream_t s, uint32_t grid, Control *ctl, const SortBuffers &sb,
                      const float **in, float *const *out, uint64_t *vkeys, uint32_t *vcounts,
                      const Batch &bt) {
  Columns<NC> cols;
  for (int c = 0; c < NC; ++c) {
    cols.in[c] = in[c];
    cols.out[c] = out[c];
  }
  k_voxel_segments<NC><<<grid, SEG_THREADS, segment_smem_bytes(NC), s>>>(
      ctl, sb, &ctl->vsort, cols, vkeys, vcounts, sb.lookback + 0, nullptr, nullptr, bt, -1);
}

}  // namespace

extern "C" srcu_status srcu_voxel_centroid_noalloc(const srcu_cloud *cloud,
                                                   const srcu_voxel_params *params,
                                                   const srcu_voxel_out *out, uint64_t *out_voxels,
                                                   void *cuda_stream) {
  if (out_voxels) *out_voxels = 0;
  if (!cloud || !params || !out) return SRCU_ERR_INVALID_ARGUMENT;
  if (cloud->n > NA_MAX_POINTS) return SRCU_ERR_INVALID_ARGUMENT;  // beyond the scratch size
  if (cloud->n_attrs > MAX_COLS - 3) return SRCU_ERR_INVALID_ARGUMENT;
  if (!cloud->on_device || !out->on_device) return SRCU_ERR_INVALID_ARGUMENT;
  if (cloud->stride > 1) return SRCU_ERR_INVALID_ARGUMENT;  // packed columns only
  if (params->leaf_size <= 0.0f) return SRCU_ERR_INVALID_ARGUMENT;  // voxel.rs:260-264
  if ((params->mode != SRCU_VOXEL_CENTROID && params->mode != SRCU_VOXEL_APPROXIMATE_FIRST) ||
      (params->attribute_policy != SRCU_ATTRIBUTE_AVERAGE &&
       params->attribute_policy != SRCU_ATTRIBUTE_FIRST))
    return SRCU_ERR_INVALID_ARGUMENT;
  const uint64_t n = cloud->n;
  if (n == 0) return SRCU_OK;
  if (!cloud->x || !cloud->y || !cloud->z || !out->x || !out->y || !out->z)
    return SRCU_ERR_MISSING_FIELD;
  for (uint32_t a = 0; a < cloud->n_attrs; ++a)
    if (!cloud->attrs || !cloud->attrs[a] || !out->attrs || !out->attrs[a])
      return SRCU_ERR_MISSING_FIELD;
  // An error left pending by the caller's own CUDA work is theirs: report it
  // before queueing anything, and leave it in place for them to read.
  if (cudaPeekAtLastError() != cudaSuccess) return SRCU_ERR_CUDA;
  int device = 0;
  if (cudaGetDevice(&device) != cudaSuccess || device < 0 || device >= NA_MAX_DEVICES) {
    cudaGetLastError();
    return SRCU_ERR_NO_DEVICE;
  }
  NoallocDevice *dev = nullptr;
  {
    const srcu_status st = noalloc_setup(device, &dev);
    if (st != SRCU_OK) return st;
  }
  cudaStream_t s = static_cast<cudaStream_t>(cuda_stream);
  unsigned char *b = dev->base;
  {
    std::lock_guard<std::mutex> lock(g_noalloc_mu);
    if (dev->epoch_host > kEpochLast) {
      if (cudaMemsetAsync(b + NA_LB_SORT, 0, NA_VKEYS - NA_LB_SORT, s) != cudaSuccess ||
          cudaMemsetAsync(b + NA_CTL + offsetof(Control, epoch), 0, sizeof(uint32_t), s) !=
              cudaSuccess) {
        cudaGetLastError();
        return SRCU_ERR_CUDA;
      }
      dev->epoch_host = 0;
      ++dev->epoch_restarts;
    }
    dev->epoch_host += EPOCHS_PER_RUN;
  }
  Control *ctl = reinterpret_cast<Control *>(b + NA_CTL);
  SortBuffers sb;
  sb.keys[0] = reinterpret_cast<uint64_t *>(b + NA_KEYS0);
  sb.keys[1] = reinterpret_cast<uint64_t *>(b + NA_KEYS1);
  sb.vals[0] = reinterpret_cast<uint32_t *>(b + NA_VALS0);
  sb.vals[1] = reinterpret_cast<uint32_t *>(b + NA_VALS1);
  sb.lookback = reinterpret_cast<uint64_t *>(b + NA_LB_SORT);
  SortBuffers seg = sb;
  seg.lookback = reinterpret_cast<uint64_t *>(b + NA_LB_SEG);
  uint64_t *vkeys = reinterpret_cast<uint64_t *>(b + NA_VKEYS);
  uint32_t *vcounts = out->counts ? out->counts : reinterpret_cast<uint32_t *>(b + NA_VCOUNTS);

  const uint32_t nc = 3 + cloud->n_attrs;
  const float *in[MAX_COLS] = {cloud->x, cloud->y, cloud->z};
  float *outc[MAX_COLS] = {out->x, out->y, out->z};
  for (uint32_t a = 0; a < cloud->n_attrs; ++a) {
    in[3 + a] = cloud->attrs[a];
    outc[3 + a] = out->attrs[a];
  }
  const uint32_t sms = uint32_t(dev->num_sms);
  Batch bt;
  bt.clouds = 1;
  bt.offsets = reinterpret_cast<const uint32_t *>(b + NA_B_OFFSETS);
  bt.bounds = reinterpret_cast<Bounds *>(b + NA_B_BOUNDS);
  bt.vplans = reinterpret_cast<VoxelPlan *>(b + NA_B_VPLAN);
  bt.cplans = nullptr;
  bt.vparams = reinterpret_cast<const VoxelParamsDev *>(b + NA_B_VPARAMS);
  bt.nparams = nullptr;
  bt.voxel_offsets = reinterpret_cast<uint32_t *>(b + NA_B_VOFF);
  VoxelParamsDev vp0{};
  vp0.leaf = params->leaf_size;
  vp0.has_origin = params->has_origin;
  for (int a = 0; a < 3; ++a) vp0.origin[a] = params->origin[a];
  vp0.agg = params->mode == SRCU_VOXEL_APPROXIMATE_FIRST ? AGG_FIRST
            : params->attribute_policy == SRCU_ATTRIBUTE_FIRST ? AGG_CENTROID_FIRST
                                                               : AGG_FAST;
  // k_begin zeroes the control block (all but the epoch) and writes the
  // cloud's offsets and parameters on every call.
  k_begin<<<1, 256, 0, s>>>(ctl, n, bt, 0u, 1, vp0, NormalParamsDev{});
  k_bounds<<<std::max<uint32_t>(1, std::min<uint32_t>(ceil_div(n, BND_THREADS * 4), sms * 8)),
             BND_THREADS, 0, s>>>(in[0], in[1], in[2], ctl, nullptr, nullptr, nullptr, bt);
  k_voxel_plans<<<1, 32, 0, s>>>(ctl, bt);
  VoxelKeySrc src;
  src.x = in[0];
  src.y = in[1];
  src.z = in[2];
  src.bt = bt;
  if (launch_sort_kernel(s, dev->num_sms, dev->occ_sort, src, ctl, ctl->hist_v, sb, EP_VSORT,
                         WK_VSORT, &ctl->vsort, n) != cudaSuccess) {
    cudaGetLastError();
    return SRCU_ERR_CUDA;
  }
  const uint32_t grid_g =
      std::min<uint32_t>(std::max<uint32_t>(1, ceil_div(n, SEG_TILE)), sms * uint32_t(dev->occ_seg));
  switch (nc) {
    case 3: noalloc_segments<3>(s, grid_g, ctl, seg, in, outc, vkeys, vcounts, bt); break;
    case 4: noalloc_segments<4>(s, grid_g, ctl, seg, in, outc, vkeys, vcounts, bt); break;
    case 5: noalloc_segments<5>(s, grid_g, ctl, seg, in, outc, vkeys, vcounts, bt); break;
    case 6: noalloc_segments<6>(s, grid_g, ctl, seg, in, outc, vkeys, vcounts, bt); break;
    case 7: noalloc_segments<7>(s, grid_g, ctl, seg, in, outc, vkeys, vcounts, bt); break;
    case 8: noalloc_segments<8>(s, grid_g, ctl, seg, in, outc, vkeys, vcounts, bt); break;
    case 9: noalloc_segments<9>(s, grid_g, ctl, seg, in, outc, vkeys, vcounts, bt); break;
    case 10: noalloc_segments<10>(s, grid_g, ctl, seg, in, outc, vkeys, vcounts, bt); break;
    case 11: noalloc_segments<11>(s, grid_g, ctl, seg, in, outc, vkeys, vcounts, bt); break;
    case 12: noalloc_segments<12>(s, grid_g, ctl, seg, in, outc, vkeys, vcounts, bt); break;
    default: return SRCU_ERR_INVALID_ARGUMENT;
  }
  if (out->keys)
    k_unpack_voxel_keys<<<std::max<uint32_t>(1, std::min<uint32_t>(ceil_div(n, 256), sms * 8)), 256,
                          0, s>>>(ctl, vkeys, out->keys, bt);
  if (cudaGetLastError() != cudaSuccess) return SRCU_ERR_CUDA;
  // Read back the status word and V (two words of the control block).
  uint32_t status = 0;
  unsigned long long voxels = 0;
  if (cudaMemcpyAsync(&status, &ctl->status, sizeof(status), cudaMemcpyDeviceToHost, s) != cudaSuccess ||
      cudaMemcpyAsync(&voxels, &ctl->n_voxels, sizeof(voxels), cudaMemcpyDeviceToHost, s) != cudaSuccess ||
      cudaStreamSynchronize(s) != cudaSuccess) {
    cudaGetLastError();
    return SRCU_ERR_CUDA;
  }
  if (status & ST_TIMEOUT) return SRCU_ERR_TIMEOUT;
  if (status & ST_KEY_OVERFLOW) return SRCU_ERR_KEY_OVERFLOW;
  if (status) return SRCU_ERR_CUDA;
  if (out_voxels) *out_voxels = voxels;
  return SRCU_OK;
}

// Test hooks for the epoch restart of the scratch on the current device.
extern "C" srcu_status srcu_noalloc_debug_set_epoch(uint32_t epoch) {
  if (epoch % EPOCHS_PER_RUN != 0) return SRCU_ERR_INVALID_ARGUMENT;
  int device = 0;
  if (cudaGetDevice(&device) != cudaSuccess || device < 0 || device >= NA_MAX_DEVICES) {
    cudaGetLastError();
    return SRCU_ERR_NO_DEVICE;
  }
  NoallocDevice *dev = nullptr;
  const srcu_status st = noalloc_setup(device, &dev);
  if (st != SRCU_OK) return st;
  std::lock_guard<std::mutex> lock(g_noalloc_mu);
  if (cudaDeviceSynchronize() != cudaSuccess ||
      cudaMemcpy(dev->base + NA_CTL + offsetof(Control, epoch), &epoch, sizeof(epoch),
                 cudaMemcpyHostToDevice) != cudaSuccess) {
    cudaGetLastError();
    return SRCU_ERR_CUDA;
  }
  dev->epoch_host = epoch;
  return SRCU_OK;
}

extern "C" srcu_status srcu_noalloc_debug_get_epoch(uint32_t *epoch, uint64_t *restarts) {
  int device = 0;
  if (cudaGetDevice(&device) != cudaSuccess || device < 0 || device >= NA_MAX_DEVICES) {
    cudaGetLastError();
    return SRCU_ERR_NO_DEVICE;
  }
  NoallocDevice *dev = nullptr;
  const srcu_status st = noalloc_setup(device, &dev);
  if (st != SRCU_OK) return st;
  std::lock_guard<std::mutex> lock(g_noalloc_mu);
  uint32_t e = 0;
  if (cudaDeviceSynchronize() != cudaSuccess ||
      cudaMemcpy(&e, dev->base + NA_CTL + offsetof(Control, epoch), sizeof(e),
                 cudaMemcpyDeviceToHost) != cudaSuccess) {
    cudaGetLastError();
    return SRCU_ERR_CUDA;
  }
  if (e != dev->epoch_host) return SRCU_ERR_CUDA;
  if (epoch) *epoch = e;
  if (restarts) *restarts = dev->epoch_restarts;
  return SRCU_OK;
}
