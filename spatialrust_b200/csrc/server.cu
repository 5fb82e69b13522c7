// server.cu -- the continuous-batching request loop (srcu_server_*).
//
// Built only on the public C ABI (include/srcuda.h) and the CUDA runtime.
// One worker thread owns every slot; a slot is a context, a stream and device
// input columns.  Small requests that are waiting when a small-request slot is
// free are packed into one batched chain; large requests get bulk slots of
// their own, so a multi-million-point map chunk never delays a frame.  A slot
// moves through the phases chain running -> (result space) -> read-back
// running -> idle, each detected with cudaEventQuery, so batches on different
// slots overlap on the device while the worker packs the next one.
//
// Host memory: submit copies a request once, into a pinned arena, from which
// the slot uploads it with one 2-D copy; results are read back into one arena
// block per batch, and each request's result columns point into it.  The
// worker thread therefore moves no bytes itself.
#include <cuda_runtime.h>

#include <algorithm>
#include <chrono>
#include <cmath>
#include <condition_variable>
#include <cstring>
#include <deque>
#include <map>
#include <mutex>
#include <thread>
#include <unordered_map>
#include <unordered_set>
#include <vector>

#include "../../include/srcuda.h"

namespace {

using Clock = std::chrono::steady_clock;

constexpr int NCOL_IN = 4;   // x, y, z, intensity
constexpr int NCOL_OUT = 8;  // x, y, z, intensity, nx, ny, nz, curvature
constexpr uint64_t OUT_BYTES_PER_VOXEL = NCOL_OUT * 4 + 4;  // + counts
// Device bytes a context holds per point of capacity for a 4-column chain
// (sort ping-pong 24, AoS copies 48, centroid columns + keys + counts 28,
// cell records 32, column ranges 72, hash table <= 32, normal outputs 20),
// plus a fixed allowance for look-back words and per-cloud plans.
constexpr uint64_t CTX_BYTES_PER_POINT = 256;
constexpr uint64_t CTX_FIXED_BYTES = 8ull << 20;
constexpr uint64_t SLOT_INPUT_BYTES_PER_POINT = NCOL_IN * sizeof(float);
constexpr uint32_t MAX_BATCH_CLOUDS = 1024;  // requests packed into one batched chain
constexpr size_t ARENA_ALIGN = 256;
constexpr size_t NO_SPACE = ~size_t(0);

size_t arena_round(size_t n) {
  return std::max<size_t>(ARENA_ALIGN, (n + ARENA_ALIGN - 1) & ~(ARENA_ALIGN - 1));
}

// First-fit allocator over one pinned region, with coalescing frees.
class PinnedArena {
 public:
  char *base = nullptr;
  size_t bytes = 0;

  bool init(size_t n) {
    bytes = arena_round(n);
    if (cudaMallocHost(reinterpret_cast<void **>(&base), bytes) != cudaSuccess) {
      cudaGetLastError();
      base = nullptr;
      return false;
    }
    free_[0] = bytes;
    return true;
  }
  void release() {
    if (base) cudaFreeHost(base);
    base = nullptr;
  }
  size_t alloc(size_t n) {
    n = arena_round(n);
    std::lock_guard<std::mutex> lock(mu_);
    for (auto it = free_.begin(); it != free_.end(); ++it) {
      if (it->second < n) continue;
      const size_t off = it->first, left = it->second - n;
      free_.erase(it);
      if (left) free_[off + n] = left;
      return off;
    }
    return NO_SPACE;
  }
  void free(size_t off, size_t n) {
    n = arena_round(n);
    std::lock_guard<std::mutex> lock(mu_);
    auto next = free_.lower_bound(off);
    if (next != free_.end() && off + n == next->first) {
      n += next->second;
      next = free_.erase(next);
    }
    if (next != free_.begin()) {
      auto prev = std::prev(next);
      if (prev->first + prev->second == off) {
        prev->second += n;
        return;
      }
    }
    free_[off] = n;
  }

 private:
  std::mutex mu_;
  std::map<size_t, size_t> free_;  // offset -> size
};

// One read-back block shared by the requests of a batch.
struct OutBlock {
  size_t off = 0, bytes = 0;
  int refs = 0;
};

struct Request {
  uint64_t id = 0;
  uint64_t n = 0;
  bool has_attr = false;
  bool bulk = false;
  size_t in_off = NO_SPACE;  // arena: x | y | z | intensity, n floats each
  srcu_voxel_params vp{};
  srcu_normal_params np{};
  Clock::time_point t_submit, t_done;
  srcu_status status = SRCU_OK;
  uint64_t voxels = 0;
  OutBlock *block = nullptr;
  uint64_t block_capacity = 0;  // voxels of the whole batch (column stride in the block)
  uint64_t block_first = 0;     // this request's first voxel in the block
};

struct Slot {
  srcu_ctx *ctx = nullptr;
  cudaStream_t stream = nullptr;
  bool bulk = false;
  uint64_t cap = 0;
  float *d_in = nullptr;  // NCOL_IN columns of cap floats
  cudaEvent_t ev_chain = nullptr, ev_out = nullptr;
  int phase = 0;  // 0 idle, 1 chain in flight, 2 waiting for result space, 3 read-back in flight
  std::vector<Request *> reqs;
  std::vector<uint64_t> voff;
  uint64_t voxels = 0;
  OutBlock *block = nullptr;
};

double percentile(std::vector<double> v, double q) {
  if (v.empty()) return 0.0;
  const size_t k = std::min(v.size() - 1, size_t(q * double(v.size() - 1) + 0.5));
  std::nth_element(v.begin(), v.begin() + k, v.end());
  return v[k];
}

}  // namespace

struct srcu_server {
  srcu_server_config cfg{};
  std::vector<Slot> slots;
  PinnedArena arena;
  std::thread worker;
  std::mutex mu;
  std::condition_variable cv_work, cv_done;
  bool stop = false;
  std::deque<Request *> pending_frames, pending_bulk;
  uint64_t pending_points = 0;
  std::deque<Request *> completed;
  std::unordered_map<uint64_t, Request *> delivered;
  std::unordered_set<uint64_t> live;  // ids submitted and not yet released
  // statistics (under mu)
  uint64_t submitted = 0, rejected = 0, n_completed = 0, failed = 0, batches = 0, points = 0;
  std::vector<double> lat_frame, lat_bulk;
  bool started = false;
  Clock::time_point t_first;

  void run();
  bool advance(Slot &s);
  void launch(Slot &s, std::vector<Request *> &&batch);
  void fail_slot(Slot &s, srcu_status st);
  void complete(Request *r);
  void drop(Request *r);
};

// Frees what a request holds in the arena.  Caller holds mu (block refcount).
void srcu_server::drop(Request *r) {
  if (r->in_off != NO_SPACE) arena.free(r->in_off, r->n * NCOL_IN * sizeof(float));
  r->in_off = NO_SPACE;
  if (r->block && --r->block->refs == 0) {
    arena.free(r->block->off, r->block->bytes);
    delete r->block;
  }
  r->block = nullptr;
  delete r;
}

void srcu_server::complete(Request *r) {
  r->t_done = Clock::now();
  if (r->in_off != NO_SPACE) arena.free(r->in_off, r->n * NCOL_IN * sizeof(float));
  r->in_off = NO_SPACE;
  const double ms = std::chrono::duration<double, std::milli>(r->t_done - r->t_submit).count();
  std::lock_guard<std::mutex> lock(mu);
  if (r->status == SRCU_OK) {
    (r->bulk ? lat_bulk : lat_frame).push_back(ms);
    ++n_completed;
  } else {
    ++failed;
  }
  completed.push_back(r);
  cv_done.notify_all();
}

void srcu_server::fail_slot(Slot &s, srcu_status st) {
  if (s.block) {
    arena.free(s.block->off, s.block->bytes);
    delete s.block;
    s.block = nullptr;
  }
  for (Request *r : s.reqs) {
    r->status = st;
    complete(r);
  }
  s.reqs.clear();
  s.phase = 0;
}

// Uploads a batch into the slot's device columns (one 2-D copy per request:
// its four arena columns into the four slot columns) and enqueues the batched
// chain; ev_chain fires when the chain is done.
void srcu_server::launch(Slot &s, std::vector<Request *> &&batch) {
  s.reqs = std::move(batch);
  const uint32_t count = uint32_t(s.reqs.size());
  std::vector<uint64_t> offsets(count + 1, 0);
  std::vector<srcu_voxel_params> vps(count);
  std::vector<srcu_normal_params> nps(count);
  bool ok = true;
  for (uint32_t b = 0; b < count && ok; ++b) {
    const Request *r = s.reqs[b];
    offsets[b + 1] = offsets[b] + r->n;
    vps[b] = r->vp;
    nps[b] = r->np;
    ok = cudaMemcpy2DAsync(s.d_in + offsets[b], s.cap * sizeof(float), arena.base + r->in_off,
                           r->n * sizeof(float), r->n * sizeof(float), NCOL_IN,
                           cudaMemcpyHostToDevice, s.stream) == cudaSuccess;
  }
  const uint64_t n = offsets[count];
  const float *attrs[1] = {s.d_in + 3 * s.cap};
  srcu_cloud cloud{s.d_in, s.d_in + s.cap, s.d_in + 2 * s.cap, attrs, 1, 1, n};
  srcu_status st = ok ? srcu_batch_voxel_normals_enqueue(s.ctx, &cloud, offsets.data(), count,
                                                         vps.data(), nps.data())
                      : SRCU_ERR_CUDA;
  if (st == SRCU_OK && cudaEventRecord(s.ev_chain, s.stream) != cudaSuccess) st = SRCU_ERR_CUDA;
  if (st != SRCU_OK) {
    cudaGetLastError();
    fail_slot(s, st);
    return;
  }
  {
    std::lock_guard<std::mutex> lock(mu);
    ++batches;
    points += n;
  }
  s.phase = 1;
}

// Advances a busy slot; true if it moved.
bool srcu_server::advance(Slot &s) {
  if (s.phase == 1) {
    if (cudaEventQuery(s.ev_chain) != cudaSuccess) return false;
    const uint32_t count = uint32_t(s.reqs.size());
    s.voff.assign(count + 1, 0);
    // Synchronises with the (finished) chain and checks its device status word.
    const srcu_status st = srcu_batch_voxel_offsets(s.ctx, s.voff.data());
    if (st != SRCU_OK) {
      fail_slot(s, st);
      return true;
    }
    s.voxels = s.voff[count];
    s.phase = 2;
  }
  if (s.phase == 2) {
    const size_t bytes = s.voxels * OUT_BYTES_PER_VOXEL;
    const size_t off = s.voxels ? arena.alloc(bytes) : 0;
    if (off == NO_SPACE) return false;  // results not yet released hold the arena
    srcu_frame_view view{};
    srcu_status st = srcu_frame_view_get(s.ctx, &view);
    if (st == SRCU_OK && s.voxels) {
      s.block = new OutBlock{off, bytes, int(s.reqs.size())};
      char *dst = arena.base + off;
      const void *src[NCOL_OUT + 1] = {view.x,  view.y,  view.z,  view.attrs[0], view.nx,
                                       view.ny, view.nz, view.curvature, view.counts};
      bool ok = true;
      for (int c = 0; c <= NCOL_OUT && ok; ++c)
        ok = cudaMemcpyAsync(dst + size_t(c) * s.voxels * 4, src[c], s.voxels * 4,
                             cudaMemcpyDeviceToHost, s.stream) == cudaSuccess;
      if (!ok) st = SRCU_ERR_CUDA;
    }
    if (st == SRCU_OK && cudaEventRecord(s.ev_out, s.stream) != cudaSuccess) st = SRCU_ERR_CUDA;
    if (st != SRCU_OK) {
      cudaGetLastError();
      fail_slot(s, st);
      return true;
    }
    s.phase = 3;
    return true;
  }
  if (s.phase == 3) {
    if (cudaEventQuery(s.ev_out) != cudaSuccess) return false;
    for (size_t b = 0; b < s.reqs.size(); ++b) {
      Request *r = s.reqs[b];
      r->voxels = s.voff[b + 1] - s.voff[b];
      r->block = s.block;
      r->block_capacity = s.voxels;
      r->block_first = s.voff[b];
      complete(r);
    }
    s.block = nullptr;
    s.reqs.clear();
    s.phase = 0;
    return true;
  }
  return false;
}

void srcu_server::run() {
  cudaSetDevice(cfg.device);
  for (;;) {
    bool progress = false;
    for (Slot &s : slots)
      if (s.phase != 0) progress |= advance(s);
    // Continuous batching: every idle slot takes what its queue holds now.
    for (Slot &s : slots) {
      if (s.phase != 0) continue;
      std::vector<Request *> batch;
      {
        std::lock_guard<std::mutex> lock(mu);
        if (s.bulk) {
          if (!pending_bulk.empty()) {
            batch.push_back(pending_bulk.front());
            pending_bulk.pop_front();
          }
        } else {
          uint64_t pts = 0;
          while (!pending_frames.empty() && batch.size() < MAX_BATCH_CLOUDS &&
                 (batch.empty() || pts + pending_frames.front()->n <= s.cap)) {
            pts += pending_frames.front()->n;
            batch.push_back(pending_frames.front());
            pending_frames.pop_front();
          }
        }
        for (Request *r : batch) pending_points -= r->n;
      }
      if (!batch.empty()) {
        launch(s, std::move(batch));
        progress = true;
      }
    }
    if (progress) continue;
    std::unique_lock<std::mutex> lock(mu);
    bool busy = false;
    for (Slot &s : slots) busy |= s.phase != 0;
    if (stop && !busy && pending_frames.empty() && pending_bulk.empty()) break;
    // Busy: a short nap before polling the events again; idle: until a submit.
    cv_work.wait_for(lock, busy ? std::chrono::microseconds(20) : std::chrono::microseconds(500));
  }
}

extern "C" {

srcu_status srcu_server_create(const srcu_server_config *config, srcu_server **out) {
  if (!out) return SRCU_ERR_INVALID_ARGUMENT;
  *out = nullptr;
  srcu_server_config c{};
  if (config) c = *config;
  if (!c.hbm_budget_bytes) c.hbm_budget_bytes = 40ull << 30;
  if (!c.frame_slots) c.frame_slots = 3;
  if (!c.bulk_slots) c.bulk_slots = 1;
  if (!c.frame_batch_points) c.frame_batch_points = 1u << 20;
  if (!c.bulk_threshold_points) c.bulk_threshold_points = 500000;
  if (!c.bulk_max_points) c.bulk_max_points = 4500000;
  if (!c.max_pending_points) c.max_pending_points = 64ull << 20;
  if (!c.host_arena_bytes) c.host_arena_bytes = 2ull << 30;
  if (c.bulk_threshold_points > c.frame_batch_points || c.bulk_max_points < c.bulk_threshold_points ||
      c.frame_batch_points > 0xFFFFFFFFull || c.bulk_max_points > 0xFFFFFFFFull)
    return SRCU_ERR_INVALID_ARGUMENT;
  const uint64_t slot_points = uint64_t(c.frame_slots) * c.frame_batch_points +
                               uint64_t(c.bulk_slots) * c.bulk_max_points;
  const uint64_t need = slot_points * (CTX_BYTES_PER_POINT + SLOT_INPUT_BYTES_PER_POINT) +
                        uint64_t(c.frame_slots + c.bulk_slots) * CTX_FIXED_BYTES;
  if (need > c.hbm_budget_bytes) return SRCU_ERR_OUT_OF_BUDGET;  // slots do not fit the budget
  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || c.device < 0 || c.device >= ndev ||
      cudaSetDevice(c.device) != cudaSuccess) {
    cudaGetLastError();
    return SRCU_ERR_NO_DEVICE;
  }
  srcu_server *sv = new srcu_server();
  sv->cfg = c;
  if (!sv->arena.init(c.host_arena_bytes)) {
    delete sv;
    return SRCU_ERR_OUT_OF_BUDGET;
  }
  const uint32_t nslots = c.frame_slots + c.bulk_slots;
  sv->slots.resize(nslots);
  srcu_status st = SRCU_OK;
  for (uint32_t i = 0; i < nslots && st == SRCU_OK; ++i) {
    Slot &s = sv->slots[i];
    s.bulk = i >= c.frame_slots;
    s.cap = s.bulk ? c.bulk_max_points : c.frame_batch_points;
    st = srcu_create(c.device, s.cap * CTX_BYTES_PER_POINT + CTX_FIXED_BYTES, &s.ctx);
    if (st != SRCU_OK) break;
    const bool ok =
        cudaStreamCreateWithFlags(&s.stream, cudaStreamNonBlocking) == cudaSuccess &&
        cudaEventCreateWithFlags(&s.ev_chain, cudaEventDisableTiming) == cudaSuccess &&
        cudaEventCreateWithFlags(&s.ev_out, cudaEventDisableTiming) == cudaSuccess &&
        cudaMalloc(&s.d_in, s.cap * NCOL_IN * sizeof(float)) == cudaSuccess &&
        cudaMemsetAsync(s.d_in, 0, s.cap * NCOL_IN * sizeof(float), s.stream) == cudaSuccess;
    if (!ok) {
      cudaGetLastError();
      st = SRCU_ERR_OUT_OF_BUDGET;
      break;
    }
    st = srcu_set_stream(s.ctx, s.stream);
    if (st != SRCU_OK) break;
    // Warm-up at full capacity (and, on batch slots, the largest batch) so no
    // request pays for a device allocation.
    const float *attrs[1] = {s.d_in + 3 * s.cap};
    srcu_cloud cloud{s.d_in, s.d_in + s.cap, s.d_in + 2 * s.cap, attrs, 1, 1, s.cap};
    const uint32_t count = s.bulk ? 1 : MAX_BATCH_CLOUDS;
    std::vector<uint64_t> offsets(count + 1);
    for (uint32_t b = 0; b <= count; ++b) offsets[b] = s.cap * b / count;
    std::vector<srcu_voxel_params> vps(count, srcu_voxel_params{1.0f, 0, {0, 0, 0}});
    std::vector<srcu_normal_params> nps(count, srcu_normal_params{1.0f, 3, 0, {0, 0, 0}, 0, 0});
    st = srcu_batch_voxel_normals_enqueue(s.ctx, &cloud, offsets.data(), count, vps.data(),
                                          nps.data());
    if (st == SRCU_OK) st = srcu_frame_check(s.ctx, nullptr, nullptr);
  }
  if (st != SRCU_OK) {
    srcu_server_destroy(sv);
    return st;
  }
  sv->worker = std::thread([sv] { sv->run(); });
  *out = sv;
  return SRCU_OK;
}

void srcu_server_destroy(srcu_server *sv) {
  if (!sv) return;
  if (sv->worker.joinable()) {
    {
      std::lock_guard<std::mutex> lock(sv->mu);
      sv->stop = true;
    }
    sv->cv_work.notify_all();
    sv->worker.join();
  }
  cudaSetDevice(sv->cfg.device);
  for (Slot &s : sv->slots) {
    if (s.stream) cudaStreamSynchronize(s.stream);
    if (s.d_in) cudaFree(s.d_in);
    if (s.ev_chain) cudaEventDestroy(s.ev_chain);
    if (s.ev_out) cudaEventDestroy(s.ev_out);
    if (s.ctx) srcu_destroy(s.ctx);
    if (s.stream) cudaStreamDestroy(s.stream);
  }
  {
    std::lock_guard<std::mutex> lock(sv->mu);
    for (Request *r : sv->pending_frames) sv->drop(r);
    for (Request *r : sv->pending_bulk) sv->drop(r);
    for (Request *r : sv->completed) sv->drop(r);
    for (auto &kv : sv->delivered) sv->drop(kv.second);
  }
  sv->arena.release();
  delete sv;
}

srcu_status srcu_server_submit(srcu_server *sv, uint64_t req_id, const srcu_cloud *cloud,
                               const srcu_voxel_params *vp, const srcu_normal_params *np) {
  const Clock::time_point t0 = Clock::now();
  if (!sv || !cloud || !vp || !np) return SRCU_ERR_INVALID_ARGUMENT;
  if (cloud->on_device || cloud->n_attrs > 1 || cloud->stride > 64) return SRCU_ERR_INVALID_ARGUMENT;
  if (cloud->n > sv->cfg.bulk_max_points) return SRCU_ERR_INVALID_ARGUMENT;
  if (cloud->n && (!cloud->x || !cloud->y || !cloud->z)) return SRCU_ERR_MISSING_FIELD;
  if (cloud->n_attrs == 1 && cloud->n && (!cloud->attrs || !cloud->attrs[0]))
    return SRCU_ERR_MISSING_FIELD;
  // The chain's own parameter checks (voxel.rs:260-264, normal.rs:109-111),
  // made here so that a bad request fails alone instead of failing its batch.
  if (vp->leaf_size <= 0.0f) return SRCU_ERR_INVALID_ARGUMENT;
  if (!(np->radius >= 0.0f) || std::isinf(np->radius)) return SRCU_ERR_INVALID_ARGUMENT;
  {
    std::lock_guard<std::mutex> lock(sv->mu);
    if (sv->live.count(req_id)) return SRCU_ERR_INVALID_ARGUMENT;  // id not yet released
    if (!sv->started) {
      sv->started = true;
      sv->t_first = t0;
    }
    if (sv->pending_points + cloud->n > sv->cfg.max_pending_points) {
      ++sv->rejected;
      return SRCU_ERR_BUSY;
    }
    sv->live.insert(req_id);
  }
  Request *r = new Request();
  r->t_submit = t0;
  r->id = req_id;
  r->n = cloud->n;
  r->has_attr = cloud->n_attrs == 1;
  r->bulk = cloud->n >= sv->cfg.bulk_threshold_points;
  r->vp = *vp;
  r->np = *np;
  if (r->n) {
    r->in_off = sv->arena.alloc(r->n * NCOL_IN * sizeof(float));
    if (r->in_off == NO_SPACE) {
      delete r;
      std::lock_guard<std::mutex> lock(sv->mu);
      sv->live.erase(req_id);
      ++sv->rejected;
      return SRCU_ERR_BUSY;
    }
    float *dst = reinterpret_cast<float *>(sv->arena.base + r->in_off);
    const float *src[NCOL_IN] = {cloud->x, cloud->y, cloud->z,
                                 r->has_attr ? cloud->attrs[0] : nullptr};
    const size_t stride = cloud->stride > 1 ? cloud->stride : 1;
    for (int c = 0; c < NCOL_IN; ++c) {
      float *d = dst + size_t(c) * r->n;
      if (!src[c]) std::memset(d, 0, r->n * sizeof(float));
      else if (stride == 1) std::memcpy(d, src[c], r->n * sizeof(float));
      else  // interleaved records: gather this field
        for (uint64_t i = 0; i < r->n; ++i) d[i] = src[c][i * stride];
    }
  }
  {
    std::lock_guard<std::mutex> lock(sv->mu);
    ++sv->submitted;
    if (r->n == 0) {  // voxel.rs:257-259, normal.rs:106-108: an empty result at once
      r->t_done = Clock::now();
      ++sv->n_completed;
      sv->completed.push_back(r);
      sv->cv_done.notify_all();
      return SRCU_OK;
    }
    sv->pending_points += r->n;
    (r->bulk ? sv->pending_bulk : sv->pending_frames).push_back(r);
  }
  sv->cv_work.notify_one();
  return SRCU_OK;
}

srcu_status srcu_server_poll(srcu_server *sv, srcu_request_result *out, uint32_t wait_us) {
  if (!sv || !out) return SRCU_ERR_INVALID_ARGUMENT;
  std::unique_lock<std::mutex> lock(sv->mu);
  if (sv->completed.empty() && wait_us)
    sv->cv_done.wait_for(lock, std::chrono::microseconds(wait_us),
                         [sv] { return !sv->completed.empty(); });
  if (sv->completed.empty()) return SRCU_ERR_BUSY;
  Request *r = sv->completed.front();
  sv->completed.pop_front();
  sv->delivered[r->id] = r;
  memset(out, 0, sizeof(*out));
  out->req_id = r->id;
  out->status = r->status;
  out->points = r->n;
  out->voxels = r->voxels;
  if (r->status == SRCU_OK && r->voxels && r->block) {
    const float *col = reinterpret_cast<const float *>(sv->arena.base + r->block->off);
    const uint64_t stride = r->block_capacity, first = r->block_first;
    const float *c[NCOL_OUT];
    for (int k = 0; k < NCOL_OUT; ++k) c[k] = col + size_t(k) * stride + first;
    out->x = c[0];
    out->y = c[1];
    out->z = c[2];
    out->intensity = r->has_attr ? c[3] : nullptr;
    out->nx = c[4];
    out->ny = c[5];
    out->nz = c[6];
    out->curvature = c[7];
    out->counts = reinterpret_cast<const uint32_t *>(col + size_t(NCOL_OUT) * stride) + first;
  }
  out->latency_ms = std::chrono::duration<double, std::milli>(r->t_done - r->t_submit).count();
  return SRCU_OK;
}

srcu_status srcu_server_release(srcu_server *sv, uint64_t req_id) {
  if (!sv) return SRCU_ERR_INVALID_ARGUMENT;
  std::lock_guard<std::mutex> lock(sv->mu);
  auto it = sv->delivered.find(req_id);
  if (it == sv->delivered.end()) return SRCU_ERR_INVALID_ARGUMENT;
  Request *r = it->second;
  sv->delivered.erase(it);
  sv->live.erase(req_id);
  sv->drop(r);
  return SRCU_OK;
}

srcu_status srcu_server_stats_get(srcu_server *sv, srcu_server_stats *st) {
  if (!sv || !st) return SRCU_ERR_INVALID_ARGUMENT;
  std::lock_guard<std::mutex> lock(sv->mu);
  memset(st, 0, sizeof(*st));
  st->submitted = sv->submitted;
  st->rejected = sv->rejected;
  st->completed = sv->n_completed;
  st->failed = sv->failed;
  st->batches = sv->batches;
  st->points = sv->points;
  st->frame_p50_ms = percentile(sv->lat_frame, 0.50);
  st->frame_p99_ms = percentile(sv->lat_frame, 0.99);
  st->bulk_p50_ms = percentile(sv->lat_bulk, 0.50);
  st->bulk_p99_ms = percentile(sv->lat_bulk, 0.99);
  std::vector<double> all = sv->lat_frame;
  all.insert(all.end(), sv->lat_bulk.begin(), sv->lat_bulk.end());
  st->all_p50_ms = percentile(all, 0.50);
  st->all_p99_ms = percentile(all, 0.99);
  if (sv->started)
    st->elapsed_s = std::chrono::duration<double>(Clock::now() - sv->t_first).count();
  return SRCU_OK;
}

srcu_status srcu_server_stats_reset(srcu_server *sv) {
  if (!sv) return SRCU_ERR_INVALID_ARGUMENT;
  std::lock_guard<std::mutex> lock(sv->mu);
  sv->lat_frame.clear();
  sv->lat_bulk.clear();
  sv->submitted = sv->rejected = sv->n_completed = sv->failed = sv->batches = sv->points = 0;
  sv->started = false;
  return SRCU_OK;
}

}  // extern "C"
