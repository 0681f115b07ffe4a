// Host side of the B200 snow step: batches of scenes, device buffers, CUDA
// graphs, the particle record <-> structure-of-arrays conversion and the C ABI
// declared in include/snow_gpu.h.
#include <cuda_runtime.h>

#include <algorithm>
#include <climits>
#include <cmath>
#include <cstring>
#include <memory>
#include <mutex>
#include <stdexcept>
#include <string>
#include <vector>

#include "snow_batch.cuh"
#include "snow_engine.hpp"
#include "snow_gpu.h"

namespace snow {

int radix_tiles(int64_t n);

thread_local std::string g_last_error;

int set_error(int code, const std::string& msg) {
  g_last_error = msg;
  return code;
}

void check_cuda(cudaError_t e, const char* what) {
  if (e != cudaSuccess) throw Error(SNOW_E_CUDA, std::string(what) + ": " + cudaGetErrorString(e));
}

static_assert(sizeof(snow_collider) == sizeof(Collider), "collider layouts must agree");

std::vector<Collider> device_colliders(const snow_collider* c, int n) {
  if (n < 0 || (n > 0 && !c)) throw Error(SNOW_E_ARG, "bad collider array");
  std::vector<Collider> out;
  for (int i = 0; i < n; ++i) {
    const snow_collider& x = c[i];
    if (x.kind != SNOW_COLLIDER_PLANE && x.kind != SNOW_COLLIDER_SPHERE && x.kind != SNOW_COLLIDER_BOX)
      throw Error(SNOW_E_ARG, "unsupported collider kind " + std::to_string(x.kind));
    if (x.kind == SNOW_COLLIDER_SPHERE && !(x.param[0] > 0.0 && std::isfinite(x.param[0])))
      throw Error(SNOW_E_ARG, "sphere collider needs a positive finite radius in param[0]");
    if (x.kind == SNOW_COLLIDER_BOX) {
      double uu = 0, ww = 0, uw = 0;
      for (int a = 0; a < 3; ++a) {
        uu += x.normal[a] * x.normal[a];
        ww += x.axis[a] * x.axis[a];
        uw += x.normal[a] * x.axis[a];
        if (!(x.extent[a] > 0.0 && std::isfinite(x.extent[a])))
          throw Error(SNOW_E_ARG, "box collider needs positive finite half extents");
      }
      if (!(std::fabs(uu - 1.0) < 1e-9 && std::fabs(ww - 1.0) < 1e-9 && std::fabs(uw) < 1e-9))
        throw Error(SNOW_E_ARG, "box collider axes (normal, axis) must be unit and orthogonal");
    }
    Collider d{};
    std::memcpy(&d, &x, sizeof d);
    d.pad = 0;
    out.push_back(d);
  }
  return out;
}

namespace {

template <typename T>
T* dalloc(size_t count) {
  void* p = nullptr;
  if (count == 0) count = 1;
  check_cuda(cudaMalloc(&p, count * sizeof(T)), "cudaMalloc");
  return static_cast<T*>(p);
}
template <typename T>
void dfree(T*& p) {
  if (p) cudaFree((void*)p);
  p = nullptr;
}

// ------------------------------------------------- record <-> SoA conversion
template <typename R>
__global__ void k_records_to_planes(const double* rec, int64_t n, R* r, double* fp, int32_t* id,
                                    int64_t st) {
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const double* p = rec + 26 * i;
#pragma unroll
  for (int k = 0; k < 8; ++k) r[k * st + i] = (R)p[k];          // x, v, m, V_p0
#pragma unroll
  for (int k = 0; k < 9; ++k) fp[k * st + i] = p[8 + k];        // F_P
#pragma unroll
  for (int k = 0; k < 9; ++k) r[(PFE + k) * st + i] = (R)p[17 + k];  // F_E
  id[i] = (int32_t)i;
}

// The same into the slots the scene's particles already occupy: slot j takes
// record id[j].  After a step the slots are block-sorted, so the next step
// reads its particles in sorted order instead of the caller's.  An id outside
// [0, n) is never read through; it sets a status bit instead.
template <typename R>
__global__ void k_records_to_planes_ordered(const double* rec, int64_t n, R* r, double* fp, const int32_t* id,
                                            int64_t st, uint32_t* status) {
  const int64_t j = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (j >= n) return;
  const int64_t src = id[j];
  if (src < 0 || src >= n) {
    atomicOr(status, ST_LOOKUP_MISS);
    return;
  }
  const double* p = rec + 26 * src;
#pragma unroll
  for (int k = 0; k < 8; ++k) r[k * st + j] = (R)p[k];
#pragma unroll
  for (int k = 0; k < 9; ++k) fp[k * st + j] = p[8 + k];
#pragma unroll
  for (int k = 0; k < 9; ++k) r[(PFE + k) * st + j] = (R)p[17 + k];
}

template <typename R>
__global__ void k_planes_to_records(double* rec, int64_t n, const R* r, const double* fp,
                                    const int32_t* id, int64_t st) {
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  double* p = rec + 26 * (int64_t)id[i];
#pragma unroll
  for (int k = 0; k < 8; ++k) p[k] = (double)r[k * st + i];
#pragma unroll
  for (int k = 0; k < 9; ++k) p[8 + k] = fp[k * st + i];
#pragma unroll
  for (int k = 0; k < 9; ++k) p[17 + k] = (double)r[(PFE + k) * st + i];
}

template <typename R>
__global__ void k_planes_to_positions(double* xyz, int64_t n, const R* r, const int32_t* id, int64_t st) {
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  double* p = xyz + 3 * (int64_t)id[i];
#pragma unroll
  for (int a = 0; a < 3; ++a) p[a] = (double)r[(PX + a) * st + i];
}

int64_t pad32(int64_t n) { return (n + 31) / 32 * 32; }

// True for host memory that is page-locked (registered or cudaHostAlloc'd).
bool page_locked(const void* p) {
  cudaPointerAttributes a{};
  if (cudaPointerGetAttributes(&a, p) != cudaSuccess) {
    cudaGetLastError();
    return false;
  }
  return a.type == cudaMemoryTypeHost;
}

}  // namespace

// Host <-> device copies of particle records.  Page-locked host memory is
// copied by direct DMA.  Pageable memory goes through two page-locked chunks
// of kXferChunk bytes: the host copy of one chunk overlaps the DMA of the
// other, and no pageable copy is left to the driver's own staging.
void Batch::ensure_pinned() {
  if (pinned_[0]) return;
  for (int k = 0; k < 2; ++k) {
    check_cuda(cudaHostAlloc((void**)&pinned_[k], kXferChunk, cudaHostAllocDefault), "cudaHostAlloc");
    check_cuda(cudaEventCreateWithFlags(&pinned_ev_[k], cudaEventDisableTiming), "cudaEventCreate");
  }
}

void Batch::copy_in(void* dst, const void* src, size_t bytes, cudaStream_t s, bool wait) {
  if (page_locked(src)) {
    // the caller may reuse its buffer once the call returns (wait), or once
    // the stream has passed the copy
    check_cuda(cudaMemcpyAsync(dst, src, bytes, cudaMemcpyHostToDevice, s), "upload copy");
    if (wait) check_cuda(cudaStreamSynchronize(s), "upload sync");
    return;
  }
  ensure_pinned();
  for (size_t off = 0, c = 0; off < bytes; off += kXferChunk, ++c) {
    const size_t len = std::min(kXferChunk, bytes - off);
    const int k = (int)(c & 1);
    check_cuda(cudaEventSynchronize(pinned_ev_[k]), "upload chunk");  // the chunk's last DMA is done
    std::memcpy(pinned_[k], static_cast<const unsigned char*>(src) + off, len);
    check_cuda(cudaMemcpyAsync(static_cast<unsigned char*>(dst) + off, pinned_[k], len, cudaMemcpyHostToDevice, s),
               "upload copy");
    check_cuda(cudaEventRecord(pinned_ev_[k], s), "upload chunk");
  }
}

void Batch::copy_out(void* dst, const void* src, size_t bytes, cudaStream_t s, bool wait) {
  if (page_locked(dst)) {
    check_cuda(cudaMemcpyAsync(dst, src, bytes, cudaMemcpyDeviceToHost, s), "download copy");
    if (wait) check_cuda(cudaStreamSynchronize(s), "download sync");
    return;
  }
  ensure_pinned();
  const size_t chunks = (bytes + kXferChunk - 1) / kXferChunk;
  auto issue = [&](size_t c) {
    const size_t off = c * kXferChunk, len = std::min(kXferChunk, bytes - off);
    const int k = (int)(c & 1);
    check_cuda(cudaMemcpyAsync(pinned_[k], static_cast<const unsigned char*>(src) + off, len,
                               cudaMemcpyDeviceToHost, s),
               "download copy");
    check_cuda(cudaEventRecord(pinned_ev_[k], s), "download chunk");
  };
  if (chunks) issue(0);
  for (size_t c = 0; c < chunks; ++c) {
    if (c + 1 < chunks) issue(c + 1);
    const size_t off = c * kXferChunk, len = std::min(kXferChunk, bytes - off);
    const int k = (int)(c & 1);
    check_cuda(cudaEventSynchronize(pinned_ev_[k]), "download chunk");
    std::memcpy(static_cast<unsigned char*>(dst) + off, pinned_[k], len);
  }
}

// ---------------------------------------------------------------- Batch impl
Batch::Batch(int precision) : prec_(precision) {
  if (precision != SNOW_FP64 && precision != SNOW_MIXED) throw Error(SNOW_E_ARG, "unknown precision");
  rsize_ = precision == SNOW_FP64 ? sizeof(double) : sizeof(float);
  d_ctr_ = dalloc<Counters>(1);
  check_cuda(cudaMemset(d_ctr_, 0, sizeof(Counters)), "cudaMemset");
  check_cuda(cudaMallocHost((void**)&h_ctr_buf_, kCtrSlots * sizeof(Counters)), "cudaMallocHost");
  std::memset(h_ctr_buf_, 0, kCtrSlots * sizeof(Counters));
  h_ctr_ = h_ctr_buf_;
  check_cuda(cudaStreamCreate(&own_stream_), "cudaStreamCreate");
}

Batch::~Batch() {
  if (pending_) cudaStreamSynchronize(pending_stream_);
  for (const Detached& d : detached_) {
    cudaEventSynchronize(d.ev);
    cudaEventDestroy(d.ev);
  }
  for (cudaEvent_t e : det_events_) cudaEventDestroy(e);
  for (HostStage& st : stage_)
    for (int k = 0; k < kStageBufs; ++k) {
      if (st.ev[k]) {
        cudaEventSynchronize(st.ev[k]);
        cudaEventDestroy(st.ev[k]);
      }
      if (st.p[k]) cudaFreeHost(st.p[k]);
    }
  drop_graph();
  for (auto& s : scenes_) free_scene(*s);
  dfree(d_scenes_);
  dfree(d_coll_);
  dfree(d_ctr_);
  if (h_ctr_buf_) cudaFreeHost(h_ctr_buf_);
  free_particle_buffers();
  free_grid();
  free_bins();
  dfree(staging_);
  dfree(d_tmp_scene_);
  free_implicit();
  for (auto& c : cache_) free_scene(c);
  for (int k = 0; k < 2; ++k) {
    if (pinned_ev_[k]) {
      cudaEventSynchronize(pinned_ev_[k]);
      cudaEventDestroy(pinned_ev_[k]);
    }
    if (pinned_[k]) cudaFreeHost(pinned_[k]);
  }
  defer_free_ = false;
  flush_released();
  if (own_stream_) cudaStreamDestroy(own_stream_);
}

void Batch::release_ptr(void* p) {
  if (!p) return;
  if (defer_free_) released_.push_back(p);
  else cudaFree(p);
}

void Batch::flush_released() {
  for (void* p : released_) cudaFree(p);
  released_.clear();
}

void Batch::free_scene(Scene& s) {
  for (int k = 0; k < 2; ++k) {
    if (s.slab) {
      s.r[k] = nullptr;
      s.fp[k] = nullptr;
      s.id[k] = nullptr;
    } else {
      dfree(s.r[k]);
      dfree(s.fp[k]);
      dfree(s.id[k]);
    }
  }
  s.slab.reset();
  dfree(s.snap);
}

void Batch::snapshot(int32_t id, cudaStream_t s) {
  step_complete();
  Scene* sc = find(id);
  const size_t rb = (size_t)sc->stride * kRealPlanes * rsize_, fb = (size_t)sc->stride * kFPPlanes * sizeof(double),
               ib = (size_t)sc->stride * sizeof(int32_t);
  if (!sc->snap) sc->snap = dalloc<unsigned char>(rb + fb + ib);
  check_cuda(cudaMemcpyAsync(sc->snap, sc->r[sc->cur], rb, cudaMemcpyDeviceToDevice, s), "snapshot");
  check_cuda(cudaMemcpyAsync(sc->snap + rb, sc->fp[sc->cur], fb, cudaMemcpyDeviceToDevice, s), "snapshot");
  check_cuda(cudaMemcpyAsync(sc->snap + rb + fb, sc->id[sc->cur], ib, cudaMemcpyDeviceToDevice, s), "snapshot");
}

void Batch::restore(int32_t id, cudaStream_t s) {
  step_complete();
  Scene* sc = find(id);
  if (!sc->snap) throw Error(SNOW_E_STATE, "restore: scene " + std::to_string(id) + " has no snapshot");
  const size_t rb = (size_t)sc->stride * kRealPlanes * rsize_, fb = (size_t)sc->stride * kFPPlanes * sizeof(double),
               ib = (size_t)sc->stride * sizeof(int32_t);
  check_cuda(cudaMemcpyAsync(sc->r[sc->cur], sc->snap, rb, cudaMemcpyDeviceToDevice, s), "restore");
  check_cuda(cudaMemcpyAsync(sc->fp[sc->cur], sc->snap + rb, fb, cudaMemcpyDeviceToDevice, s), "restore");
  check_cuda(cudaMemcpyAsync(sc->id[sc->cur], sc->snap + rb + fb, ib, cudaMemcpyDeviceToDevice, s), "restore");
  boxes_dirty_ = true;  // the particles moved back
}

void Batch::free_particle_buffers() {
  for (int k = 0; k < 2; ++k) {
    release(keys_[k]);
    release(vals_[k]);
  }
  release(hist_);
  release(fixups_);
  release(digit_total_);
  cap_p_ = 0;
}

void Batch::free_bins() {
  release(bins_);
  release(bin_off_);
  release(occ_);
  release(idmap_);
  release(bin_state_);
  cap_bins_ = 0;
}

// Dense key bins for key boxes of up to `bins` cells (rounded up to whole
// scan tiles).  Counts and occupancy start at zero; every step leaves them so.
void Batch::ensure_bins(int64_t bins) {
  bins = (bins + kBinTile - 1) / kBinTile * kBinTile;
  if (bins <= cap_bins_) return;
  free_bins();
  bins_ = dalloc<uint32_t>((size_t)bins);
  bin_off_ = dalloc<uint32_t>((size_t)bins);
  occ_ = dalloc<uint8_t>((size_t)(bins / 64));
  idmap_ = dalloc<int32_t>((size_t)(bins / 64));
  bin_state_ = dalloc<unsigned long long>((size_t)(bins / kBinTile + 1));
  cap_bins_ = bins;
  bins_dirty_ = true;
  // the next step's counts G2P emitted into the old bins are gone: a fresh key
  // space (and a re-measure unless the caller sizes the bins)
  keyspace_ready_ = false;
  if (!host_sized_) boxes_dirty_ = true;
}

// Chooses the sort for the coming steps: dense bins with 2x headroom over
// `key_blocks` block keys when that fits kMaxDenseBins, else the radix sort.
// Clears the counts if a step may have left some behind.
void Batch::size_dense(int64_t key_blocks, cudaStream_t s) {
  const int64_t need = 2 * key_blocks * 64 + 16 * kBinTile;
  const bool was = dense_;
  dense_ = want_dense_ && need <= kMaxDenseBins;
  if (dense_ != was) boxes_dirty_ = true;  // keys G2P emitted for the other sort are not used
  if (!dense_) return;
  ensure_bins(need);
  if (bins_dirty_) {
    check_cuda(cudaMemsetAsync(bins_, 0, (size_t)cap_bins_ * sizeof(uint32_t), s), "clear bins");
    check_cuda(cudaMemsetAsync(occ_, 0, (size_t)(cap_bins_ / 64), s), "clear bins");
    check_cuda(cudaMemsetAsync(bin_state_, 0, (size_t)(cap_bins_ / kBinTile + 1) * sizeof(unsigned long long), s),
               "clear bins");
    bins_dirty_ = false;
  }
}

void Batch::free_grid() {
  release(htab_);
  release(blk_);
  release(acc_);
  release(vel_);
  release(item_hdr_);
  cap_items_ = 0;
  cap_blocks_ = 0;
  hcap_ = 0;
}

void Batch::drop_graph() {
  if (gexec_) cudaGraphExecDestroy(gexec_);
  gexec_ = nullptr;
}

Scene* Batch::find(int32_t id) {
  for (auto& s : scenes_)
    if (s->sid == id) return s.get();
  throw Error(SNOW_E_STATE, "unknown scene id " + std::to_string(id));
}

void Batch::ensure_staging(int64_t n) {
  if (n <= staging_cap_) return;
  release(staging_);
  staging_ = dalloc<double>((size_t)std::max<int64_t>(n, 1) * 26);
  staging_cap_ = n;
}

static void validate_params(const snow_step_params* p) {
  if (!p) throw Error(SNOW_E_ARG, "params is NULL");
  if (!(p->grid_spacing > 0.0) || !std::isfinite(p->grid_spacing))
    throw Error(SNOW_E_ARG, "grid_spacing must be positive and finite");
  if (!std::isfinite(p->time_step)) throw Error(SNOW_E_ARG, "time_step must be finite");
}

int32_t Batch::add_scene(const double* records, int64_t n, const snow_step_params* params,
                         const snow_collider* colliders, int n_colliders, cudaStream_t s, bool wait) {
  if (n < 0 || (n > 0 && !records)) throw Error(SNOW_E_ARG, "bad particle array");
  if (n > INT32_MAX) throw Error(SNOW_E_ARG, "at most 2^31-1 particles per scene");
  validate_params(params);
  auto sc = std::make_unique<Scene>();
  sc->sid = next_id_++;
  sc->n = n;
  sc->stride = pad32(std::max<int64_t>(n, 1));
  // reuse the smallest cached buffer set that fits (at most twice the size)
  int best = -1;
  for (int c = 0; c < (int)cache_.size(); ++c)
    if (cache_[c].stride >= sc->stride && cache_[c].stride <= 2 * sc->stride &&
        (best < 0 || cache_[c].stride < cache_[best].stride))
      best = c;
  if (best >= 0) {
    Scene& c = cache_[best];
    cached_bytes_ -= scene_bytes(c.stride);
    sc->stride = c.stride;
    for (int k = 0; k < 2; ++k) {
      sc->r[k] = c.r[k];
      sc->fp[k] = c.fp[k];
      sc->id[k] = c.id[k];
    }
    sc->slab = std::move(c.slab);
    cache_.erase(cache_.begin() + best);
  } else {
    for (int k = 0; k < 2; ++k) {
      sc->r[k] = dalloc<unsigned char>((size_t)sc->stride * kRealPlanes * rsize_);
      sc->fp[k] = dalloc<double>((size_t)sc->stride * kFPPlanes);
      sc->id[k] = dalloc<int32_t>((size_t)sc->stride);
    }
  }
  sc->params = *params;
  set_colliders(*sc, colliders, n_colliders);
  Scene* raw = sc.get();
  scenes_.push_back(std::move(sc));
  dirty_ = true;
  upload(raw->sid, records, n, s, wait);
  return raw->sid;
}

void Batch::set_colliders(Scene& sc, const snow_collider* c, int n) {
  sc.colliders = device_colliders(c, n);
}

void Batch::remove_scene(int32_t id) {
  step_complete();
  for (size_t k = 0; k < scenes_.size(); ++k)
    if (scenes_[k]->sid == id) {
      // Keep the buffers for a later scene (serving admits and retires scenes
      // continuously); the cache holds at most cache_limit_ bytes.  This
      // batch has no work in flight (step_complete above; a copy left in
      // flight by wait = false has passed, by the caller's contract), so no
      // device-wide wait is needed.
      dfree(scenes_[k]->snap);
      Scene c;
      c.stride = scenes_[k]->stride;
      for (int b = 0; b < 2; ++b) {
        c.r[b] = scenes_[k]->r[b];
        c.fp[b] = scenes_[k]->fp[b];
        c.id[b] = scenes_[k]->id[b];
        scenes_[k]->r[b] = nullptr;
        scenes_[k]->fp[b] = nullptr;
        scenes_[k]->id[b] = nullptr;
      }
      c.slab = std::move(scenes_[k]->slab);
      cache_.push_back(c);
      cached_bytes_ += scene_bytes(c.stride);
      while (cached_bytes_ > cache_limit_ && !cache_.empty()) {
        cached_bytes_ -= scene_bytes(cache_.front().stride);
        free_scene(cache_.front());
        cache_.erase(cache_.begin());
      }
      scenes_.erase(scenes_.begin() + k);
      dirty_ = true;
      return;
    }
  throw Error(SNOW_E_STATE, "unknown scene id " + std::to_string(id));
}

void Batch::set_params(int32_t id, const snow_step_params* params, const snow_collider* c, int n) {
  validate_params(params);
  Scene* sc = find(id);
  sc->params = *params;
  set_colliders(*sc, c, n);
  params_dirty_ = true;
  force_dirty_ = true;
}

void Batch::upload(int32_t id, const double* records, int64_t n, cudaStream_t s, bool wait, bool keep_order) {
  step_complete();
  Scene* sc = find(id);
  if (n != sc->n) throw Error(SNOW_E_ARG, "upload: particle count differs from the scene's");
  if (n == 0) return;
  ensure_staging(n);
  copy_in(staging_, records, (size_t)n * 26 * sizeof(double), s, wait);
  const unsigned g = (unsigned)((n + 255) / 256);
  if (keep_order && prec_ == SNOW_FP64)
    k_records_to_planes_ordered<double><<<g, 256, 0, s>>>(staging_, n, (double*)sc->r[sc->cur], sc->fp[sc->cur],
                                                           sc->id[sc->cur], sc->stride, &d_ctr_->status);
  else if (keep_order)
    k_records_to_planes_ordered<float><<<g, 256, 0, s>>>(staging_, n, (float*)sc->r[sc->cur], sc->fp[sc->cur],
                                                          sc->id[sc->cur], sc->stride, &d_ctr_->status);
  else if (prec_ == SNOW_FP64)
    k_records_to_planes<double><<<g, 256, 0, s>>>(staging_, n, (double*)sc->r[sc->cur],
                                                   sc->fp[sc->cur], sc->id[sc->cur], sc->stride);
  else
    k_records_to_planes<float><<<g, 256, 0, s>>>(staging_, n, (float*)sc->r[sc->cur],
                                                  sc->fp[sc->cur], sc->id[sc->cur], sc->stride);
  check_cuda(cudaGetLastError(), "upload kernel");
  boxes_dirty_ = true;
  force_dirty_ = true;
}

void Batch::download(int32_t id, double* records, int64_t n, cudaStream_t s, bool wait) {
  step_complete();
  Scene* sc = find(id);
  if (n != sc->n) throw Error(SNOW_E_ARG, "download: particle count differs from the scene's");
  if (n == 0) return;
  ensure_staging(n);
  const unsigned g = (unsigned)((n + 255) / 256);
  if (prec_ == SNOW_FP64)
    k_planes_to_records<double><<<g, 256, 0, s>>>(staging_, n, (const double*)sc->r[sc->cur],
                                                   sc->fp[sc->cur], sc->id[sc->cur], sc->stride);
  else
    k_planes_to_records<float><<<g, 256, 0, s>>>(staging_, n, (const float*)sc->r[sc->cur],
                                                  sc->fp[sc->cur], sc->id[sc->cur], sc->stride);
  check_cuda(cudaGetLastError(), "download kernel");
  copy_out(records, staging_, (size_t)n * 26 * sizeof(double), s, wait);
}

void Batch::download_positions(int32_t id, double* xyz, int64_t n, cudaStream_t s) {
  step_complete();
  Scene* sc = find(id);
  if (n != sc->n) throw Error(SNOW_E_ARG, "download_positions: particle count differs from the scene's");
  if (n == 0) return;
  ensure_staging(n);
  const unsigned g = (unsigned)((n + 255) / 256);
  if (prec_ == SNOW_FP64)
    k_planes_to_positions<double><<<g, 256, 0, s>>>(staging_, n, (const double*)sc->r[sc->cur], sc->id[sc->cur],
                                                     sc->stride);
  else
    k_planes_to_positions<float><<<g, 256, 0, s>>>(staging_, n, (const float*)sc->r[sc->cur], sc->id[sc->cur],
                                                    sc->stride);
  check_cuda(cudaGetLastError(), "download kernel");
  copy_out(xyz, staging_, (size_t)n * 3 * sizeof(double), s, true);
}

SceneDev Batch::scene_dev(const Scene& sc, int64_t begin) const {
  SceneDev d{};
  for (int k = 0; k < 2; ++k) {
    d.r[k] = sc.r[k];
    d.fp[k] = sc.fp[k];
    d.id[k] = sc.id[k];
  }
  d.stride = sc.stride;
  d.n = sc.n;
  d.begin = begin;
  d.cur = sc.cur;
  d.active = 1;
  const snow_step_params& p = sc.params;
  d.dx = p.grid_spacing;
  d.dt = p.time_step;
  for (int a = 0; a < 3; ++a) d.g[a] = p.gravity[a];
  d.mu0 = p.mu_0;
  d.lambda0 = p.lambda_0;
  d.xi = p.hardening_coefficient;
  d.theta_c = p.max_compression;
  d.theta_s = p.max_stretch;
  d.alpha = p.alpha;
  for (int a = 0; a < 3; ++a) {
    d.nb_lo[a] = INT_MAX;
    d.nb_hi[a] = INT_MIN;
  }
  return d;
}

int auto_chunk(int64_t particles, int precision) {
  const int64_t per_sm = precision == SNOW_FP64 ? 2 : 3;
  const int64_t per = particles / (4 * per_sm * (int64_t)sm_count());
  int c = 256;
  while (c < 1024 && 2 * c <= per) c *= 2;
  return c;
}

void Batch::reserve(int64_t particles, int64_t staging, int scenes, int colliders) {
  if (particles < 0 || staging < 0 || scenes < 0 || colliders < 0) throw Error(SNOW_E_ARG, "negative reservation");
  step_complete();
  ensure_particle_buffers(particles);
  if (staging > 0) ensure_staging(staging);
  if (!d_tmp_scene_) d_tmp_scene_ = dalloc<SceneDev>(1);
  if (scenes > d_scenes_cap_) {
    release(d_scenes_);
    d_scenes_cap_ = scenes;
    d_scenes_ = dalloc<SceneDev>(d_scenes_cap_);
    dirty_ = true;  // the tables are written again before the next step
  }
  if (colliders > d_coll_cap_) {
    release(d_coll_);
    d_coll_cap_ = colliders;
    d_coll_ = dalloc<Collider>(d_coll_cap_);
    dirty_ = true;
  }
}

void Batch::ensure_particle_buffers(int64_t total) {
  if (total <= cap_p_) return;
  free_particle_buffers();
  // The next step's keys G2P emitted lived in the old buffers: the next step
  // computes every key again (a fresh key space), and measures the boxes
  // again unless the caller sizes the grid and bins (host-sized).
  keyspace_ready_ = false;
  if (!host_sized_) boxes_dirty_ = true;
  const int64_t cap = std::max<int64_t>(total, 1024);
  for (int k = 0; k < 2; ++k) {
    keys_[k] = dalloc<uint32_t>((size_t)cap);
    vals_[k] = dalloc<uint32_t>((size_t)cap);
  }
  ntiles_cap_ = radix_tiles(cap);
  hist_ = dalloc<uint32_t>((size_t)ntiles_cap_ * (1 << kRadixBits));
  if (prec_ == SNOW_MIXED) fixups_ = dalloc<int4>((size_t)cap);
  digit_total_ = dalloc<uint32_t>(1 << kRadixBits);
  cap_p_ = cap;
}

// Work items: one per chunk of the sorted particles, plus one more for every
// block run that starts inside a chunk.
void Batch::ensure_items() {
  const int64_t need = cap_p_ / chunk_ + cap_blocks_ + 64;
  if (need <= cap_items_) return;
  release(item_hdr_);
  item_hdr_ = dalloc<BlockHeader>((size_t)need);
  cap_items_ = (int32_t)need;
}

void Batch::ensure_grid(int64_t blocks) {
  if (blocks <= cap_blocks_) {
    ensure_items();
    return;
  }
  free_grid();
  const int64_t cap = std::max<int64_t>(blocks, 256);
  cap_blocks_ = (int32_t)cap;
  uint32_t h = 1;
  while (h < 2 * (uint64_t)cap) h <<= 1;
  hcap_ = h;
  htab_ = dalloc<unsigned long long>(h);
  blk_ = dalloc<int4>((size_t)cap);
  acc_ = dalloc<unsigned char>((size_t)cap * 64 * kAccCh * rsize_);
  vel_ = dalloc<unsigned char>((size_t)cap * 64 * kVelCh * rsize_);
  // zeroed on the batch's own stream and waited for alone: launches left in
  // flight on other streams (which use the old grid) are not waited for
  check_cuda(cudaMemsetAsync(acc_, 0, (size_t)cap * 64 * kAccCh * rsize_, own_stream_), "cudaMemset");
  check_cuda(cudaMemsetAsync(vel_, 0, (size_t)cap * 64 * kVelCh * rsize_, own_stream_), "cudaMemset");
  check_cuda(cudaStreamSynchronize(own_stream_), "cudaMemset");
  ensure_items();
}

BatchDev Batch::dev(SceneDev* scenes, int num_scenes, int64_t total) const {
  BatchDev b{};
  b.scenes = scenes;
  b.num_scenes = num_scenes;
  b.total = total;
  b.colliders = d_coll_;
  for (int k = 0; k < 2; ++k) {
    b.keys[k] = keys_[k];
    b.vals[k] = vals_[k];
  }
  b.hist = hist_;
  b.digit_total = digit_total_;
  b.ntiles = radix_tiles(std::max<int64_t>(total, 1));
  b.htab = htab_;
  b.hmask = hcap_ - 1;
  b.cap_blocks = cap_blocks_;
  b.blk = blk_;
  b.item_hdr = item_hdr_;
  b.cap_items = cap_items_;
  b.chunk = chunk_;
  b.fixups = fixups_;
  b.cap_fixups = fixups_ ? cap_p_ : 0;
  b.acc = acc_;
  b.vel = vel_;
  b.ctr = d_ctr_;
  b.imp_mass = imp_beta_ > 0.0 ? imp_nodes_ : nullptr;
  b.dense = dense_ ? 1 : 0;
  b.cap_bins = cap_bins_;
  b.bins = bins_;
  b.bin_off = bin_off_;
  b.occ = occ_;
  b.idmap = idmap_;
  b.bin_state = bin_state_;
  return b;
}

// Brings the device scene table, colliders, sort buffers and grid in line
// with the host's scenes after any change (scenes added or removed, particles
// uploaded, parameters changed): uploads the host copy of the table, measures
// every scene's block box from its particles, and grows the grid to twice the
// box volume so that the scenes can move.  Captured graphs stay valid unless a
// buffer moved (step() compares the launch arguments).
void Batch::prepare(cudaStream_t s) {
  if (!(dirty_ || boxes_dirty_ || params_dirty_)) return;
  keyspace_ready_ = false;  // the boxes are measured afresh below
  total_ = 0;
  table_.clear();
  coll_.clear();
  for (auto& sc : scenes_) {
    SceneDev d = scene_dev(*sc, total_);
    d.coll_begin = (int32_t)coll_.size();
    d.coll_count = (int32_t)sc->colliders.size();
    coll_.insert(coll_.end(), sc->colliders.begin(), sc->colliders.end());
    table_.push_back(d);
    total_ += sc->n;
  }
  if (chunk_auto_) {
    const int c = auto_chunk(total_, prec_);
    if (c != chunk_) {
      chunk_ = c;
      cap_items_ = 0;  // re-sized by ensure_grid below
    }
  }
  if ((int)table_.size() > d_scenes_cap_) {
    release(d_scenes_);
    d_scenes_cap_ = std::max<int>(16, (int)table_.size() * 2);
    d_scenes_ = dalloc<SceneDev>(d_scenes_cap_);
  }
  if ((int)coll_.size() > d_coll_cap_ || !d_coll_) {
    release(d_coll_);
    d_coll_cap_ = std::max<int>(16, (int)coll_.size() * 2);
    d_coll_ = dalloc<Collider>(d_coll_cap_);
  }
  if (!table_.empty()) staged_upload(stage_[0], d_scenes_, table_.data(), table_.size() * sizeof(SceneDev), s, "scene table");
  if (!coll_.empty()) staged_upload(stage_[1], d_coll_, coll_.data(), coll_.size() * sizeof(Collider), s, "colliders");
  ensure_particle_buffers(total_);
  const BatchDev b = dev(d_scenes_, (int)table_.size(), total_);
  if (prec_ == SNOW_FP64)
    StepLaunch<double>::bbox_init(b, s);
  else
    StepLaunch<float>::bbox_init(b, s);
  check_cuda(cudaGetLastError(), "bbox");
  if (host_sized_ && !boxes_dirty_ && cap_blocks_ > 0) {
    // the boxes are measured on the device for the key space; the grid and
    // bins are the caller's reservation
    ensure_items();
    num_dev_scenes_ = (int)table_.size();
    dirty_ = params_dirty_ = false;
    return;
  }
  std::vector<SceneDev> measured(table_.size());
  if (!measured.empty())
    check_cuda(cudaMemcpyAsync(measured.data(), d_scenes_, measured.size() * sizeof(SceneDev),
                               cudaMemcpyDeviceToHost, s),
               "scene table readback");
  check_cuda(cudaStreamSynchronize(s), "sync");
  int64_t vol = 0;
  for (const SceneDev& d : measured) {
    if (d.nb_lo[0] > d.nb_hi[0]) continue;
    int64_t v = 1;
    for (int a = 0; a < 3; ++a) v *= (int64_t)(d.nb_hi[a] - d.nb_lo[a] + 4);
    vol += v;
  }
  const int64_t want = std::max<int64_t>(2 * vol + 1024, 2 * last_blocks_ + 1024);
  ensure_grid(std::min<int64_t>(want, std::max<int64_t>(8 * total_ + 64, 1024)));
  size_dense(std::max<int64_t>(vol, last_key_blocks_), s);
  num_dev_scenes_ = (int)table_.size();
  dirty_ = boxes_dirty_ = params_dirty_ = false;
}

template <typename R>
void Batch::launch_step(const BatchDev& b, cudaStream_t s, cudaEvent_t* ev) {
  auto mark = [&](int k) {
    if (ev) cudaEventRecord(ev[k], s);
  };
  mark(0);
  // the key boxes of this step were prepared by the previous step's last
  // launch (or by step() before the first one)
  StepLaunch<R>::keys(b, s);
  radix_sort(b, s);
  StepLaunch<R>::blocks(b, s);
  mark(1);
  StepLaunch<R>::p2g(b, P2G_PRE, s);
  mark(2);
  StepLaunch<R>::grid_update(b, s);
  if (b.imp_mass) implicit_solve<R>(b, s);
  mark(3);
  StepLaunch<R>::g2p(b, G2P_FULL, s);
  StepLaunch<R>::fixup(b, s);
  StepLaunch<R>::finish_and_keyspace(b, s);
  mark(4);
}

void Batch::step(int n_steps, snow_step_timings* timings, cudaStream_t s) {
  step_launch(n_steps, timings, s);
  step_complete();
}

// Moves scene `id` of `from` (same precision) into this batch without copying
// its particles; returns its id here.  The server sets scenes up in a separate
// batch while this one steps, then moves them in.
int32_t Batch::adopt_scene(Batch& from, int32_t id) {
  step_complete();
  if (from.prec_ != prec_) throw Error(SNOW_E_ARG, "adopt_scene: precisions differ");
  for (size_t k = 0; k < from.scenes_.size(); ++k)
    if (from.scenes_[k]->sid == id) {
      std::unique_ptr<Scene> sc = std::move(from.scenes_[k]);
      from.scenes_.erase(from.scenes_.begin() + k);
      from.dirty_ = true;
      sc->sid = next_id_++;
      const int32_t sid = sc->sid;
      scenes_.push_back(std::move(sc));
      dirty_ = true;
      force_dirty_ = true;
      return sid;
    }
  throw Error(SNOW_E_STATE, "unknown scene id " + std::to_string(id));
}

// Launches n_steps steps on stream s without waiting for them; step_complete()
// waits and checks their status.
void Batch::step_launch(int n_steps, snow_step_timings* timings, cudaStream_t s) {
  if (n_steps < 0) throw Error(SNOW_E_ARG, "negative step count");
  if (pending_) step_complete();
  if (n_steps == 0 || scenes_.empty()) return;
  // The legacy NULL stream cannot be captured into a graph: run on the batch's
  // own (blocking) stream instead, which orders itself with NULL-stream work.
  if (!s) s = own_stream_;
  prepare(s);
  if (imp_beta_ > 0.0) ensure_implicit();  // sized for this step's grid and particles
  const BatchDev b = dev(d_scenes_, num_dev_scenes_, total_);
  if (force_dirty_) {
    // P2G reads each particle's force matrix, which G2P keeps current from step
    // to step; compute it afresh after an upload, setup() or parameter change.
    if (prec_ == SNOW_FP64)
      StepLaunch<double>::prepare_force(b, s);
    else
      StepLaunch<float>::prepare_force(b, s);
    check_cuda(cudaGetLastError(), "prepare force");
    force_dirty_ = false;
  }
  if (!keyspace_ready_) {
    // key boxes of the first step; every step ends by preparing the next one's
    if (prec_ == SNOW_FP64)
      StepLaunch<double>::keyspace(b, s, false);
    else
      StepLaunch<float>::keyspace(b, s, false);
    keyspace_ready_ = true;
  }
  auto one = [&](cudaEvent_t* ev) {
    if (prec_ == SNOW_FP64)
      launch_step<double>(b, s, ev);
    else
      launch_step<float>(b, s, ev);
  };
  if (timings) {
    cudaEvent_t ev[5];
    for (auto& e : ev) check_cuda(cudaEventCreate(&e), "event");
    for (int k = 0; k < n_steps; ++k) {
      one(ev);
      check_cuda(cudaEventSynchronize(ev[4]), "step");
      float ms[4];
      for (int q = 0; q < 4; ++q) cudaEventElapsedTime(&ms[q], ev[q], ev[q + 1]);
      timings->stencil += ms[0];
      timings->p2g += ms[1];
      timings->grid_velocity += ms[2];
      timings->stress_update += ms[3];
    }
    for (auto& e : ev) cudaEventDestroy(e);
  } else if (use_graphs_ && imp_beta_ == 0.0) {  // the implicit solve reads back scalars: no graph
    int k = 0;
    if (!gexec_ && !graph_warm_) {
      // the batch's first step eagerly (initialises per-kernel launch
      // settings); every later call captures or replays, also one step at a
      // time as the drop-in step() calls it
      one(nullptr);
      check_cuda(cudaGetLastError(), "step launch");
      ++k;
      graph_warm_ = true;
    }
    if (k < n_steps && (!gexec_ || std::memcmp(&graph_args_, &b, sizeof b) != 0)) {
      cudaGraph_t g;
      check_cuda(cudaStreamBeginCapture(s, cudaStreamCaptureModeThreadLocal), "capture");
      one(nullptr);
      check_cuda(cudaStreamEndCapture(s, &g), "capture end");
      {
        size_t nodes = 0;
        check_cuda(cudaGraphGetNodes(g, nullptr, &nodes), "graph nodes");
        std::vector<cudaGraphNode_t> list(nodes);
        check_cuda(cudaGraphGetNodes(g, list.data(), &nodes), "graph nodes");
        graph_kernels_ = 0;
        for (cudaGraphNode_t nd : list) {
          cudaGraphNodeType type;
          check_cuda(cudaGraphNodeGetType(nd, &type), "graph node type");
          if (type == cudaGraphNodeTypeKernel) ++graph_kernels_;
        }
      }
      // A buffer moved or the scenes changed: when the step launches the same
      // kernels, only their arguments and grids differ and the executable
      // graph is updated in place; otherwise it is instantiated anew.
      bool updated = false;
      if (gexec_) {
        cudaGraphExecUpdateResultInfo info{};
        updated = cudaGraphExecUpdate(gexec_, g, &info) == cudaSuccess;
        if (!updated) {
          cudaGetLastError();
          drop_graph();
        }
      }
      if (!updated) {
        const cudaError_t e = cudaGraphInstantiate(&gexec_, g, 0);
        cudaGraphDestroy(g);
        check_cuda(e, "graph instantiate");
      } else {
        cudaGraphDestroy(g);
      }
      graph_args_ = b;
    }
    for (; k < n_steps; ++k) check_cuda(cudaGraphLaunch(gexec_, s), "graph launch");
  } else {
    for (int k = 0; k < n_steps; ++k) one(nullptr);
  }
  check_cuda(cudaGetLastError(), "step launch");
  for (auto& sc : scenes_) sc->cur ^= (n_steps & 1);
  check_cuda(cudaMemcpyAsync(h_ctr_, d_ctr_, sizeof(Counters), cudaMemcpyDeviceToHost, s), "status");
  pending_ = true;
  pending_stream_ = s;
}

void Batch::step_complete() {
  if (!pending_) return;
  pending_ = false;
  check_cuda(cudaStreamSynchronize(pending_stream_), "step");
  // the stream sync covered the launches left behind too
  for (const Detached& d : detached_) det_events_.push_back(d.ev);
  detached_.clear();
  absorb(*h_ctr_);
}

void Batch::step_detach() {
  if (!pending_) return;
  if ((int)detached_.size() >= kCtrSlots - 1) complete_detached();
  cudaEvent_t ev = nullptr;
  if (!det_events_.empty()) {
    ev = det_events_.back();
    det_events_.pop_back();
  } else {
    check_cuda(cudaEventCreateWithFlags(&ev, cudaEventDisableTiming), "cudaEventCreate");
  }
  check_cuda(cudaEventRecord(ev, pending_stream_), "cudaEventRecord");
  detached_.push_back(Detached{ev, h_ctr_});
  // the next launch's counters go to a slot no launch in flight writes
  for (int k = 0; k < kCtrSlots; ++k) {
    Counters* c = h_ctr_buf_ + k;
    bool used = false;
    for (const Detached& d : detached_) used |= d.ctr == c;
    if (!used) {
      h_ctr_ = c;
      break;
    }
  }
  pending_ = false;
}

void Batch::complete_detached() {
  if (detached_.empty()) return;
  const Detached d = detached_.front();
  detached_.pop_front();
  det_events_.push_back(d.ev);
  check_cuda(cudaEventSynchronize(d.ev), "step");
  absorb(*d.ctr);
}

void Batch::absorb(const Counters& c) {
  last_status_ = c.status;
  last_blocks_ = (int64_t)c.last_blocks;
  last_key_blocks_ = (int64_t)c.key_blocks;
  // Keep 2x headroom: grow the grid and the bins before the next call if the
  // last step came close.
  if (last_blocks_ * 2 > cap_blocks_) boxes_dirty_ = true;
  if (dense_ && last_key_blocks_ * 64 * 2 > cap_bins_) boxes_dirty_ = true;
  check_status();
}

void Batch::staged_upload(HostStage& st, void* dst, const void* src, size_t bytes, cudaStream_t s, const char* what) {
  const int k = st.next;
  st.next = (st.next + 1) % kStageBufs;
  if (st.ev[k]) check_cuda(cudaEventSynchronize(st.ev[k]), what);  // its last copy has passed
  else check_cuda(cudaEventCreateWithFlags(&st.ev[k], cudaEventDisableTiming), "cudaEventCreate");
  if (st.cap[k] < bytes) {
    if (st.p[k]) cudaFreeHost(st.p[k]);
    st.p[k] = nullptr;
    st.cap[k] = 0;
    check_cuda(cudaMallocHost(&st.p[k], 2 * bytes), "cudaMallocHost");
    st.cap[k] = 2 * bytes;
  }
  std::memcpy(st.p[k], src, bytes);
  check_cuda(cudaMemcpyAsync(dst, st.p[k], bytes, cudaMemcpyHostToDevice, s), what);
  check_cuda(cudaEventRecord(st.ev[k], s), what);
}

void Batch::check_status() {
  const uint32_t st = last_status_;
  if (!st) return;
  cudaMemset(&d_ctr_->status, 0, sizeof(uint32_t));
  bins_dirty_ = true;  // a step that stopped early may leave counts behind
  boxes_dirty_ = true;
  keyspace_ready_ = false;
  if (st & ST_BIN_OVERFLOW)
    throw Error(SNOW_E_CAPACITY, "scene key boxes outgrew the dense bins (" + std::to_string(cap_bins_) +
                                     "); the step result is not valid");
  if (st & ST_SCAN_STALL) throw Error(SNOW_E_STATE, "bin scan stalled; the step result is not valid");
  if (st & (ST_BLOCK_OVERFLOW | ST_HASH_FULL))
    throw Error(SNOW_E_CAPACITY, "grid block capacity exceeded (" + std::to_string(cap_blocks_) +
                                     " blocks); the step result is not valid");
  if (st & ST_NONFINITE) throw Error(SNOW_E_NONFINITE, "a particle position became NaN or infinite");
  if (st & ST_KEY_OVERFLOW)
    throw Error(SNOW_E_KEYRANGE, "scene extent exceeds the 32-bit block key range");
  if (st & (ST_OUT_OF_BOX | ST_LOOKUP_MISS))
    throw Error(SNOW_E_STATE, "internal grid inconsistency (status " + std::to_string(st) + ")");
}

// setup() for one scene: a private one-scene view over the batch's buffers.
void Batch::setup(int32_t id, double dx, cudaStream_t s, int64_t box_blocks, bool wait) {
  step_complete();
  keyspace_ready_ = false;  // setup's own steps reuse the counters
  if (!(dx > 0.0)) throw Error(SNOW_E_ARG, "grid_spacing must be positive");
  Scene* sc = find(id);
  if (sc->n == 0) return;
  if (!d_tmp_scene_) d_tmp_scene_ = dalloc<SceneDev>(1);
  SceneDev d = scene_dev(*sc, 0);
  d.dx = dx;
  check_cuda(cudaMemcpyAsync(d_tmp_scene_, &d, sizeof d, cudaMemcpyHostToDevice, s), "tmp scene");
  ensure_particle_buffers(sc->n);
  {
    // measure this scene's block box at the setup spacing and size the grid for it
    const BatchDev b0 = dev(d_tmp_scene_, 1, sc->n);
    if (prec_ == SNOW_FP64)
      StepLaunch<double>::bbox_init(b0, s);
    else
      StepLaunch<float>::bbox_init(b0, s);
    int64_t vol = box_blocks;
    if (vol < 0) {
      check_cuda(cudaMemcpyAsync(&d, d_tmp_scene_, sizeof d, cudaMemcpyDeviceToHost, s), "box");
      check_cuda(cudaStreamSynchronize(s), "sync");
      vol = 1;
      for (int a = 0; a < 3; ++a) vol *= (int64_t)(d.nb_hi[a] - d.nb_lo[a] + 4);
    }
    // 2x headroom, as for steps: a batch that sets up scenes one after
    // another regrows (and frees) its grid only when the box doubles
    ensure_grid(std::min<int64_t>(2 * vol + 1024, 8 * sc->n + 1024));
    size_dense(vol, s);
  }
  const BatchDev b = dev(d_tmp_scene_, 1, sc->n);
  auto run = [&](auto tag) {
    using R = decltype(tag);
    StepLaunch<R>::keyspace(b, s, true);
    StepLaunch<R>::keys(b, s);
    radix_sort(b, s);
    StepLaunch<R>::blocks(b, s);
    StepLaunch<R>::p2g(b, P2G_MASS, s);
    StepLaunch<R>::g2p(b, G2P_VOLUME, s);
    StepLaunch<R>::zero_grid(b, s);
  };
  if (prec_ == SNOW_FP64)
    run(double{});
  else
    run(float{});
  check_cuda(cudaGetLastError(), "setup launch");
  check_cuda(cudaMemcpyAsync(h_ctr_, d_ctr_, sizeof(Counters), cudaMemcpyDeviceToHost, s), "status");
  force_dirty_ = true;  // V_p0 changed
  if (!wait) return;
  check_cuda(cudaStreamSynchronize(s), "setup");
  collect_status();
}

// Status flags accumulate in the counters until read here, so one read covers
// every setup left in flight before it.
void Batch::collect_status() {
  last_status_ = h_ctr_->status;
  check_status();
}

void Batch::reserve_grid(int64_t blocks, int64_t key_blocks, cudaStream_t s) {
  if (blocks < 0 || key_blocks < 0) throw Error(SNOW_E_ARG, "negative reservation");
  step_complete();
  if (blocks > 0) ensure_grid(blocks);
  if (key_blocks > 0) size_dense(key_blocks, s);
}

void Batch::reserve_scenes(const std::vector<int64_t>& sizes, int64_t max_bytes) {
  const auto al = [](size_t x) { return (x + 255) / 256 * 256; };
  std::vector<int64_t> strides;
  size_t total = 0;
  int64_t bytes = 0;
  // sizes that a cached buffer set would serve (add_scene's rule: the
  // smallest at most twice the size), each cached set counted once
  std::vector<bool> taken(cache_.size(), false);
  for (int64_t n : sizes) {
    const int64_t st = pad32(std::max<int64_t>(n, 1));
    int best = -1;
    for (int c = 0; c < (int)cache_.size(); ++c)
      if (!taken[c] && cache_[c].stride >= st && cache_[c].stride <= 2 * st &&
          (best < 0 || cache_[c].stride < cache_[best].stride))
        best = c;
    if (best >= 0) {
      taken[best] = true;
      continue;
    }
    if (bytes + scene_bytes(st) > max_bytes) break;
    bytes += scene_bytes(st);
    strides.push_back(st);
    total += 2 * (al((size_t)st * kRealPlanes * rsize_) + al((size_t)st * kFPPlanes * 8) + al((size_t)st * 4));
  }
  if (strides.empty()) return;
  unsigned char* base = dalloc<unsigned char>(total);
  std::shared_ptr<void> slab(base, [](void* p) { cudaFree(p); });
  size_t off = 0;
  for (int64_t st : strides) {
    Scene c;
    c.stride = st;
    for (int k = 0; k < 2; ++k) {
      c.r[k] = base + off;
      off += al((size_t)st * kRealPlanes * rsize_);
      c.fp[k] = reinterpret_cast<double*>(base + off);
      off += al((size_t)st * kFPPlanes * 8);
      c.id[k] = reinterpret_cast<int32_t*>(base + off);
      off += al((size_t)st * 4);
    }
    c.slab = slab;
    cache_.push_back(c);
    cached_bytes_ += scene_bytes(st);
  }
  cache_limit_ = std::max(cache_limit_, cached_bytes_);
}

// Work-item-size autotuner.  Each candidate runs from the same snapshot of the
// particle state (restored afterwards), two warm-up steps (the second captures
// the step graph), then `trial_steps` timed steps on the stream.
int Batch::autotune(int trial_steps, double* best_ms, cudaStream_t s) {
  if (trial_steps <= 0) throw Error(SNOW_E_ARG, "trial_steps must be positive");
  if (scenes_.empty()) throw Error(SNOW_E_STATE, "empty batch");
  if (!s) s = own_stream_;
  struct Snap {
    Scene* sc;
    int cur;
    unsigned char* buf;
    size_t r_bytes, fp_bytes, id_bytes;
  };
  std::vector<Snap> snaps;
  for (auto& sc : scenes_) {
    Snap sn{sc.get(), sc->cur, nullptr, (size_t)sc->stride * kRealPlanes * rsize_,
            (size_t)sc->stride * kFPPlanes * sizeof(double), (size_t)sc->stride * sizeof(int32_t)};
    sn.buf = dalloc<unsigned char>(sn.r_bytes + sn.fp_bytes + sn.id_bytes);
    check_cuda(cudaMemcpyAsync(sn.buf, sc->r[sc->cur], sn.r_bytes, cudaMemcpyDeviceToDevice, s), "snapshot");
    check_cuda(cudaMemcpyAsync(sn.buf + sn.r_bytes, sc->fp[sc->cur], sn.fp_bytes, cudaMemcpyDeviceToDevice, s), "snapshot");
    check_cuda(cudaMemcpyAsync(sn.buf + sn.r_bytes + sn.fp_bytes, sc->id[sc->cur], sn.id_bytes,
                               cudaMemcpyDeviceToDevice, s), "snapshot");
    snaps.push_back(sn);
  }
  auto restore = [&] {
    for (auto& sn : snaps) {
      Scene* sc = sn.sc;
      sc->cur = sn.cur;
      check_cuda(cudaMemcpyAsync(sc->r[sc->cur], sn.buf, sn.r_bytes, cudaMemcpyDeviceToDevice, s), "restore");
      check_cuda(cudaMemcpyAsync(sc->fp[sc->cur], sn.buf + sn.r_bytes, sn.fp_bytes, cudaMemcpyDeviceToDevice, s),
                 "restore");
      check_cuda(cudaMemcpyAsync(sc->id[sc->cur], sn.buf + sn.r_bytes + sn.fp_bytes, sn.id_bytes,
                                 cudaMemcpyDeviceToDevice, s), "restore");
    }
    boxes_dirty_ = true;
    force_dirty_ = true;
  };
  const int candidates[] = {64, 128, 256, 512, 1024};
  const bool dense_allowed = want_dense_;
  int best = chunk_;
  bool best_dense = want_dense_;
  double best_t = 1e300;
  cudaEvent_t e0, e1;
  check_cuda(cudaEventCreate(&e0), "event");
  check_cuda(cudaEventCreate(&e1), "event");
  for (int m = 0; m < (dense_allowed ? 2 : 1); ++m)
  for (int c : candidates) {
    const bool dense = dense_allowed && m == 0;
    set_chunk(c);
    set_dense(dense);
    restore();
    step(2, nullptr, s);
    check_cuda(cudaEventRecord(e0, s), "event");
    step(trial_steps, nullptr, s);
    check_cuda(cudaEventRecord(e1, s), "event");
    check_cuda(cudaEventSynchronize(e1), "event");
    float ms = 0;
    cudaEventElapsedTime(&ms, e0, e1);
    if (ms < best_t) {
      best_t = ms;
      best = c;
      best_dense = dense;
    }
  }
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  set_chunk(best);
  set_dense(best_dense);
  restore();
  check_cuda(cudaStreamSynchronize(s), "restore");
  for (auto& sn : snaps) dfree(sn.buf);
  if (best_ms) *best_ms = best_t / trial_steps;
  return best;
}

int64_t Batch::device_bytes() const {
  int64_t b = 0;
  for (auto& sc : scenes_) b += 2 * sc->stride * (kRealPlanes * (int64_t)rsize_ + kFPPlanes * 8 + 4);
  b += cap_p_ * 16 + (int64_t)ntiles_cap_ * (1 << kRadixBits) * 4;
  if (prec_ == SNOW_MIXED) b += cap_p_ * (int64_t)sizeof(int4);
  b += (int64_t)cap_blocks_ * (64 * (kAccCh + kVelCh) * (int64_t)rsize_ + 16) + (int64_t)hcap_ * 8;
  b += (int64_t)cap_items_ * (int64_t)sizeof(BlockHeader);
  b += cap_bins_ * 8 + cap_bins_ / 64 * 5 + (cap_bins_ / kBinTile + 1) * 8;
  b += staging_cap_ * 208;
  b += cached_bytes_;
  return b;
}

}  // namespace snow

// =================================================================== C ABI
using snow::Batch;
using snow::Error;

struct snow_gpu_batch {
  std::unique_ptr<Batch> impl;
};

namespace {
template <typename F>
int guarded(F&& f) {
  try {
    f();
    return SNOW_OK;
  } catch (const Error& e) {
    return snow::set_error(e.code, e.what());
  } catch (const std::exception& e) {
    return snow::set_error(SNOW_E_ARG, e.what());
  }
}
cudaStream_t as_stream(void* s) { return static_cast<cudaStream_t>(s); }
}  // namespace

extern "C" {

int snow_gpu_abi_version(void) { return SNOW_GPU_ABI_VERSION; }
const char* snow_gpu_last_error(void) { return snow::g_last_error.c_str(); }

int snow_gpu_init(int device) {
  return guarded([&] {
    int n = 0;
    snow::check_cuda(cudaGetDeviceCount(&n), "cudaGetDeviceCount");
    if (device < 0 || device >= n) throw Error(SNOW_E_ARG, "no CUDA device " + std::to_string(device));
    snow::check_cuda(cudaSetDevice(device), "cudaSetDevice");
    snow::check_cuda(cudaFree(nullptr), "context");
  });
}

int snow_gpu_make_plane(const double point[3], const double normal[3], double friction,
                        snow_collider* out) {
  if (!point || !normal || !out) return snow::set_error(SNOW_E_ARG, "NULL argument");
  std::memset(out, 0, sizeof *out);
  out->kind = SNOW_COLLIDER_PLANE;
  const double len = std::sqrt(normal[0] * normal[0] + normal[1] * normal[1] + normal[2] * normal[2]);
  for (int a = 0; a < 3; ++a) {
    out->point[a] = point[a];
    out->normal[a] = len > 0.0 ? normal[a] / len : normal[a];
  }
  out->friction = friction;
  return SNOW_OK;
}

int snow_gpu_batch_create(snow_gpu_batch** out, int precision) {
  return guarded([&] {
    if (!out) throw Error(SNOW_E_ARG, "out is NULL");
    auto* b = new snow_gpu_batch;
    try {
      b->impl = std::make_unique<Batch>(precision);
    } catch (...) {
      delete b;
      throw;
    }
    *out = b;
  });
}

int snow_gpu_batch_destroy(snow_gpu_batch* batch) {
  return guarded([&] {
    if (!batch) return;
    cudaDeviceSynchronize();
    delete batch;
  });
}

#define SNOW_BATCH_OR_FAIL \
  if (!batch || !batch->impl) throw Error(SNOW_E_ARG, "batch is NULL")

int snow_gpu_batch_add_scene(snow_gpu_batch* batch, const double* records, int64_t n,
                             const snow_step_params* params, const snow_collider* colliders,
                             int n_colliders, int32_t* scene_id, void* stream) {
  return guarded([&] {
    SNOW_BATCH_OR_FAIL;
    const int32_t id = batch->impl->add_scene(records, n, params, colliders, n_colliders, as_stream(stream));
    if (scene_id) *scene_id = id;
  });
}
int snow_gpu_batch_remove_scene(snow_gpu_batch* batch, int32_t scene_id) {
  return guarded([&] {
    SNOW_BATCH_OR_FAIL;
    batch->impl->remove_scene(scene_id);
  });
}
int snow_gpu_batch_set_params(snow_gpu_batch* batch, int32_t scene_id, const snow_step_params* params,
                              const snow_collider* colliders, int n_colliders) {
  return guarded([&] {
    SNOW_BATCH_OR_FAIL;
    batch->impl->set_params(scene_id, params, colliders, n_colliders);
  });
}
int snow_gpu_batch_upload(snow_gpu_batch* batch, int32_t scene_id, const double* records, int64_t n,
                          void* stream) {
  return guarded([&] {
    SNOW_BATCH_OR_FAIL;
    batch->impl->upload(scene_id, records, n, as_stream(stream));
  });
}
int snow_gpu_batch_download(snow_gpu_batch* batch, int32_t scene_id, double* records, int64_t n,
                            void* stream) {
  return guarded([&] {
    SNOW_BATCH_OR_FAIL;
    batch->impl->download(scene_id, records, n, as_stream(stream));
  });
}
int snow_gpu_batch_download_positions(snow_gpu_batch* batch, int32_t scene_id, double* xyz, int64_t n,
                                      void* stream) {
  return guarded([&] {
    SNOW_BATCH_OR_FAIL;
    if (n > 0 && !xyz) throw Error(SNOW_E_ARG, "NULL position buffer");
    batch->impl->download_positions(scene_id, xyz, n, as_stream(stream));
  });
}
int snow_gpu_batch_snapshot(snow_gpu_batch* batch, int32_t scene_id, void* stream) {
  return guarded([&] {
    SNOW_BATCH_OR_FAIL;
    batch->impl->snapshot(scene_id, as_stream(stream));
  });
}
int snow_gpu_batch_restore(snow_gpu_batch* batch, int32_t scene_id, void* stream) {
  return guarded([&] {
    SNOW_BATCH_OR_FAIL;
    batch->impl->restore(scene_id, as_stream(stream));
  });
}
int snow_gpu_batch_setup(snow_gpu_batch* batch, int32_t scene_id, double grid_spacing, void* stream) {
  return guarded([&] {
    SNOW_BATCH_OR_FAIL;
    batch->impl->setup(scene_id, grid_spacing, as_stream(stream));
  });
}
int snow_gpu_batch_step(snow_gpu_batch* batch, int n_steps, snow_step_timings* timings, void* stream) {
  return guarded([&] {
    SNOW_BATCH_OR_FAIL;
    batch->impl->step(n_steps, timings, as_stream(stream));
  });
}
int snow_gpu_batch_scene_count(snow_gpu_batch* batch) {
  return batch && batch->impl ? batch->impl->scene_count() : SNOW_E_ARG;
}
int64_t snow_gpu_batch_particles(snow_gpu_batch* batch) {
  return batch && batch->impl ? batch->impl->particles() : SNOW_E_ARG;
}
int64_t snow_gpu_batch_device_bytes(snow_gpu_batch* batch) {
  return batch && batch->impl ? batch->impl->device_bytes() : SNOW_E_ARG;
}
int snow_gpu_batch_status(snow_gpu_batch* batch, uint32_t* status, int64_t* used, int64_t* cap) {
  return guarded([&] {
    SNOW_BATCH_OR_FAIL;
    if (status) *status = batch->impl->last_status();
    if (used) *used = batch->impl->last_blocks();
    if (cap) *cap = batch->impl->capacity_blocks();
  });
}
int snow_gpu_batch_autotune(snow_gpu_batch* batch, int trial_steps, int* chosen, double* ms_per_step,
                            void* stream) {
  return guarded([&] {
    SNOW_BATCH_OR_FAIL;
    const int c = batch->impl->autotune(trial_steps, ms_per_step, as_stream(stream));
    if (chosen) *chosen = c;
  });
}
int64_t snow_gpu_batch_fp64_projections(snow_gpu_batch* batch) {
  return batch && batch->impl ? batch->impl->last_fp64_projections() : SNOW_E_ARG;
}
int snow_gpu_batch_set_chunk(snow_gpu_batch* batch, int chunk) {
  return guarded([&] {
    SNOW_BATCH_OR_FAIL;
    batch->impl->set_chunk(chunk);
  });
}
int snow_gpu_batch_chunk(snow_gpu_batch* batch) {
  return batch && batch->impl ? batch->impl->chunk() : SNOW_E_ARG;
}
int snow_gpu_batch_set_implicit(snow_gpu_batch* batch, double beta, double tolerance, int max_iterations) {
  return guarded([&] {
    SNOW_BATCH_OR_FAIL;
    batch->impl->set_implicit(beta, tolerance, max_iterations);
  });
}
int snow_gpu_batch_implicit_stats(snow_gpu_batch* batch, int* iterations, double* residual) {
  return guarded([&] {
    SNOW_BATCH_OR_FAIL;
    batch->impl->implicit_stats(iterations, residual);
  });
}
int snow_gpu_batch_sort_mode(snow_gpu_batch* batch) {
  return batch && batch->impl ? (batch->impl->dense() ? 1 : 0) : SNOW_E_ARG;
}
int snow_gpu_batch_graph_kernels(snow_gpu_batch* batch) {
  return batch && batch->impl ? batch->impl->graph_kernels() : SNOW_E_ARG;
}
int snow_gpu_batch_set_dense(snow_gpu_batch* batch, int enable) {
  return guarded([&] {
    SNOW_BATCH_OR_FAIL;
    batch->impl->set_dense(enable != 0);
  });
}
int snow_gpu_batch_set_graphs(snow_gpu_batch* batch, int enable) {
  return guarded([&] {
    SNOW_BATCH_OR_FAIL;
    batch->impl->set_graphs(enable != 0);
  });
}

// One-scene convenience entry points on host records (the literal drop-in:
// upload, run, download on every call).
static std::mutex g_single_mu;
static std::unique_ptr<Batch> g_single;
// True while the one-scene batch's id plane is a permutation of its records
// (the last call on it completed): the next step call uploads into the slots
// the last step left, in block-sorted order.
static bool g_single_ordered = false;

static Batch& single_batch() {
  if (!g_single) g_single = std::make_unique<Batch>(SNOW_FP64);
  return *g_single;
}

int snow_gpu_setup(double* records, int64_t n, double grid_spacing) {
  std::lock_guard<std::mutex> lk(g_single_mu);
  return guarded([&] {
    if (n < 0 || (n > 0 && !records)) throw Error(SNOW_E_ARG, "bad particle array");
    if (n == 0) return;
    Batch& b = single_batch();
    g_single_ordered = false;
    b.clear();
    snow_step_params p{};
    p.grid_spacing = grid_spacing;
    const int32_t id = b.add_scene(records, n, &p, nullptr, 0, nullptr);
    b.setup(id, grid_spacing, nullptr);
    b.download(id, records, n, nullptr);
    g_single_ordered = true;
  });
}

int snow_gpu_step(double* records, int64_t n, const snow_step_params* params,
                  const snow_collider* colliders, int n_colliders, int n_steps,
                  snow_step_timings* timings) {
  std::lock_guard<std::mutex> lk(g_single_mu);
  return guarded([&] {
    if (n < 0 || (n > 0 && !records)) throw Error(SNOW_E_ARG, "bad particle array");
    if (n == 0 || n_steps == 0) return;
    Batch& b = single_batch();
    int32_t id;
    const bool ordered = g_single_ordered;
    g_single_ordered = false;
    if (b.scene_count() == 1 && b.particles() == n) {
      id = b.first_id();
      b.set_params(id, params, colliders, n_colliders);
      b.upload(id, records, n, nullptr, true, ordered);
    } else {
      b.clear();
      id = b.add_scene(records, n, params, colliders, n_colliders, nullptr);
    }
    b.step(n_steps, timings, nullptr);
    b.download(id, records, n, nullptr);
    g_single_ordered = true;
  });
}

}  // extern "C"
