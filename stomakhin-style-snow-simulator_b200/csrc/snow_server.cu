// Continuous-batching server for independent snow scenes (no counterpart in
// the reference, which steps one scene in a loop).
//
// Requests -- a particle set, its step parameters and colliders, a number of
// steps and an arrival time -- are queued, then admitted as their arrival time
// passes and the device-memory budget and scene slots allow.  Admitted scenes
// stay resident; every tick advances all of them together by the same number
// of steps (one launch per kernel for the whole batch, replayed from a CUDA
// graph), at most until the next scene finishes; requests that arrive are
// uploaded and set up, and finished scenes copied back, on other streams
// while a tick runs.  A finished scene is copied
// back, removed, and its latency (arrival to result) recorded.  Scenes do not
// interact, so each result is the one the scene would get alone.
#include <algorithm>
#include <chrono>
#include <cmath>
#include <deque>
#include <memory>
#include <numeric>
#include <thread>
#include <vector>

#include "snow_engine.hpp"
#include "snow_gpu.h"

namespace snow {
namespace {

using clock_t_ = std::chrono::steady_clock;

struct Request {
  int64_t id = 0;
  std::vector<double> records;
  snow_step_params params{};
  std::vector<snow_collider> colliders;
  int64_t steps = 0;
  double arrival = 0.0;   // seconds on the server clock
  // progress
  int32_t scene = -1;
  int64_t remaining = 0;
  double admitted = -1.0, finished = -1.0;
  int64_t bytes = 0;
  bool rejected = false;
  bool pinned = false;  // records page-locked with cudaHostRegister
  int64_t box_blocks = 0;       // upper bound on the block box at the grid spacing
  cudaEvent_t done = nullptr;   // the admission's setup, then the result copy, has passed
};

// Upper bound on a scene's block box at spacing dx (4^3-node blocks, halo and
// one block of rounding slack per side included): the step's own measure is
// prod(hi - lo + 4) over the block coordinates of the stencil bases.
int64_t host_box_blocks(const double* rec, int64_t n, double dx) {
  if (n == 0) return 0;
  double lo[3], hi[3];
  for (int a = 0; a < 3; ++a) lo[a] = hi[a] = rec[a];
  for (int64_t i = 0; i < n; ++i)
    for (int a = 0; a < 3; ++a) {
      const double x = rec[26 * i + a];
      if (!std::isfinite(x)) throw Error(SNOW_E_NONFINITE, "request has a non-finite particle position");
      lo[a] = std::min(lo[a], x);
      hi[a] = std::max(hi[a], x);
    }
  int64_t v = 1;
  for (int a = 0; a < 3; ++a) {
    const double bl = std::floor(std::floor(lo[a] / dx) - 1.0) / 4.0, bh = std::floor(std::floor(hi[a] / dx) - 1.0) / 4.0;
    if (!(std::fabs(bl) < 2e9 && std::fabs(bh) < 2e9)) throw Error(SNOW_E_KEYRANGE, "request extent out of range");
    v *= (int64_t)(std::floor(bh) - std::floor(bl)) + 6;
  }
  return v;
}

}  // namespace

class Server {
 public:
  Server(int precision, int64_t budget, int max_scenes, int max_tick_steps)
      : batch_(precision), admit_(precision), retired_(precision), prec_(precision), budget_(budget), max_scenes_(max_scenes),
        max_tick_(max_tick_steps) {}
  ~Server() {
    try {
      batch_.step_complete();
    } catch (...) {
    }
    for (auto& r : reqs_) {
      if (r->pinned) cudaHostUnregister(r->records.data());
      if (r->done) cudaEventDestroy(r->done);
    }
    for (cudaEvent_t e : {ev_base_, ev_start_, ev_end_})
      if (e) cudaEventDestroy(e);
    if (main_s_) cudaStreamDestroy(main_s_);
    if (admit_s_stream_) cudaStreamDestroy(admit_s_stream_);
    if (retire_s_stream_) cudaStreamDestroy(retire_s_stream_);
  }
  Server(const Server&) = delete;
  Server& operator=(const Server&) = delete;

  int64_t submit(const double* rec, int64_t n, const snow_step_params* p, const snow_collider* c, int nc,
                 int64_t steps, double arrival) {
    if (n < 0 || (n > 0 && !rec) || steps < 0 || !p || nc < 0 || (nc > 0 && !c))
      throw Error(SNOW_E_ARG, "bad request");
    if (!(p->grid_spacing > 0.0) || !std::isfinite(p->grid_spacing))
      throw Error(SNOW_E_ARG, "grid_spacing must be positive and finite");
    const int64_t box = host_box_blocks(rec, n, p->grid_spacing);
    auto r = std::make_unique<Request>();
    r->id = (int64_t)reqs_.size();
    r->box_blocks = box;
    r->records.assign(rec, rec + n * 26);
    // page-lock the request's records so uploads and result copies run as
    // direct DMA (without it they go through the batch's staging chunks)
    if (n > 0 && cudaHostRegister(r->records.data(), r->records.size() * sizeof(double), cudaHostRegisterDefault) ==
                     cudaSuccess)
      r->pinned = true;
    else
      cudaGetLastError();
    r->params = *p;
    r->colliders.assign(c, c + nc);
    r->steps = steps;
    r->arrival = arrival;
    r->bytes = footprint(n);
    reqs_.push_back(std::move(r));
    return reqs_.back()->id;
  }

  // Device bytes a scene of n particles holds: two particle buffers, sort
  // buffers, and its share of the grid (about one 4x4x4 block per 32
  // particles, with the grid's 2x headroom).
  int64_t per_particle_bytes() const {
    const int64_t real = prec_ == SNOW_FP64 ? 8 : 4;
    return 2 * (kRealPlanes * real + kFPPlanes * 8 + 4) + 16 + 26 * 8 / 4;
  }
  int64_t footprint(int64_t n) const {
    const int64_t real = prec_ == SNOW_FP64 ? 8 : 4;
    const int64_t grid = 2 * ((n + 31) / 32) * 64 * (kAccCh + kVelCh) * real;
    return n * per_particle_bytes() + grid + (1 << 16);
  }

  // The loop allocates nothing: streams, events and every buffer that scales
  // with the requests are made before it (a cudaMalloc or cudaFree inside it
  // can wait for the tick in flight).  Each pass launches a tick of steps for
  // the live scenes, then, while it runs, issues the setup of newly arrived
  // requests in a second batch on a second stream and the result copies of
  // finished scenes on a third, without waiting for either; after the tick it
  // moves the set-up scenes whose work has passed into the live batch
  // (without copying their particles), finished scenes out of it, and
  // releases scenes whose results have arrived.
  void run(cudaStream_t s) {
    const auto t0 = clock_t_::now();
    auto now = [&] { return std::chrono::duration<double>(clock_t_::now() - t0).count(); };
    if (!s) s = main_stream();
    std::vector<Request*> order;
    for (auto& r : reqs_)
      if (r->finished < 0 && !r->rejected) order.push_back(r.get());
    std::stable_sort(order.begin(), order.end(), [](Request* a, Request* b) { return a->arrival < b->arrival; });
    std::deque<Request*> pending(order.begin(), order.end());
    std::vector<Request*> live, admitting, leaving;
    int64_t used = 0;
    ticks_log_.clear();
    bool base_recorded = false;
    double t_phase = now();
    batch_.set_chunk(work_item_ ? work_item_ : auto_work_item(order));
    reserve(order, s);
    admit_s_ += now() - t_phase;
    while (!pending.empty() || !live.empty() || !admitting.empty() || !leaving.empty()) {
      // launch this tick (the steps run while the host admits and retires below)
      int64_t k = 0;
      t_phase = now();
      snow_server_tick tick{};
      tick.host_start_s = t_phase;
      if (!live.empty()) {
        k = max_tick_;
        for (Request* r : live) {
          k = std::min(k, r->remaining);
          tick.particles += (int64_t)r->records.size() / 26;
        }
        if (!base_recorded) {
          check_cuda(cudaEventRecord(ev_base_, s), "cudaEventRecord");
          base_recorded = true;
        }
        check_cuda(cudaEventRecord(ev_start_, s), "cudaEventRecord");
        batch_.step_launch((int)k, nullptr, s);
        check_cuda(cudaEventRecord(ev_end_, s), "cudaEventRecord");
      }
      step_s_ += now() - t_phase;
      // issue the setup of every arrived request that fits, in arrival order
      t_phase = now();
      while (!pending.empty() && pending.front()->arrival <= now()) {
        Request* r = pending.front();
        if (r->bytes > budget_) {  // can never fit
          r->rejected = true;
          pending.pop_front();
          ++rejected_;
          continue;
        }
        if (used + r->bytes > budget_ || (int)(live.size() + admitting.size()) >= max_scenes_) break;
        pending.pop_front();
        const int64_t n = (int64_t)r->records.size() / 26;
        r->scene = admit_.add_scene(r->records.data(), n, &r->params, r->colliders.data(),
                                    (int)r->colliders.size(), admit_stream(), /*wait=*/!r->pinned);
        admit_.setup(r->scene, r->params.grid_spacing, admit_stream(), r->box_blocks, /*wait=*/false);
        check_cuda(cudaEventRecord(r->done, admit_stream()), "cudaEventRecord");
        r->remaining = r->steps;
        r->admitted = now();
        used += r->bytes;
        admitting.push_back(r);
        peak_scenes_ = std::max<int64_t>(peak_scenes_, (int64_t)(live.size() + admitting.size()));
        peak_bytes_ = std::max(peak_bytes_, used);
      }
      admit_s_ += now() - t_phase;
      // release the scenes whose results have arrived
      t_phase = now();
      collect_results(leaving, used, now, false);
      retire_s_ += now() - t_phase;
      // complete the tick
      if (k > 0) {
        t_phase = now();
        batch_.step_complete();
        step_s_ += now() - t_phase;
        ++ticks_;
        for (Request* r : live) {
          r->remaining -= k;
          particle_steps_ += k * ((int64_t)r->records.size() / 26);
        }
        float a = 0.f, b = 0.f;
        check_cuda(cudaEventSynchronize(ev_end_), "cudaEventSynchronize");
        check_cuda(cudaEventElapsedTime(&a, ev_base_, ev_start_), "cudaEventElapsedTime");
        check_cuda(cudaEventElapsedTime(&b, ev_base_, ev_end_), "cudaEventElapsedTime");
        tick.host_end_s = now();
        tick.device_start_s = a * 1e-3;
        tick.device_end_s = b * 1e-3;
        tick.steps = k;
        tick.scenes = (int64_t)live.size();
      }
      if (live.empty() && !admitting.empty())  // nothing to step: wait for the first setup
        check_cuda(cudaEventSynchronize(admitting.front()->done), "cudaEventSynchronize");
      // set-up scenes join the live batch
      t_phase = now();
      bool joined = false;
      for (size_t i = 0; i < admitting.size();) {
        Request* r = admitting[i];
        const cudaError_t q = cudaEventQuery(r->done);
        if (q == cudaErrorNotReady) {
          ++i;
          continue;
        }
        check_cuda(q, "admission");
        if (!joined) admit_.collect_status();  // flags of every setup that has passed
        joined = true;
        r->scene = batch_.adopt_scene(admit_, r->scene);
        live.push_back(r);
        admitting.erase(admitting.begin() + i);
        ++tick.admitted;
      }
      admit_s_ += now() - t_phase;
      // finished scenes leave the live batch without a copy; their results are
      // copied back on the retire stream while the next tick runs
      t_phase = now();
      for (size_t i = 0; i < live.size();) {
        Request* r = live[i];
        if (r->remaining > 0) {
          ++i;
          continue;
        }
        r->scene = retired_.adopt_scene(batch_, r->scene);
        retired_.download(r->scene, r->records.data(), (int64_t)r->records.size() / 26, retire_stream(),
                          /*wait=*/!r->pinned);
        check_cuda(cudaEventRecord(r->done, retire_stream()), "cudaEventRecord");
        leaving.push_back(r);
        live.erase(live.begin() + i);
        ++tick.retired;
      }
      if (live.empty() && admitting.empty()) {
        // nothing runs: finish the copies back, or wait for the next arrival
        collect_results(leaving, used, now, true);
        if (!pending.empty()) {
          const double wait = pending.front()->arrival - now();
          if (wait > 0) std::this_thread::sleep_for(std::chrono::duration<double>(std::min(wait, 0.01)));
        }
      }
      retire_s_ += now() - t_phase;
      if (k > 0) ticks_log_.push_back(tick);
    }
    wall_ += now();
  }

  const std::vector<snow_server_tick>& ticks() const { return ticks_log_; }

  // 0 = automatic (auto_work_item), else a power of two in [32, 1024].
  void set_work_item(int particles) {
    if (particles != 0 && (particles < 32 || particles > 1024 || (particles & (particles - 1))))
      throw Error(SNOW_E_ARG, "work item size must be 0 or a power of two in [32, 1024]");
    work_item_ = particles;
  }

  const Request& req(int64_t id) const {
    if (id < 0 || id >= (int64_t)reqs_.size()) throw Error(SNOW_E_ARG, "unknown request id");
    return *reqs_[id];
  }

  void stats(snow_server_stats* st) const {
    std::vector<double> lat;
    for (auto& r : reqs_)
      if (r->finished >= 0) lat.push_back(r->finished - r->arrival);
    std::sort(lat.begin(), lat.end());
    auto pct = [&](double q) {
      if (lat.empty()) return 0.0;
      const double pos = q * (lat.size() - 1);
      const size_t i = (size_t)pos;
      const double f = pos - i;
      return i + 1 < lat.size() ? lat[i] * (1 - f) + lat[i + 1] * f : lat[i];
    };
    st->completed = (int64_t)lat.size();
    st->rejected = rejected_;
    st->peak_scenes = peak_scenes_;
    st->peak_bytes = peak_bytes_;
    st->ticks = ticks_;
    st->particle_steps = particle_steps_;
    st->wall_s = wall_;
    st->p50_s = pct(0.50);
    st->p99_s = pct(0.99);
    st->mean_s = lat.empty() ? 0.0 : std::accumulate(lat.begin(), lat.end(), 0.0) / lat.size();
    st->particle_steps_per_s = wall_ > 0 ? particle_steps_ / wall_ : 0.0;
    st->admit_s = admit_s_;
    st->step_s = step_s_;
    st->retire_s = retire_s_;
  }

 private:
  // Releases the finished scenes whose result copies have passed (all of
  // them, waiting, when `wait`); their buffers go back to the admission batch
  // for reuse.
  template <typename Now>
  void collect_results(std::vector<Request*>& leaving, int64_t& used, Now&& now, bool wait) {
    bool any = false;
    for (size_t i = 0; i < leaving.size();) {
      Request* r = leaving[i];
      if (wait) check_cuda(cudaEventSynchronize(r->done), "cudaEventSynchronize");
      const cudaError_t q = cudaEventQuery(r->done);
      if (q == cudaErrorNotReady) {
        ++i;
        continue;
      }
      check_cuda(q, "result copy");
      retired_.remove_scene(r->scene);
      r->finished = now();
      used -= r->bytes;
      leaving.erase(leaving.begin() + i);
      any = true;
    }
    if (any) retired_.give_cache(admit_);
  }

  // Particles per P2G/G2P work item for the live batch, fixed for the run:
  // auto_chunk of all admissible requests' particles (measured on the
  // 48-request stream: 3.29, 3.26, 3.08e9 particle-steps/s at 1024, 512, 256).
  int auto_work_item(const std::vector<Request*>& order) const {
    int64_t live = 0;
    for (Request* r : order)
      if (r->bytes <= budget_) live += (int64_t)r->records.size() / 26;
    return auto_chunk(std::min(live, budget_ / per_particle_bytes()), prec_);
  }

  // Everything the loop needs, made before it: streams, events, and buffers
  // sized for the requests (the live batch's particle buffers, grid and key
  // bins for all admissible requests at once; the admission batch's for the
  // largest; the particle buffers of every request that fits the budget).
  void reserve(const std::vector<Request*>& order, cudaStream_t s) {
    admit_stream();
    retire_stream();
    for (cudaEvent_t* e : {&ev_base_, &ev_start_, &ev_end_})
      if (!*e) check_cuda(cudaEventCreate(e), "cudaEventCreate");
    int64_t live_n = 0, scene_max = 0, box_sum = 0, box_max = 0, grid_max = 0, colliders = 0;
    std::vector<int64_t> sizes;
    for (Request* r : order) {
      if (!r->done) check_cuda(cudaEventCreateWithFlags(&r->done, cudaEventDisableTiming), "cudaEventCreate");
      if (r->bytes > budget_) continue;
      const int64_t n = (int64_t)r->records.size() / 26;
      live_n += n;
      scene_max = std::max(scene_max, n);
      box_sum += r->box_blocks;
      box_max = std::max(box_max, r->box_blocks);
      grid_max = std::max(grid_max, std::min<int64_t>(2 * r->box_blocks + 1024, 8 * n + 1024));
      sizes.push_back(n);
      colliders += (int64_t)r->colliders.size();
    }
    live_n = std::min(live_n, budget_ / per_particle_bytes());
    const int slots = (int)std::min<int64_t>((int64_t)sizes.size(), max_scenes_);
    batch_.reserve(live_n, 0, slots, (int)std::min<int64_t>(colliders, INT32_MAX));
    batch_.reserve_grid(std::min<int64_t>(2 * box_sum + 1024, std::max<int64_t>(8 * live_n + 64, 1024)), box_sum, s);
    admit_.reserve(scene_max, scene_max);
    admit_.reserve_grid(grid_max, box_max, admit_stream());
    admit_.reserve_scenes(sizes, budget_);
    retired_.reserve(0, scene_max);
    check_cuda(cudaStreamSynchronize(s), "reserve");
    check_cuda(cudaStreamSynchronize(admit_stream()), "reserve");
  }

  cudaStream_t main_stream() {
    if (!main_s_) check_cuda(cudaStreamCreateWithFlags(&main_s_, cudaStreamNonBlocking), "cudaStreamCreate");
    return main_s_;
  }
  // Admission and result copies run beside the live batch's tick at the
  // highest stream priority, so their short kernels start at the tick's next
  // kernel boundary instead of after the whole tick.
  static cudaStream_t side_stream() {
    int least = 0, greatest = 0;
    cudaDeviceGetStreamPriorityRange(&least, &greatest);
    cudaStream_t st = nullptr;
    check_cuda(cudaStreamCreateWithPriority(&st, cudaStreamNonBlocking, greatest), "cudaStreamCreate");
    return st;
  }
  cudaStream_t retire_stream() {
    if (!retire_s_stream_) retire_s_stream_ = side_stream();
    return retire_s_stream_;
  }
  cudaStream_t admit_stream() {
    if (!admit_s_stream_) admit_s_stream_ = side_stream();
    return admit_s_stream_;
  }

  Batch batch_;
  Batch admit_;    // new scenes are set up here while batch_ steps
  Batch retired_;  // finished scenes are copied back from here while batch_ steps
  cudaStream_t main_s_ = nullptr, admit_s_stream_ = nullptr, retire_s_stream_ = nullptr;
  cudaEvent_t ev_base_ = nullptr, ev_start_ = nullptr, ev_end_ = nullptr;
  std::vector<snow_server_tick> ticks_log_;
  int prec_;
  int64_t budget_;
  int max_scenes_;
  int64_t max_tick_;
  int work_item_ = 0;
  std::vector<std::unique_ptr<Request>> reqs_;
  int64_t rejected_ = 0, peak_scenes_ = 0, peak_bytes_ = 0, ticks_ = 0, particle_steps_ = 0;
  double wall_ = 0.0, admit_s_ = 0.0, step_s_ = 0.0, retire_s_ = 0.0;
};

}  // namespace snow

struct snow_gpu_server {
  std::unique_ptr<snow::Server> impl;
};

namespace {
template <typename F>
int guarded(F&& f) {
  try {
    f();
    return SNOW_OK;
  } catch (const snow::Error& e) {
    return snow::set_error(e.code, e.what());
  } catch (const std::exception& e) {
    return snow::set_error(SNOW_E_ARG, e.what());
  }
}
}  // namespace

extern "C" {

int snow_gpu_server_create(snow_gpu_server** out, int precision, int64_t hbm_budget_bytes, int max_scenes,
                           int max_steps_per_tick) {
  return guarded([&] {
    if (!out || hbm_budget_bytes <= 0 || max_scenes <= 0 || max_steps_per_tick <= 0)
      throw snow::Error(SNOW_E_ARG, "bad server configuration");
    auto* s = new snow_gpu_server;
    try {
      s->impl = std::make_unique<snow::Server>(precision, hbm_budget_bytes, max_scenes, max_steps_per_tick);
    } catch (...) {
      delete s;
      throw;
    }
    *out = s;
  });
}

int snow_gpu_server_destroy(snow_gpu_server* server) {
  return guarded([&] {
    cudaDeviceSynchronize();
    delete server;
  });
}

int snow_gpu_server_submit(snow_gpu_server* server, const double* records, int64_t n,
                           const snow_step_params* params, const snow_collider* colliders, int n_colliders,
                           int64_t steps, double arrival_s, int64_t* request_id) {
  return guarded([&] {
    if (!server) throw snow::Error(SNOW_E_ARG, "server is NULL");
    const int64_t id = server->impl->submit(records, n, params, colliders, n_colliders, steps, arrival_s);
    if (request_id) *request_id = id;
  });
}

int snow_gpu_server_run(snow_gpu_server* server, void* stream) {
  return guarded([&] {
    if (!server) throw snow::Error(SNOW_E_ARG, "server is NULL");
    server->impl->run(static_cast<cudaStream_t>(stream));
  });
}

int snow_gpu_server_result(snow_gpu_server* server, int64_t request_id, double* records, int64_t n,
                           double* latency_s) {
  return guarded([&] {
    if (!server) throw snow::Error(SNOW_E_ARG, "server is NULL");
    const auto& r = server->impl->req(request_id);
    if (r.rejected) throw snow::Error(SNOW_E_CAPACITY, "request was rejected: larger than the memory budget");
    if (r.finished < 0) throw snow::Error(SNOW_E_STATE, "request has not completed");
    if (n != (int64_t)r.records.size() / 26) throw snow::Error(SNOW_E_ARG, "particle count differs");
    std::copy(r.records.begin(), r.records.end(), records);
    if (latency_s) *latency_s = r.finished - r.arrival;
  });
}

int snow_gpu_server_stats(snow_gpu_server* server, snow_server_stats* stats) {
  return guarded([&] {
    if (!server || !stats) throw snow::Error(SNOW_E_ARG, "NULL argument");
    server->impl->stats(stats);
  });
}

int snow_gpu_server_set_work_item(snow_gpu_server* server, int particles) {
  return guarded([&] {
    if (!server) throw snow::Error(SNOW_E_ARG, "server is NULL");
    server->impl->set_work_item(particles);
  });
}

int snow_gpu_server_ticks(snow_gpu_server* server, snow_server_tick* out, int64_t capacity, int64_t* count) {
  return guarded([&] {
    if (!server || !count || capacity < 0 || (capacity > 0 && !out)) throw snow::Error(SNOW_E_ARG, "bad argument");
    const auto& t = server->impl->ticks();
    *count = (int64_t)t.size();
    std::copy_n(t.begin(), std::min<int64_t>(capacity, (int64_t)t.size()), out);
  });
}

}  // extern "C"
