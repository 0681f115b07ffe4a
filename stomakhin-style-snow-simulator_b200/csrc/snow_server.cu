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
//
// Requests may be submitted from any thread, also while run() loops.  In
// streaming mode run() keeps serving (waiting for submissions when idle) until
// close() is called and every request is done; otherwise it returns once the
// requests submitted so far are done.  Device buffers are reserved before the
// loop for the requests already queued, and grown, with headroom and between
// ticks, only when a request submitted later does not fit what is reserved.
#include <algorithm>
#include <atomic>
#include <chrono>
#include <cmath>
#include <condition_variable>
#include <deque>
#include <memory>
#include <mutex>
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
  double admitted = -1.0;
  std::atomic<double> finished{-1.0};  // set by the loop once the result is in `records`
  int64_t bytes = 0;
  std::atomic<bool> rejected{false};
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
    // Copies into the requests' page-locked records may still be in flight
    // when run() left by an exception: let them finish before the records are
    // unregistered and the streams destroyed.
    for (cudaStream_t st : {admit_s_stream_, retire_s_stream_, main_s_})
      if (st) cudaStreamSynchronize(st);
    cudaGetLastError();
    for (auto& r : reqs_) {
      if (r->pinned) cudaHostUnregister(r->records.data());
      if (r->done) cudaEventDestroy(r->done);
    }
    if (ev_base_) cudaEventDestroy(ev_base_);
    for (int k = 0; k < kTickEvents; ++k)
      for (cudaEvent_t e : {ev_start_[k], ev_end_[k]})
        if (e) cudaEventDestroy(e);
    if (main_s_) cudaStreamDestroy(main_s_);
    if (admit_s_stream_) cudaStreamDestroy(admit_s_stream_);
    if (retire_s_stream_) cudaStreamDestroy(retire_s_stream_);
  }
  Server(const Server&) = delete;
  Server& operator=(const Server&) = delete;

  // Thread-safe; may be called while run() loops.  arrival < 0 stamps the
  // request with the current time on the server clock (0 before run()).
  int64_t submit(const double* rec, int64_t n, const snow_step_params* p, const snow_collider* c, int nc,
                 int64_t steps, double arrival) {
    if (n < 0 || (n > 0 && !rec) || steps < 0 || !p || nc < 0 || (nc > 0 && !c))
      throw Error(SNOW_E_ARG, "bad request");
    if (!(p->grid_spacing > 0.0) || !std::isfinite(p->grid_spacing))
      throw Error(SNOW_E_ARG, "grid_spacing must be positive and finite");
    if (!std::isfinite(arrival)) throw Error(SNOW_E_ARG, "arrival time must be finite");
    device_colliders(c, nc);  // reject bad colliders at submission, not inside the loop
    const int64_t box = host_box_blocks(rec, n, p->grid_spacing);
    auto r = std::make_unique<Request>();
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
    r->bytes = footprint(n);
    check_cuda(cudaEventCreateWithFlags(&r->done, cudaEventDisableTiming), "cudaEventCreate");
    std::lock_guard<std::mutex> lk(mu_);
    if (closed_) {
      if (r->pinned) cudaHostUnregister(r->records.data());
      cudaEventDestroy(r->done);
      throw Error(SNOW_E_STATE, "the server is closed to new requests");
    }
    r->arrival = arrival >= 0.0 ? arrival : (running_ ? seconds_since(t0_) : 0.0);
    r->id = (int64_t)reqs_.size();
    incoming_.push_back(r.get());
    reqs_.push_back(std::move(r));
    cv_.notify_all();
    return reqs_.back()->id;
  }

  // Streaming mode: run() waits for further submissions when it has nothing
  // to do, until close().
  void set_streaming(bool on) {
    std::lock_guard<std::mutex> lk(mu_);
    streaming_ = on;
    cv_.notify_all();
  }
  // No more submissions: run() returns once every queued request is done.
  void close() {
    std::lock_guard<std::mutex> lk(mu_);
    closed_ = true;
    cv_.notify_all();
  }
  int64_t reservations() const { return reservations_; }

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

  // The loop allocates nothing for the requests queued when it starts:
  // streams, events and every buffer that scales with them are made before it
  // (a cudaMalloc or cudaFree inside it can wait for the tick in flight).
  // Requests submitted while it runs are reserved for between ticks
  // (grow_for), in doublings, and their particle buffers allocated while a
  // tick runs (carve_for).  Each pass leaves the tick launched by the last
  // pass in flight, moves the scenes that finish with it out of the live batch
  // (their result copies queued on a third stream behind it) and the set-up
  // scenes whose work has passed into it (without copying their particles),
  // and queues the next tick behind the ones in flight on the same stream;
  // then, while the ticks run, it issues the setup of newly arrived requests
  // in a second batch on a second stream, releases scenes whose results have
  // arrived, and last waits for the oldest tick beyond kQueuedTicks.  The
  // device thus finds ticks queued when one ends, also while a pass of host
  // work takes longer than a tick.
  void run(cudaStream_t s) {
    std::vector<Request*> order;
    {
      std::lock_guard<std::mutex> lk(mu_);
      if (running_) throw Error(SNOW_E_STATE, "run() is already running");
      running_ = true;
      t0_ = clock_t_::now();
      order.swap(incoming_);
    }
    struct Stop {  // run() may leave by an exception: the server stays usable
      Server* sv;
      ~Stop() {
        std::lock_guard<std::mutex> lk(sv->mu_);
        sv->running_ = false;
      }
    } stop{this};
    const auto t0 = t0_;
    auto now = [&] { return std::chrono::duration<double>(clock_t_::now() - t0).count(); };
    if (!s) s = main_stream();
    std::stable_sort(order.begin(), order.end(), [](Request* a, Request* b) { return a->arrival < b->arrival; });
    std::deque<Request*> pending(order.begin(), order.end());
    std::vector<Request*> live, admitting, leaving, carve;
    // ticks in flight, oldest first: up to kQueuedTicks are queued on the
    // device ahead of the host, so that a pass of host work longer than one
    // tick does not leave the device idle
    struct Flight {
      bool on = false;
      int64_t k = 0;
      int ev = 0;  // its pair of ev_start_ / ev_end_
      snow_server_tick tick{};
    };
    std::deque<Flight> flights;
    int ev_next = 0;
    int64_t used = 0;
    ticks_log_.clear();
    bool base_recorded = false;
    double t_phase = now();
    batch_.set_chunk(work_item_ ? work_item_ : auto_work_item(order));
    batch_.set_host_sized(true);
    // buffers that a reservation replaces while ticks, setups or result copies
    // are in flight stay allocated until the loop is idle (a cudaFree would
    // wait for the whole device)
    struct Released {
      Server* sv;
      void flush() {
        for (Batch* b : {&sv->batch_, &sv->admit_, &sv->retired_}) b->flush_released();
      }
      ~Released() {
        flush();
        for (Batch* b : {&sv->batch_, &sv->admit_, &sv->retired_}) b->set_deferred_free(false);
      }
    } released{this};
    for (Batch* b : {&batch_, &admit_, &retired_}) b->set_deferred_free(true);
    reserve(order, s);
    admit_s_ += now() - t_phase;
    for (;;) {
      // The tick launched by the last pass stays in flight while this pass
      // reserves for new requests, moves scenes in and out and queues the next
      // tick behind it on the same stream; only then does the host wait, for
      // the oldest tick beyond the kQueuedTicks it keeps queued, so the device
      // runs tick after tick without a gap for the host's work.
      batch_.step_detach();
      // requests submitted since the last pass join the queue in arrival order
      std::vector<Request*> fresh;
      bool more_may_come;
      {
        std::lock_guard<std::mutex> lk(mu_);
        fresh.swap(incoming_);
        more_may_come = streaming_ && !closed_;
      }
      if (!fresh.empty()) {
        t_phase = now();
        grow_for(fresh, live, admitting, s);
        carve.insert(carve.end(), fresh.begin(), fresh.end());
        std::stable_sort(fresh.begin(), fresh.end(), [](Request* a, Request* b) { return a->arrival < b->arrival; });
        std::deque<Request*> merged;
        std::merge(pending.begin(), pending.end(), fresh.begin(), fresh.end(), std::back_inserter(merged),
                   [](Request* a, Request* b) { return a->arrival < b->arrival; });
        pending.swap(merged);
        admit_s_ += now() - t_phase;
      }
      if (pending.empty() && live.empty() && admitting.empty() && leaving.empty() && flights.empty()) {
        if (!more_may_come) break;
        released.flush();  // idle: nothing in flight reads the replaced buffers
        std::unique_lock<std::mutex> lk(mu_);
        cv_.wait_for(lk, std::chrono::milliseconds(5),
                     [&] { return !incoming_.empty() || closed_ || !streaming_; });
        continue;
      }
      // scenes that finish with the tick in flight leave the live batch now
      // (without a copy); their results are copied back on the retire stream
      // once that tick has passed, while the next one runs
      t_phase = now();
      int64_t admitted_now = 0;
      for (size_t i = 0; i < live.size();) {
        Request* r = live[i];
        if (r->remaining > 0) {
          ++i;
          continue;
        }
        r->scene = retired_.adopt_scene(batch_, r->scene);
        // their last tick is the newest in flight
        if (!flights.empty())
          check_cuda(cudaStreamWaitEvent(retire_stream(), ev_end_[flights.back().ev], 0), "cudaStreamWaitEvent");
        retired_.download(r->scene, r->records.data(), (int64_t)r->records.size() / 26, retire_stream(),
                          /*wait=*/!r->pinned);
        check_cuda(cudaEventRecord(r->done, retire_stream()), "cudaEventRecord");
        leaving.push_back(r);
        live.erase(live.begin() + i);
      }
      retire_s_ += now() - t_phase;
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
        ++admitted_now;
      }
      admit_s_ += now() - t_phase;
      // launch the next tick (it runs while the host admits and retires below)
      Flight next;
      t_phase = now();
      int64_t k = max_tick_;
      for (Request* r : live) k = std::min(k, r->remaining);
      if (!live.empty() && k > 0) {
        next.on = true;
        next.k = k;
        next.ev = ev_next;
        ev_next = (ev_next + 1) % kTickEvents;
        next.tick.host_start_s = t_phase;
        next.tick.steps = k;
        next.tick.scenes = (int64_t)live.size();
        next.tick.admitted = admitted_now;
        for (Request* r : live) next.tick.particles += (int64_t)r->records.size() / 26;
        if (!base_recorded) {
          check_cuda(cudaEventRecord(ev_base_, s), "cudaEventRecord");
          base_recorded = true;
        }
        check_cuda(cudaEventRecord(ev_start_[next.ev], s), "cudaEventRecord");
        batch_.step_launch((int)k, nullptr, s);
        check_cuda(cudaEventRecord(ev_end_[next.ev], s), "cudaEventRecord");
        for (Request* r : live) {
          r->remaining -= k;
          next.tick.retired += r->remaining == 0;  // these finish with this tick
        }
      }
      step_s_ += now() - t_phase;
      // particle buffers for the requests that arrived since the last pass,
      // allocated while the ticks run
      t_phase = now();
      if (!carve.empty()) {
        carve_for(carve);
        carve.clear();
      }
      // issue the setup of every arrived request that fits, in arrival order
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
      // complete the oldest ticks, keeping kQueuedTicks queued behind them
      // (all of them when this pass queued none: nothing is left to run)
      if (next.on) flights.push_back(next);
      while (flights.size() > (next.on ? (size_t)kQueuedTicks : 0)) {
        Flight& f = flights.front();
        t_phase = now();
        batch_.complete_detached();
        check_cuda(cudaEventSynchronize(ev_end_[f.ev]), "cudaEventSynchronize");
        float a = 0.f, b = 0.f;
        check_cuda(cudaEventElapsedTime(&a, ev_base_, ev_start_[f.ev]), "cudaEventElapsedTime");
        check_cuda(cudaEventElapsedTime(&b, ev_base_, ev_end_[f.ev]), "cudaEventElapsedTime");
        f.tick.host_end_s = now();
        f.tick.device_start_s = a * 1e-3;
        f.tick.device_end_s = b * 1e-3;
        ++ticks_;
        particle_steps_ += f.k * f.tick.particles;
        ticks_log_.push_back(f.tick);
        step_s_ += now() - t_phase;
        flights.pop_front();
      }
      if (flights.empty() && live.empty() && !admitting.empty())  // nothing to step: wait for the first setup
        check_cuda(cudaEventSynchronize(admitting.front()->done), "cudaEventSynchronize");
      if (flights.empty() && live.empty() && admitting.empty()) {
        // nothing runs: finish the copies back, or wait for the next arrival
        t_phase = now();
        collect_results(leaving, used, now, true);
        if (!pending.empty()) {
          const double wait = pending.front()->arrival - now();
          if (wait > 0) std::this_thread::sleep_for(std::chrono::duration<double>(std::min(wait, 0.01)));
        }
        retire_s_ += now() - t_phase;
      }
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

  // The request's result, once run() has completed it (thread-safe).
  void result(int64_t id, double* records, int64_t n, double* latency_s) {
    Request* r = nullptr;
    {
      std::lock_guard<std::mutex> lk(mu_);
      if (id < 0 || id >= (int64_t)reqs_.size()) throw Error(SNOW_E_ARG, "unknown request id");
      r = reqs_[id].get();
    }
    if (r->rejected) throw Error(SNOW_E_CAPACITY, "request was rejected: larger than the memory budget");
    const double fin = r->finished.load();
    if (fin < 0) throw Error(SNOW_E_STATE, "request has not completed");
    if (n != (int64_t)r->records.size() / 26) throw Error(SNOW_E_ARG, "particle count differs");
    std::copy(r->records.begin(), r->records.end(), records);
    if (latency_s) *latency_s = fin - r->arrival;
  }

  void stats(snow_server_stats* st) {
    std::lock_guard<std::mutex> lk(mu_);
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
    st->reservations = reservations_;
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

  // What a set of requests needs reserved at once.
  struct Need {
    int64_t live_n = 0, scene_max = 0, box_sum = 0, box_max = 0, grid_max = 0, colliders = 0, slots = 0;
    std::vector<int64_t> sizes;
    void add(const Request& r) {
      const int64_t n = (int64_t)r.records.size() / 26;
      live_n += n;
      scene_max = std::max(scene_max, n);
      box_sum += r.box_blocks;
      box_max = std::max(box_max, r.box_blocks);
      grid_max = std::max(grid_max, std::min<int64_t>(2 * r.box_blocks + 1024, 8 * n + 1024));
      colliders += (int64_t)r.colliders.size();
      ++slots;
      sizes.push_back(n);
    }
  };

  // Reserves `need` (capped by the budget and the scene slots) in the live,
  // admission and retirement batches.  A tick may be in flight (detached from
  // the live batch): it keeps the buffers it was launched with.
  void reserve_need(const Need& need, cudaStream_t s, bool carve_scenes) {
    const int64_t live_n = std::min(need.live_n, budget_ / per_particle_bytes());
    const int slots = (int)std::min<int64_t>(need.slots, max_scenes_);
    batch_.reserve(live_n, 0, slots, (int)std::min<int64_t>(need.colliders, INT32_MAX));
    batch_.reserve_grid(std::min<int64_t>(2 * need.box_sum + 1024, std::max<int64_t>(8 * live_n + 64, 1024)),
                        need.box_sum, s);
    admit_.reserve(need.scene_max, need.scene_max);
    admit_.reserve_grid(need.grid_max, need.box_max, admit_stream());
    if (carve_scenes) admit_.reserve_scenes(need.sizes, budget_);
    retired_.reserve(0, need.scene_max);
    // no wait: the clears above are ordered on the streams that use the new
    // buffers, and the replaced ones stay allocated (deferred frees) while
    // the ticks, setups and copies in flight still read them
    reserved_ = need;
    ++reservations_;
  }

  // Everything the loop needs, made before it: streams, events, and buffers
  // sized for the requests (the live batch's particle buffers, grid and key
  // bins for all admissible requests at once; the admission batch's for the
  // largest; the particle buffers of every request that fits the budget).
  void reserve(const std::vector<Request*>& order, cudaStream_t s) {
    admit_stream();
    retire_stream();
    if (!ev_base_) check_cuda(cudaEventCreate(&ev_base_), "cudaEventCreate");
    for (int k = 0; k < kTickEvents; ++k)
      for (cudaEvent_t* e : {&ev_start_[k], &ev_end_[k]})
        if (!*e) check_cuda(cudaEventCreate(e), "cudaEventCreate");
    Need need;
    for (Request* r : order)
      if (r->bytes <= budget_) need.add(*r);
    reserve_need(need, s, true);
  }

  // Requests submitted while the loop runs: when the scenes that may be live
  // together with them (the live and admitting ones, the queue and these) need
  // more than is reserved, reserve twice that need, so that a stream of
  // requests causes a logarithmic number of reservations.  Runs between
  // ticks; the batches grow by themselves in any case, this only moves the
  // allocations out of the ticks and batches them.
  void grow_for(const std::vector<Request*>& fresh, const std::vector<Request*>& live,
                const std::vector<Request*>& admitting, cudaStream_t s) {
    Need need;
    for (const auto* group : {&live, &admitting})
      for (Request* r : *group) need.add(*r);
    for (Request* r : fresh)
      if (r->bytes <= budget_) need.add(*r);
    const Need& have = reserved_;
    if (need.live_n <= have.live_n && need.scene_max <= have.scene_max && need.box_sum <= have.box_sum &&
        need.grid_max <= have.grid_max && need.colliders <= have.colliders && need.slots <= have.slots)
      return;
    Need twice = need;
    twice.live_n = 2 * std::max(need.live_n, have.live_n);
    twice.box_sum = 2 * std::max(need.box_sum, have.box_sum);
    twice.colliders = 2 * std::max(need.colliders, have.colliders);
    twice.slots = 2 * std::max(need.slots, have.slots);
    twice.scene_max = std::max(need.scene_max, have.scene_max);
    twice.box_max = std::max(need.box_max, have.box_max);
    twice.grid_max = std::max(need.grid_max, have.grid_max);
    reserve_need(twice, s, false);
  }

  // Particle buffers for fresh requests, carved from one allocation: admitting
  // them then allocates nothing, and the buffers of finished scenes stay
  // cached for later ones instead of being freed (a cudaFree inside the loop
  // waits for the tick in flight).  The allocation issues no stream work, so
  // the loop makes it while a tick runs.
  void carve_for(const std::vector<Request*>& fresh) {
    std::vector<int64_t> sizes;
    for (Request* r : fresh)
      if (r->bytes <= budget_) sizes.push_back((int64_t)r->records.size() / 26);
    admit_.reserve_scenes(sizes, budget_);
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
  // ticks queued on the device ahead of the host (the engine keeps up to three
  // launches in flight), and the event pairs of the ticks in flight
  static constexpr int kQueuedTicks = 2;
  static constexpr int kTickEvents = kQueuedTicks + 2;
  cudaEvent_t ev_base_ = nullptr, ev_start_[kTickEvents] = {}, ev_end_[kTickEvents] = {};
  std::vector<snow_server_tick> ticks_log_;
  int prec_;
  int64_t budget_;
  int max_scenes_;
  int64_t max_tick_;
  int work_item_ = 0;
  // Submissions (any thread) and the loop share these under mu_.
  std::mutex mu_;
  std::condition_variable cv_;
  std::deque<std::unique_ptr<Request>> reqs_;  // every request, by id (stable addresses)
  std::vector<Request*> incoming_;             // submitted, not yet taken by run()
  bool streaming_ = false, closed_ = false, running_ = false;
  clock_t_::time_point t0_ = clock_t_::now();  // the server clock starts with run()
  static double seconds_since(clock_t_::time_point t) {
    return std::chrono::duration<double>(clock_t_::now() - t).count();
  }
  Need reserved_;
  int64_t reservations_ = 0;
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
    if (n > 0 && !records) throw snow::Error(SNOW_E_ARG, "records is NULL");
    server->impl->result(request_id, records, n, latency_s);
  });
}

int snow_gpu_server_set_streaming(snow_gpu_server* server, int on) {
  return guarded([&] {
    if (!server) throw snow::Error(SNOW_E_ARG, "server is NULL");
    server->impl->set_streaming(on != 0);
  });
}

int snow_gpu_server_close(snow_gpu_server* server) {
  return guarded([&] {
    if (!server) throw snow::Error(SNOW_E_ARG, "server is NULL");
    server->impl->close();
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
