// Host-side batch engine (C++ view of include/snow_gpu.h).
#pragma once

#include <cuda_runtime.h>

#include <algorithm>
#include <deque>
#include <memory>
#include <stdexcept>
#include <string>
#include <vector>

#include "snow_batch.cuh"
#include "snow_gpu.h"

namespace snow {

struct Error : std::runtime_error {
  int code;
  Error(int c, const std::string& m) : std::runtime_error(m), code(c) {}
};

int set_error(int code, const std::string& msg);

// Particles per P2G/G2P work item for `particles` in a batch of `precision`:
// the largest power of two in [256, 1024] that still leaves about four items
// per resident CTA of the particle kernels (2 per SM in FP64, 3 in the mixed
// form).  Larger items stage a grid block's node tile fewer times; too few
// items leave SMs idle at the end of each pass.  Measured on one B200: a 4M
// particle sphere steps 10% faster at 1024 than at 256 (FP64 1.63 vs 1.82 ms,
// mixed 0.89 vs 0.98 ms); two tori of 650k particles step fastest at 512 in
// FP64 (0.3154 vs 0.3196 ms at 256) and at 256-512 in the mixed form, and
// 13% slower at 1024.
int auto_chunk(int64_t particles, int precision);
void check_cuda(cudaError_t e, const char* what);

// Checks a caller's collider array (kinds, finite positive sphere radius, box
// axes unit and orthogonal, box half extents finite and positive) and returns
// it as device records; throws Error(SNOW_E_ARG) on the first bad entry.
std::vector<Collider> device_colliders(const snow_collider* c, int n);

// One scene: its particle planes (two buffers), parameters and colliders.
struct Scene {
  int32_t sid = 0;  // handle returned to the caller
  int64_t n = 0;
  int64_t stride = 0;
  int cur = 0;
  void* r[2] = {nullptr, nullptr};
  double* fp[2] = {nullptr, nullptr};
  int32_t* id[2] = {nullptr, nullptr};
  snow_step_params params{};
  std::vector<Collider> colliders;
  unsigned char* snap = nullptr;  // snapshot of the particle state (snapshot())
  // Set when r/fp/id are carved from one shared allocation (reserve_scenes),
  // which is freed when its last piece is dropped; else each is its own.
  std::shared_ptr<void> slab;
};

class Batch {
 public:
  explicit Batch(int precision);
  ~Batch();
  Batch(const Batch&) = delete;
  Batch& operator=(const Batch&) = delete;

  // wait = false (page-locked records only): the copies are left in flight on
  // stream s; the caller keeps `records` untouched, and the scene in this
  // batch, until s has passed them.
  int32_t add_scene(const double* records, int64_t n, const snow_step_params* params,
                    const snow_collider* colliders, int n_colliders, cudaStream_t s, bool wait = true);
  void remove_scene(int32_t id);
  void set_params(int32_t id, const snow_step_params* params, const snow_collider* c, int n);
  // keep_order: slot j of the scene takes record id[j], the order its last
  // step left (block-sorted), instead of record j; only valid while the
  // scene's id plane is a permutation of [0, n), i.e. after a step or upload
  // that completed without an error.
  void upload(int32_t id, const double* records, int64_t n, cudaStream_t s, bool wait = true,
              bool keep_order = false);
  void download(int32_t id, double* records, int64_t n, cudaStream_t s, bool wait = true);
  void download_positions(int32_t id, double* xyz, int64_t n, cudaStream_t s);
  // box_blocks >= 0: an upper bound on the scene's block box at dx (in 4^3
  // blocks, halo included) known to the caller, which sizes the grid without
  // reading the box back.  wait = false: the setup is left in flight on s and
  // its status is read by collect_status() once s has passed it.
  void setup(int32_t id, double dx, cudaStream_t s, int64_t box_blocks = -1, bool wait = true);
  void collect_status();
  // Grid blocks and key blocks to size the grid and the dense bins for now.
  void reserve_grid(int64_t blocks, int64_t key_blocks, cudaStream_t s);
  // Allocates particle buffers for scenes of these sizes into the cache of
  // removed scenes' buffers, up to `max_bytes`, carved from one allocation.
  void reserve_scenes(const std::vector<int64_t>& sizes, int64_t max_bytes);
  void step(int n_steps, snow_step_timings* timings, cudaStream_t s);
  void step_launch(int n_steps, snow_step_timings* timings, cudaStream_t s);
  void step_complete();
  // Leaves the launched steps in flight without waiting for them, so that
  // scenes can join and leave and the next steps be launched behind them on
  // the same stream (each launch's status goes to its own counter slot);
  // complete_detached() waits for the oldest launch left in flight and checks
  // its status.  At most kCtrSlots - 1 launches are left behind: detaching
  // another first completes the oldest.
  void step_detach();
  void complete_detached();
  // Deferred frees: buffers that growth replaces are kept until
  // flush_released() instead of freed at once (a cudaFree waits for the whole
  // device, launches left in flight included, which may still read them).
  void set_deferred_free(bool on) { defer_free_ = on; }
  void flush_released();
  int32_t adopt_scene(Batch& from, int32_t id);
  // Sizes the particle-indexed step buffers for `particles` in total, the
  // host-transfer staging for scenes of up to `staging` particles and the
  // device scene and collider tables, so that membership changes within those
  // sizes allocate and free nothing (a cudaFree waits for the whole device).
  void reserve(int64_t particles, int64_t staging, int scenes = 0, int colliders = 0);
  // Hands the cached buffers of removed scenes to another batch.
  void give_cache(Batch& to) {
    for (auto& c : cache_) to.cache_.push_back(c);
    to.cached_bytes_ += cached_bytes_;
    to.cache_limit_ = std::max(to.cache_limit_, cache_limit_);
    cache_.clear();
    cached_bytes_ = 0;
  }
  // A device copy of a scene's particle state, and putting it back (the
  // scene then continues from there).  One snapshot per scene.
  void snapshot(int32_t id, cudaStream_t s);
  void restore(int32_t id, cudaStream_t s);
  int autotune(int trial_steps, double* best_ms, cudaStream_t s);

  int scene_count() const { return (int)scenes_.size(); }
  int64_t particles() const {
    int64_t t = 0;
    for (auto& s : scenes_) t += s->n;
    return t;
  }
  int32_t first_id() const { return scenes_.empty() ? -1 : scenes_.front()->sid; }
  void clear() {
    while (!scenes_.empty()) remove_scene(scenes_.back()->sid);
  }
  uint32_t last_status() const { return last_status_; }
  int64_t last_blocks() const { return last_blocks_; }
  int64_t last_fp64_projections() const { return prec_ == SNOW_MIXED ? (int64_t)h_ctr_->last_fp64 : 0; }
  int64_t capacity_blocks() const { return cap_blocks_; }
  // Particles per P2G/G2P work item (a power of two, 32..1024).  Until set
  // (here or by autotune) it follows the batch's particle count: auto_chunk.
  // Host-sized batches (the server's live batch): the caller reserves the grid
  // and the key bins for the scenes it adds (reserve_grid), so a change of
  // scenes alone does not read the measured boxes back to size them; growth
  // past the reservation's headroom (step_complete) still does.
  void set_host_sized(bool on) { host_sized_ = on; }
  void set_chunk(int chunk) {
    if (chunk < 32 || chunk > 1024 || (chunk & (chunk - 1))) throw Error(SNOW_E_ARG, "chunk must be a power of two in [32, 1024]");
    chunk_ = chunk;
    chunk_auto_ = false;
    cap_items_ = 0;  // re-sized on the next prepare
    boxes_dirty_ = true;
  }
  int chunk() const { return chunk_; }
  void set_graphs(bool on) {
    use_graphs_ = on;
    drop_graph();
  }
  // Counting sort over dense key bins (default) or the radix sort with the
  // block hash table; the latter is also taken when the key boxes would need
  // more than kMaxDenseBins bins.
  void set_dense(bool on) {
    want_dense_ = on;
    boxes_dirty_ = true;
  }
  bool dense() const { return dense_; }
  // Kernel launches in one replay of the captured step graph (0 before capture).
  int graph_kernels() const { return graph_kernels_; }
  // Semi-implicit velocity update (snow_implicit.cu): beta = 0 is the explicit
  // step; beta > 0 solves (I + beta dt^2 M^-1 H) v = v* by conjugate residuals
  // to the relative `tolerance` or `max_iterations`.  Steps then run eagerly.
  void set_implicit(double beta, double tolerance, int max_iterations) {
    if (!(beta >= 0.0 && beta <= 1.0) || !(tolerance > 0.0) || max_iterations < 1)
      throw Error(SNOW_E_ARG, "implicit update: beta in [0, 1], tolerance > 0, max_iterations >= 1");
    imp_beta_ = beta;
    imp_tol2_ = tolerance * tolerance;
    imp_max_iter_ = max_iterations;
    drop_graph();
  }
  void implicit_stats(int* iterations, double* residual) const {
    if (iterations) *iterations = last_imp_iters_;
    if (residual) *residual = last_imp_res_;
  }
  // Buffers of the solve for the current grid and particles, and the solve
  // itself on the velocities in vel[0..2] (the grid update's output, or
  // velocities loaded there); apply_only: vel[0..2] <- A vel[0..2] instead.
  void ensure_implicit();
  void free_implicit();
  template <typename R>
  void implicit_solve(const BatchDev& b, cudaStream_t s, bool apply_only = false);
  static constexpr int64_t kMaxDenseBins = int64_t(1) << 26;
  int64_t device_bytes() const;
  int precision() const { return prec_; }
  Scene* find(int32_t id);

  // Buffers for the single-stage entry points.
  BatchDev dev(SceneDev* scenes, int num_scenes, int64_t total) const;
  SceneDev* device_scenes() const { return d_scenes_; }
  int device_scene_count() const { return num_dev_scenes_; }
  void prepare(cudaStream_t s);
  int64_t total() const { return total_; }
  void check_status();
  Counters* host_counters() { return h_ctr_; }
  Counters* device_counters() { return d_ctr_; }
  void set_last_status(uint32_t st) { last_status_ = st; }

 private:
  void free_scene(Scene& s);
  void free_particle_buffers();
  void free_grid();
  void drop_graph();
  void ensure_staging(int64_t n);
  void ensure_pinned();
  void copy_in(void* dst, const void* src, size_t bytes, cudaStream_t s, bool wait);
  void copy_out(void* dst, const void* src, size_t bytes, cudaStream_t s, bool wait);
  int64_t scene_bytes(int64_t stride) const {
    return 2 * stride * (kRealPlanes * (int64_t)rsize_ + kFPPlanes * 8 + 4);
  }
  void ensure_particle_buffers(int64_t total);
  void ensure_grid(int64_t blocks);
  void ensure_items();
  void ensure_bins(int64_t bins);
  void free_bins();
  void size_dense(int64_t key_blocks, cudaStream_t s);
  void set_colliders(Scene& sc, const snow_collider* c, int n);
  SceneDev scene_dev(const Scene& sc, int64_t begin) const;
  template <typename R>
  void launch_step(const BatchDev& b, cudaStream_t s, cudaEvent_t* ev);

  int prec_;
  size_t rsize_;
  std::vector<std::unique_ptr<Scene>> scenes_;
  int32_t next_id_ = 0;
  bool dirty_ = true, boxes_dirty_ = true, params_dirty_ = false;
  bool use_graphs_ = true;
  bool force_dirty_ = true;  // particles' force matrices must be recomputed
  bool keyspace_ready_ = false;  // the device holds the next step's key boxes
  bool pending_ = false;  // steps launched, status not read yet
  cudaStream_t pending_stream_ = nullptr;
  // launches left in flight by step_detach(), oldest first: the event after
  // each and its counter slot
  struct Detached {
    cudaEvent_t ev;
    Counters* ctr;
  };
  std::deque<Detached> detached_;
  std::vector<cudaEvent_t> det_events_;  // events of completed ones, for reuse
  static constexpr int kCtrSlots = 4;
  void absorb(const Counters& c);
  bool defer_free_ = false;
  std::vector<void*> released_;
  void release_ptr(void* p);
  template <typename T>
  void release(T*& p) {
    release_ptr((void*)p);
    p = nullptr;
  }
  // Page-locked staging of the scene and collider tables prepare() uploads,
  // kStageBufs per table used in turn, each reused only once its last copy
  // passed: uploads queued behind detached launches read theirs while the
  // next prepare() writes another.
  static constexpr int kStageBufs = 4;
  struct HostStage {
    void* p[kStageBufs] = {};
    size_t cap[kStageBufs] = {};
    cudaEvent_t ev[kStageBufs] = {};
    int next = 0;
  };
  HostStage stage_[2];
  void staged_upload(HostStage& st, void* dst, const void* src, size_t bytes, cudaStream_t s, const char* what);
  int64_t total_ = 0;
  int num_dev_scenes_ = 0;

  SceneDev* d_scenes_ = nullptr;
  int d_scenes_cap_ = 0;
  SceneDev* d_tmp_scene_ = nullptr;
  Collider* d_coll_ = nullptr;
  int d_coll_cap_ = 0;
  Counters* d_ctr_ = nullptr;
  Counters* h_ctr_ = nullptr;      // the slot the next launch's counters go to
  Counters* h_ctr_buf_ = nullptr;  // kCtrSlots page-locked slots

  uint32_t* keys_[2] = {nullptr, nullptr};
  uint32_t* vals_[2] = {nullptr, nullptr};
  uint32_t* hist_ = nullptr;
  int4* fixups_ = nullptr;
  uint32_t* digit_total_ = nullptr;
  uint32_t* bins_ = nullptr;
  uint32_t* bin_off_ = nullptr;
  uint8_t* occ_ = nullptr;
  int32_t* idmap_ = nullptr;
  unsigned long long* bin_state_ = nullptr;
  int64_t cap_bins_ = 0;
  bool want_dense_ = true, dense_ = false, bins_dirty_ = false;
  int64_t last_key_blocks_ = 0;
  int graph_kernels_ = 0;
  int64_t cap_p_ = 0;
  int ntiles_cap_ = 0;

  unsigned long long* htab_ = nullptr;
  uint32_t hcap_ = 0;
  int32_t cap_blocks_ = 0;
  int4* blk_ = nullptr;
  void* acc_ = nullptr;
  void* vel_ = nullptr;
  BlockHeader* item_hdr_ = nullptr;
  int32_t cap_items_ = 0;
  int32_t chunk_ = 256;
  bool chunk_auto_ = true;
  bool host_sized_ = false;

  double* staging_ = nullptr;
  int64_t staging_cap_ = 0;
  static constexpr size_t kXferChunk = size_t(16) << 20;
  unsigned char* pinned_[2] = {nullptr, nullptr};
  cudaEvent_t pinned_ev_[2] = {nullptr, nullptr};
  // particle buffers of removed scenes, reused by later scenes
  static constexpr int64_t kSceneCacheBytes = int64_t(8) << 30;
  int64_t cache_limit_ = kSceneCacheBytes;  // raised by reserve_scenes()
  std::vector<Scene> cache_;
  int64_t cached_bytes_ = 0;

  cudaGraphExec_t gexec_ = nullptr;
  bool graph_warm_ = false;  // a step ran eagerly: later steps may be captured
  BatchDev graph_args_{};
  std::vector<SceneDev> table_;
  std::vector<Collider> coll_;
  cudaStream_t own_stream_ = nullptr;
  uint32_t last_status_ = 0;
  int64_t last_blocks_ = 0;

  // semi-implicit update
  double imp_beta_ = 0.0, imp_tol2_ = 1e-12;
  int imp_max_iter_ = 50;
  void* imp_nodes_ = nullptr;   // R[16][imp_cap_nodes_]: mass, r, p, Ar, Ap, df
  void* imp_parts_ = nullptr;   // R[17][imp_cap_p_]: polar factors and Lame parameters
  double* imp_dots_ = nullptr;  // 4 dot-product accumulators, then the apply's item counter
  double* imp_host_ = nullptr;  // page-locked copy of the accumulators
  double imp_read_[4] = {0, 0, 0, 0};
  int64_t imp_cap_nodes_ = 0, imp_cap_p_ = 0;
  int last_imp_iters_ = 0;
  double last_imp_res_ = 0.0;

 public:
  void ensure_grid_public(int64_t blocks) { ensure_grid(blocks); }
  void ensure_particle_buffers_public(int64_t total) { ensure_particle_buffers(total); }
};

}  // namespace snow
