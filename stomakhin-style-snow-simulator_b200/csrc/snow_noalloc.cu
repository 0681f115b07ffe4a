// snow_gpu_step_noalloc: the one-scene FP64 step for callers that must not
// allocate device memory.
//
// Some hosts cannot call cudaMalloc from the code that drives the solver: a
// plugin living inside an application that owns the GPU's memory pool (and
// forbids or traps other allocations), or a real-time loop where an
// allocation's implicit device synchronisation is not acceptable.  This entry
// point runs the same kernels as snow_gpu_step on the same host particle
// records, but every piece of device scratch it needs -- the particle planes,
// sort keys, block hash table, grid blocks, counters and the staging copy of
// the records -- is carved out of one file-scope __device__ array of fixed
// size.  It calls no cudaMalloc, cudaFree or allocating library routine.
//
// Limits: at most kMaxParticles particles, kMaxBlocks grid blocks and
// kMaxColliders colliders per call; larger inputs are rejected with
// SNOW_E_ARG, and a step that needs more grid blocks fails with
// SNOW_E_CAPACITY.  The array (about 26 MB) is held on every GPU that loads
// the library until the process exits.
//
// Set-up: the first call on a device (with that device current) looks the
// array's address up with cudaGetSymbolAddress and caches it per device.  With
// lazy module loading (the CUDA default) that first lookup is also when the
// driver loads this module on the device and reserves the array, which can
// synchronise the device or fail if the application has used up its memory.
// A call with n = 0 does only this set-up, so a caller can pay that cost up
// front, e.g. at start-up.  Every call waits for its own copies (it
// synchronises the stream it is given), so it must not be called while that
// stream is being captured into a CUDA graph.
//
// All calls share the one array: calls that overlap on the GPU (different
// streams or host threads) race and must be serialised by the caller.  Each
// call re-zeroes the grid accumulators and counters it relies on, so the
// previous call's leftovers never leak into its result.  On any error the
// caller's records are left as they were.
#include <cuda_runtime.h>

#include <climits>
#include <cstring>
#include <mutex>
#include <string>

#include "snow_batch.cuh"
#include "snow_engine.hpp"
#include "snow_gpu.h"

namespace snow {

int radix_tiles(int64_t n);

namespace {

constexpr int64_t kMaxParticles = 16384;
constexpr int32_t kMaxBlocks = 2048;
constexpr int kMaxColliders = 16;
constexpr uint32_t kHashSlots = 4096;  // power of two, twice kMaxBlocks
constexpr int kTiles = (int)((kMaxParticles + 2047) / 2048);
constexpr int kChunk = 256;
constexpr int kItems = (int)(kMaxParticles / kChunk) + kMaxBlocks + 64;

constexpr size_t up256(size_t x) { return (x + 255) / 256 * 256; }

// Byte offsets of every region inside the arena.
struct Layout {
  size_t staging, r0, r1, fp0, fp1, id0, id1, k0, k1, v0, v1, hist, dtot, htab, blk, item_hdr, acc,
      vel, ctr, scene, coll, total;
  constexpr Layout()
      : staging(0), r0(0), r1(0), fp0(0), fp1(0), id0(0), id1(0), k0(0), k1(0), v0(0), v1(0),
        hist(0), dtot(0), htab(0), blk(0), item_hdr(0), acc(0), vel(0), ctr(0), scene(0), coll(0),
        total(0) {
    size_t o = 0;
    auto take = [&o](size_t bytes) {
      const size_t at = o;
      o = up256(o + bytes);
      return at;
    };
    const size_t N = (size_t)kMaxParticles;
    staging = take(N * 26 * sizeof(double));
    r0 = take(N * kRealPlanes * sizeof(double));
    r1 = take(N * kRealPlanes * sizeof(double));
    fp0 = take(N * kFPPlanes * sizeof(double));
    fp1 = take(N * kFPPlanes * sizeof(double));
    id0 = take(N * sizeof(int32_t));
    id1 = take(N * sizeof(int32_t));
    k0 = take(N * sizeof(uint32_t));
    k1 = take(N * sizeof(uint32_t));
    v0 = take(N * sizeof(uint32_t));
    v1 = take(N * sizeof(uint32_t));
    hist = take((size_t)kTiles * (1 << kRadixBits) * sizeof(uint32_t));
    dtot = take((1 << kRadixBits) * sizeof(uint32_t));
    htab = take(kHashSlots * sizeof(unsigned long long));
    blk = take((size_t)kMaxBlocks * sizeof(int4));
    item_hdr = take((size_t)kItems * sizeof(BlockHeader));
    acc = take((size_t)kMaxBlocks * 64 * kAccCh * sizeof(double));
    vel = take((size_t)kMaxBlocks * 64 * kVelCh * sizeof(double));
    ctr = take(sizeof(Counters));
    scene = take(sizeof(SceneDev));
    coll = take((size_t)kMaxColliders * sizeof(Collider));
    total = o;
  }
};
constexpr Layout kLayout{};

// The scratch array.  Host code must not pass this name to a kernel: on the
// host it is only a stand-in symbol; its device address comes from
// cudaGetSymbolAddress (arena_for_current_device).
static __device__ __align__(256) unsigned char g_noalloc_scratch[kLayout.total];

constexpr int kMaxDevices = 64;
std::mutex g_arena_mu;
void* g_arena[kMaxDevices] = {};

unsigned char* arena_for_current_device() {
  int dev = 0;
  check_cuda(cudaGetDevice(&dev), "cudaGetDevice");
  if (dev < 0 || dev >= kMaxDevices) throw Error(SNOW_E_ARG, "device index out of range");
  std::lock_guard<std::mutex> lk(g_arena_mu);
  if (!g_arena[dev]) {
    void* p = nullptr;
    const cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
    if (e != cudaSuccess || !p)
      throw Error(SNOW_E_CUDA, std::string("cudaGetSymbolAddress(scratch): ") + cudaGetErrorString(e));
    g_arena[dev] = p;
  }
  return static_cast<unsigned char*>(g_arena[dev]);
}

__global__ void k_noalloc_records_in(const double* rec, int64_t n, double* r, double* fp, int32_t* id,
                                     int64_t st) {
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const double* p = rec + 26 * i;
  for (int k = 0; k < 8; ++k) r[k * st + i] = p[k];
  for (int k = 0; k < 9; ++k) fp[k * st + i] = p[8 + k];
  for (int k = 0; k < 9; ++k) r[(PFE + k) * st + i] = p[17 + k];
  id[i] = (int32_t)i;
}

__global__ void k_noalloc_records_out(double* rec, int64_t n, const double* r, const double* fp,
                                      const int32_t* id, int64_t st) {
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  double* p = rec + 26 * (int64_t)id[i];
  for (int k = 0; k < 8; ++k) p[k] = r[k * st + i];
  for (int k = 0; k < 9; ++k) p[8 + k] = fp[k * st + i];
  for (int k = 0; k < 9; ++k) p[17 + k] = r[(PFE + k) * st + i];
}

}  // namespace
}  // namespace snow

using namespace snow;

extern "C" int snow_gpu_step_noalloc(double* records, int64_t n, const snow_step_params* params,
                                     const snow_collider* colliders, int n_colliders, int n_steps,
                                     void* stream) {
  try {
    if (n < 0 || (n > 0 && !records)) throw Error(SNOW_E_ARG, "bad particle array");
    if (n > kMaxParticles)
      throw Error(SNOW_E_ARG, "snow_gpu_step_noalloc: " + std::to_string(n) +
                                  " particles exceed its fixed scratch limit of " +
                                  std::to_string(kMaxParticles));
    if (n_colliders < 0 || n_colliders > kMaxColliders || (n_colliders > 0 && !colliders))
      throw Error(SNOW_E_ARG, "snow_gpu_step_noalloc: at most " + std::to_string(kMaxColliders) +
                                  " colliders");
    if (!params || !(params->grid_spacing > 0.0)) throw Error(SNOW_E_ARG, "bad step parameters");
    if (n_steps < 0) throw Error(SNOW_E_ARG, "negative step count");
    const std::vector<Collider> cols = device_colliders(colliders, n_colliders);
    unsigned char* A = arena_for_current_device();  // per-device set-up (see the header comment)
    if (n == 0 || n_steps == 0) return SNOW_OK;

    cudaStream_t s = static_cast<cudaStream_t>(stream);
    const Layout& L = kLayout;
    const int64_t st = kMaxParticles;
    double* staging = reinterpret_cast<double*>(A + L.staging);
    double* r[2] = {reinterpret_cast<double*>(A + L.r0), reinterpret_cast<double*>(A + L.r1)};
    double* fp[2] = {reinterpret_cast<double*>(A + L.fp0), reinterpret_cast<double*>(A + L.fp1)};
    int32_t* id[2] = {reinterpret_cast<int32_t*>(A + L.id0), reinterpret_cast<int32_t*>(A + L.id1)};
    Counters* ctr = reinterpret_cast<Counters*>(A + L.ctr);
    SceneDev* scene = reinterpret_cast<SceneDev*>(A + L.scene);
    Collider* coll = reinterpret_cast<Collider*>(A + L.coll);

    // Everything that must start at zero, since the array keeps the last call's contents.
    check_cuda(cudaMemsetAsync(A + L.acc, 0, (size_t)kMaxBlocks * 64 * kAccCh * sizeof(double), s), "clear grid");
    check_cuda(cudaMemsetAsync(ctr, 0, sizeof(Counters), s), "clear counters");

    check_cuda(cudaMemcpyAsync(staging, records, (size_t)n * 26 * sizeof(double), cudaMemcpyHostToDevice, s),
               "upload records");
    const unsigned g = (unsigned)((n + 255) / 256);
    k_noalloc_records_in<<<g, 256, 0, s>>>(staging, n, r[0], fp[0], id[0], st);

    SceneDev sd{};
    for (int k = 0; k < 2; ++k) {
      sd.r[k] = r[k];
      sd.fp[k] = fp[k];
      sd.id[k] = id[k];
    }
    sd.stride = st;
    sd.n = n;
    sd.begin = 0;
    sd.cur = 0;
    sd.active = 1;
    sd.dx = params->grid_spacing;
    sd.dt = params->time_step;
    for (int a = 0; a < 3; ++a) sd.g[a] = params->gravity[a];
    sd.mu0 = params->mu_0;
    sd.lambda0 = params->lambda_0;
    sd.xi = params->hardening_coefficient;
    sd.theta_c = params->max_compression;
    sd.theta_s = params->max_stretch;
    sd.alpha = params->alpha;
    sd.coll_begin = 0;
    sd.coll_count = n_colliders;
    for (int a = 0; a < 3; ++a) {
      sd.nb_lo[a] = INT_MAX;
      sd.nb_hi[a] = INT_MIN;
    }
    check_cuda(cudaMemcpyAsync(scene, &sd, sizeof sd, cudaMemcpyHostToDevice, s), "scene");
    if (n_colliders > 0)
      check_cuda(cudaMemcpyAsync(coll, cols.data(), sizeof(Collider) * n_colliders, cudaMemcpyHostToDevice, s),
                 "colliders");

    BatchDev b{};
    b.scenes = scene;
    b.num_scenes = 1;
    b.total = n;
    b.colliders = coll;
    b.keys[0] = reinterpret_cast<uint32_t*>(A + L.k0);
    b.keys[1] = reinterpret_cast<uint32_t*>(A + L.k1);
    b.vals[0] = reinterpret_cast<uint32_t*>(A + L.v0);
    b.vals[1] = reinterpret_cast<uint32_t*>(A + L.v1);
    b.hist = reinterpret_cast<uint32_t*>(A + L.hist);
    b.digit_total = reinterpret_cast<uint32_t*>(A + L.dtot);
    b.ntiles = radix_tiles(n);
    b.htab = reinterpret_cast<unsigned long long*>(A + L.htab);
    b.hmask = kHashSlots - 1;
    b.cap_blocks = kMaxBlocks;
    b.blk = reinterpret_cast<int4*>(A + L.blk);
    b.item_hdr = reinterpret_cast<BlockHeader*>(A + L.item_hdr);
    b.cap_items = kItems;
    b.chunk = kChunk;
    b.acc = A + L.acc;
    b.vel = A + L.vel;
    b.ctr = ctr;

    StepLaunch<double>::bbox_init(b, s);
    for (int k = 0; k < n_steps; ++k) {
      StepLaunch<double>::keyspace(b, s, false);
      StepLaunch<double>::keys(b, s);
      radix_sort(b, s);
      StepLaunch<double>::blocks(b, s);
      StepLaunch<double>::p2g(b, P2G_FULL, s);
      StepLaunch<double>::grid_update(b, s);
      StepLaunch<double>::g2p(b, G2P_FULL, s);
      StepLaunch<double>::finish(b, s);
    }
    const int cur = n_steps & 1;  // k_finish swaps the buffers once per step
    k_noalloc_records_out<<<g, 256, 0, s>>>(staging, n, r[cur], fp[cur], id[cur], st);
    check_cuda(cudaGetLastError(), "noalloc step launch");
    // The status first: the caller's records are only overwritten by a valid result.
    Counters h{};
    check_cuda(cudaMemcpyAsync(&h, ctr, sizeof h, cudaMemcpyDeviceToHost, s), "status");
    check_cuda(cudaStreamSynchronize(s), "noalloc step");
    if (h.status & (ST_BLOCK_OVERFLOW | ST_HASH_FULL))
      throw Error(SNOW_E_CAPACITY, "snow_gpu_step_noalloc: the scene needs more than " +
                                       std::to_string(kMaxBlocks) + " grid blocks; the result is not valid");
    if (h.status & ST_NONFINITE) throw Error(SNOW_E_NONFINITE, "a particle position became NaN or infinite");
    if (h.status & ST_KEY_OVERFLOW) throw Error(SNOW_E_KEYRANGE, "scene extent exceeds the block key range");
    if (h.status) throw Error(SNOW_E_STATE, "internal grid inconsistency (status " + std::to_string(h.status) + ")");
    check_cuda(cudaMemcpyAsync(records, staging, (size_t)n * 26 * sizeof(double), cudaMemcpyDeviceToHost, s),
               "download records");
    check_cuda(cudaStreamSynchronize(s), "noalloc download");
    return SNOW_OK;
  } catch (const Error& e) {
    return set_error(e.code, e.what());
  } catch (const std::exception& e) {
    return set_error(SNOW_E_ARG, e.what());
  }
}
