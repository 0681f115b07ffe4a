// The explicit MPM snow step as fused sm_100a kernels over a batch of scenes.
//
//   keyspace     (1 block)  per-scene key boxes and key bases, sort bit count,
//                            counter resets
//   keys         (1/particle) block key + cell of every particle; with dense
//                            bins, per-key counts (warp-aggregated atomics)
//   bins         (persistent, chained scan over the key bins)
//                            sorted offsets per key, grid block ids per block
//                            key (prefix over keys whose -{0,1}^3 neighbours
//                            hold particles), work items per particle run
//   scatter      (1/particle) counting-sort scatter; work items' neighbour ids
//   (fallback for key boxes beyond the dense bins: radix_sort.cu, then
//    blocks: one pass building the block hash table and the work items)
//   p2g          (persistent, 1 CTA per particle block)
//                            stencil weights, hardening, stress, and the
//                            scatter of mass, momentum and force into a shared
//                            8x8x8-node tile; one global atomic per touched node
//                            per block when the tile is flushed
//   grid_update  (1/node)    v = p/m + dt (f/m + g), collisions at the node,
//                            the FLIP increment, accumulators re-zeroed
//   g2p          (persistent, 1 CTA per particle block)
//                            gather of grad v, PIC and FLIP terms from a shared
//                            tile; elastoplastic update; PIC/FLIP blend; particle
//                            collisions; advection; block-sorted write-back and
//                            the bounding box for the next step
//   finish       (1 block)   swap the particle buffers
//
// Reference stages (src/grid.cpp:359-450): stencil = keys/sort/blocks,
// P2G + force_constitutive + force_grid_accumulation = p2g, grid_velocity +
// grid_collisions = grid_update, stress_update + G2P + particle_collisions +
// position_update = g2p.
#include <cuda_runtime.h>

#include <algorithm>
#include <atomic>
#include <climits>
#include <cstdio>
#include <type_traits>

#include "snow_batch.cuh"
#include "snow_engine.hpp"

namespace snow {

int radix_tiles(int64_t n);

namespace {

template <typename R>
struct Vec;
template <>
struct Vec<float> {
  using two = float2;
};
template <>
struct Vec<double> {
  using two = double2;
};

// 7 x 7 x 7 node tile of a block and its +{0,1}^3 neighbours, x fastest.  The
// y and z strides put the 32 nodes a warp's lanes own in one P2G atomic
// (x in {0,1} + 2k, all (y, z) columns) on 32 distinct banks for float, and
// each half-warp's 16 on distinct 8-byte bank pairs for double.
template <typename R>
struct TileShape;
template <>
struct TileShape<float> {
  static constexpr int Y = 8, Z = 58, N = 408;
};
template <>
struct TileShape<double> {
  static constexpr int Y = 9, Z = 68, N = 470;
};
template <typename R>
SNOW_HD int tile_index(int x, int y, int z) {
  return x + TileShape<R>::Y * y + TileShape<R>::Z * z;
}

__device__ __forceinline__ const uint32_t* sorted_keys(const BatchDev& b) {
  const uint32_t passes = (b.ctr->sort_bits + kRadixBits - 1) / kRadixBits;
  return b.keys[passes & 1];
}
__device__ __forceinline__ const uint32_t* sorted_vals(const BatchDev& b) {
  if (b.dense) return b.vals[1];
  const uint32_t passes = (b.ctr->sort_bits + kRadixBits - 1) / kRadixBits;
  return b.vals[passes & 1];
}
__device__ __forceinline__ void flag(const BatchDev& b, uint32_t bit) { atomicOr(&b.ctr->status, bit); }

// Block coordinate of the particle at x (floor division of the stencil base by 4).
template <typename R>
__device__ __forceinline__ int block_coord(R x, R dx, int& cell) {
  const int base = stencil_base(x / dx);
  cell = base & 3;
  return base >> 2;
}

template <typename R>
struct PlaneView {
  const R* r;
  const double* fp;
  const int32_t* id;
  int64_t st;
  __device__ R at(int plane, int64_t i) const { return r[plane * st + i]; }
};

// ------------------------------------------------------------------ bbox init
// Atomic min/max into a scene's box, skipped when it cannot improve the value
// already there (after the first few updates almost every one is skipped).
__device__ __forceinline__ void box_update(SceneDev& sc, const int lo[3], const int hi[3]) {
  for (int a = 0; a < 3; ++a) {
    if (lo[a] < *(volatile int*)&sc.nb_lo[a]) atomicMin(&sc.nb_lo[a], lo[a]);
    if (hi[a] > *(volatile int*)&sc.nb_hi[a]) atomicMax(&sc.nb_hi[a], hi[a]);
  }
}

template <typename R>
__global__ void __launch_bounds__(256) k_bbox_init(const BatchDev b) {
  const int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  const bool valid = t < b.total;
  int s = -1;
  int lo[3] = {INT_MAX, INT_MAX, INT_MAX};
  int hi[3] = {INT_MIN, INT_MIN, INT_MIN};
  if (valid) {
    s = scene_of(b, t);
    const SceneDev& sc = b.scenes[s];
    const R* r = (const R*)sc.r[sc.cur];
    const int64_t i = t - sc.begin;
    for (int a = 0; a < 3; ++a) {
      const R x = r[(PX + a) * sc.stride + i];
      if (!isfinite((double)x)) {
        flag(b, ST_NONFINITE);
        continue;
      }
      int cell;
      lo[a] = hi[a] = block_coord(x, (R)sc.dx, cell);
    }
  }
  // One update per warp when its particles belong to one scene (the usual case).
  const unsigned full = 0xffffffffu;
  const int s0 = __shfl_sync(full, s, 0);
  if (__all_sync(full, s == s0 || s < 0)) {
    for (int a = 0; a < 3; ++a) {
      lo[a] = __reduce_min_sync(full, lo[a]);
      hi[a] = __reduce_max_sync(full, hi[a]);
    }
    if ((threadIdx.x & 31) == 0 && s0 >= 0) box_update(b.scenes[s0], lo, hi);
  } else if (valid) {
    box_update(b.scenes[s], lo, hi);
  }
}

// ------------------------------------------------------------------ keyspace
// One CTA sets up the key space of a step: 1024 threads take up to 1024
// scenes in one round of each prefix (a served batch holds hundreds).
constexpr int kKeyspaceThreads = 1024;

// Exclusive prefix of one count per scene over the block (up to 1024 threads,
// scenes in rounds of blockDim.x): writes each scene's base and count through
// `put` and returns the total (to every thread).
template <typename Count, typename Put>
__device__ unsigned long long scene_prefix(const BatchDev& b, Count&& count, Put&& put) {
  __shared__ unsigned long long s_carry;
  __shared__ unsigned long long s_warp[32];
  if (threadIdx.x == 0) s_carry = 0;
  __syncthreads();
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  for (int base = 0; base < b.num_scenes; base += blockDim.x) {
    const int s = base + threadIdx.x;
    const unsigned long long cnt = s < b.num_scenes ? count(s) : 0ull;
    unsigned long long x = cnt;
    for (int o = 1; o < 32; o <<= 1) {
      const unsigned long long y = __shfl_up_sync(0xffffffffu, x, o);
      if (lane >= o) x += y;
    }
    if (lane == 31) s_warp[warp] = x;
    __syncthreads();
    unsigned long long before = 0;
    for (int w = 0; w < warp; ++w) before += s_warp[w];
    const unsigned long long incl = s_carry + before + x;
    if (s < b.num_scenes) put(s, incl - cnt, cnt);
    __syncthreads();
    if (threadIdx.x == blockDim.x - 1) s_carry = incl;
    __syncthreads();
  }
  const unsigned long long total = s_carry;
  __syncthreads();  // s_carry is reset by the next call
  return total;
}

__device__ __forceinline__ uint32_t clamp32(unsigned long long v) {
  return (uint32_t)(v > 0xFFFFFFFFull ? 0xFFFFFFFFull : v);
}

// Key boxes of the coming step.  kSwap: also swap every scene's particle
// buffers first (the end of a step: the same launch then prepares the next
// step's keys).
//
// The sorting box of the coming step is the emission box the step just ended
// wrote its particles' keys against, when it wrote them all (emit_ok and no
// emit_fail; keys_ready then tells the keys kernel to do nothing); otherwise
// the particles' own block box, one block of margin on the high side (the
// keys kernel computes the keys).  The emission box for the coming step's G2P
// is the particles' block box grown by one block on every side, plus the same
// high margin: emit_ok when those boxes fit the dense bins.
template <bool kSwap>
__global__ void __launch_bounds__(kKeyspaceThreads) k_keyspace(const BatchDev b) {
  __shared__ int s_emitted, s_cleanup;
  if (kSwap)
    for (int s = threadIdx.x; s < b.num_scenes; s += blockDim.x) b.scenes[s].cur ^= 1;
  if (threadIdx.x == 0) {
    const bool armed = b.ctr->emit_ok != 0;  // the G2P that just ran may have written keys and counts
    const bool tried = kSwap && b.dense && armed;
    s_emitted = tried && !b.ctr->emit_fail;
    // Block keys whose counts were written and will not be consumed: those of
    // a G2P that gave up part way (its emission boxes), or, on a fresh start,
    // those a finished step left for the next one (the current key boxes,
    // which are then the emission boxes that G2P wrote against).
    unsigned long long eb = 0;
    if (kSwap) {
      if (tried && b.ctr->emit_fail) eb = b.ctr->emit_blocks;
    } else if (b.ctr->keys_ready) {
      eb = b.ctr->key_blocks;
    }
    s_cleanup = eb && b.bins && b.occ && eb * 64 <= (unsigned long long)b.cap_bins ? (int)eb : 0;
  }
  __syncthreads();
  const bool emitted = s_emitted != 0;
  if (s_cleanup) {
    // Counts and occupancy G2P wrote that no step will consume: G2P gave up
    // part way (a particle left its emission box, which a particle moving less
    // than a block per step never does), or this is a fresh start (after an
    // upload, setup, a change of scenes or of buffers) and the keys kernel sorts.
    uint4* bins4 = reinterpret_cast<uint4*>(b.bins);
    for (int64_t k = threadIdx.x; k < (int64_t)s_cleanup * 16; k += blockDim.x) bins4[k] = make_uint4(0, 0, 0, 0);
    for (int64_t k = threadIdx.x; k < (int64_t)s_cleanup; k += blockDim.x) b.occ[k] = 0;
    __syncthreads();
  }
  // a scene's particle block box (empty: a one-block box keeps the keys of any
  // particles inside this scene's key range)
  auto measured = [&](const SceneDev& sc, int lo[3], int dim[3], int grow) {
    bool empty = false;
    for (int a = 0; a < 3; ++a) empty |= sc.nb_lo[a] > sc.nb_hi[a];
    for (int a = 0; a < 3; ++a) {
      lo[a] = empty ? 0 : sc.nb_lo[a] - grow;
      dim[a] = empty ? (sc.n > 0 ? 2 : 0) : (sc.nb_hi[a] - sc.nb_lo[a] + 2 + 2 * grow);
    }
  };
  const unsigned long long total = scene_prefix(
      b,
      [&](int s) {
        SceneDev& sc = b.scenes[s];
        int lo[3], dim[3];
        if (emitted) {
          for (int a = 0; a < 3; ++a) lo[a] = sc.elo[a], dim[a] = sc.edim[a];
        } else {
          measured(sc, lo, dim, 0);
        }
        for (int a = 0; a < 3; ++a) sc.lo[a] = lo[a], sc.dim[a] = dim[a];
        return (unsigned long long)dim[0] * dim[1] * dim[2];
      },
      [&](int s, unsigned long long base, unsigned long long cnt) {
        b.scenes[s].key_base = clamp32(base);
        b.scenes[s].key_count = clamp32(cnt);
      });
  const unsigned long long etotal = scene_prefix(
      b,
      [&](int s) {
        SceneDev& sc = b.scenes[s];
        int lo[3], dim[3];
        measured(sc, lo, dim, 1);
        for (int a = 0; a < 3; ++a) {
          sc.elo[a] = lo[a];
          sc.edim[a] = dim[a];
          sc.nb_lo[a] = INT_MAX;
          sc.nb_hi[a] = INT_MIN;
        }
        return (unsigned long long)dim[0] * dim[1] * dim[2];
      },
      [&](int s, unsigned long long base, unsigned long long) { b.scenes[s].ekey_base = clamp32(base); });
  if (threadIdx.x == 0) {
    uint32_t bits = 6;
    if (total > (1ull << 26)) {
      atomicOr(&b.ctr->status, ST_KEY_OVERFLOW);
      bits = 32;
    } else {
      uint32_t kb = 0;
      while ((1ull << kb) < total) ++kb;
      bits += kb;
    }
    Counters* c = b.ctr;
    c->last_blocks = c->n_blocks;  // what the host reads after the last step
    c->last_fp64 = c->fp64_projections;
    c->sort_bits = bits;
    c->key_blocks = (uint32_t)min(total, (unsigned long long)UINT32_MAX);
    if (b.dense && total * 64 > (unsigned long long)b.cap_bins) atomicOr(&c->status, ST_BIN_OVERFLOW);
    c->keys_ready = emitted ? 1u : 0u;
    c->emit_fail = 0;
    c->emit_ok = (b.dense && etotal <= (1ull << 26) && etotal * 64 <= (unsigned long long)b.cap_bins) ? 1u : 0u;
    c->emit_blocks = (uint32_t)min(etotal, (unsigned long long)UINT32_MAX);
    c->bin_ticket = 0;
    c->n_blocks = 0;
    c->work_p2g = c->work_grid = c->work_g2p = c->work_aux = 0;
    c->n_items = 0;
    c->fp64_projections = 0;
  }
}

// ---------------------------------------------------------------------- keys
// Dense bins hold every key of this step's key boxes.
__device__ __forceinline__ bool bins_fit(const BatchDev& b) {
  return (int64_t)b.ctr->key_blocks * 64 <= b.cap_bins;
}

// Runs of equal keys among a warp's consecutive lanes (particles arrive
// nearly sorted, so a warp holds a few long runs): the lane where this lane's
// run starts and the run's length.  Equal keys in separate runs stay separate
// runs, which keeps counts and positions consistent.
__device__ __forceinline__ void key_run(uint32_t key, int lane, int& first, int& len) {
  const uint32_t prev = __shfl_up_sync(0xffffffffu, key, 1);
  const unsigned starts = __ballot_sync(0xffffffffu, lane == 0 || key != prev);
  const unsigned upto = (2u << lane) - 1u;  // lanes 0..lane (all ones for lane 31)
  first = 31 - __clz(starts & upto);
  const unsigned after = starts & ~upto;
  len = (after ? __ffs(after) - 1 : 32) - first;
}

// Sort key of every particle (and its index within its scene).  With dense
// bins, also the per-key particle counts (one atomic per run of equal keys in
// a warp: the particles arrive nearly sorted from the previous step) and the
// occupancy of each block key; the tile states of the bin scan are cleared.
// Nothing to do when the previous step's G2P wrote all of it (keys_ready).
// Grid-stride over warps of 32 consecutive particles, so that a launch with
// nothing to do ends after a small grid.
template <typename R>
__device__ __forceinline__ void keys_for(const BatchDev& b, int64_t t, bool dense);

template <typename R>
__global__ void __launch_bounds__(256) k_keys(const BatchDev b) {
  if (b.ctr->keys_ready) return;
  const bool dense = b.dense && bins_fit(b);
  const int64_t stride = (int64_t)gridDim.x * blockDim.x;
  const int64_t t0 = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (dense) {
    const int64_t ntiles = ((int64_t)b.ctr->key_blocks * 64 + kBinTile - 1) / kBinTile;
    for (int64_t j = t0; j < ntiles; j += stride) b.bin_state[j] = 0;
  }
  const int64_t span = (b.total + 31) / 32 * 32;  // whole warps: key_run uses every lane
  for (int64_t t = t0; t < span; t += stride) keys_for<R>(b, t, dense);
}

template <typename R>
__device__ __forceinline__ void keys_for(const BatchDev& b, int64_t t, bool dense) {
  const bool valid = t < b.total;
  uint32_t key = 0xFFFFFFFFu;
  if (valid) {
    const int s = scene_of(b, t);
    const SceneDev& sc = b.scenes[s];
    const R* r = (const R*)sc.r[sc.cur];
    const int64_t i = t - sc.begin;
    const R dx = (R)sc.dx;
    int blk[3], cell[3];
    bool ok = true;
    for (int a = 0; a < 3; ++a) {
      const R x = r[(PX + a) * sc.stride + i];
      if (!isfinite((double)x)) {
        ok = false;
        blk[a] = sc.lo[a];
        cell[a] = 0;
        continue;
      }
      blk[a] = block_coord(x, dx, cell[a]);
      if (blk[a] < sc.lo[a] || blk[a] > sc.lo[a] + sc.dim[a] - 2) {
        ok = false;
        blk[a] = sc.lo[a];
      }
    }
    if (!ok) flag(b, ST_OUT_OF_BOX);
    const uint32_t bk = block_key(sc, blk[0], blk[1], blk[2]);
    key = (bk << 6) | (uint32_t)(cell[0] + 4 * cell[1] + 16 * cell[2]);
    // boxes beyond the 32-bit key range: the step only reports the error, so
    // every particle gets key 0 (a valid key) and no index goes astray
    if (b.ctr->status & ST_KEY_OVERFLOW) key = 0;
    b.keys[0][t] = key;
    b.vals[0][t] = (uint32_t)i;
  }
  if (!dense) return;
  const int lane = threadIdx.x & 31;
  int first, len;
  key_run(key, lane, first, len);
  if (valid && lane == first) {
    atomicAdd(&b.bins[key], (uint32_t)len);
    b.occ[key >> 6] = 1;
  }
}

// ---------------------------------------------------------------- dense bins
// Index of the scene whose key range holds block key bk (the last scene with
// key_base <= bk: scenes with empty boxes share the next scene's base).
__device__ __forceinline__ int scene_of_key(const BatchDev& b, uint32_t bk) {
  int lo = 0, hi = b.num_scenes - 1;
  while (lo < hi) {
    const int mid = (lo + hi + 1) >> 1;
    if (b.scenes[mid].key_base <= bk) lo = mid; else hi = mid - 1;
  }
  return lo;
}

// Chained-scan tile state: flag in bits 62-63 (1 aggregate, 2 inclusive
// prefix), particles in bits 0-35, grid blocks in bits 36-61.
constexpr unsigned long long kTileAgg = 1ull << 62, kTileIncl = 2ull << 62;
constexpr unsigned long long kTileVal = (1ull << 62) - 1;
constexpr int kBlkShift = 36;
constexpr unsigned long long kPartMask = (1ull << kBlkShift) - 1;

__device__ __forceinline__ unsigned long long warp_sum64(unsigned long long v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}

// One pass over the dense bins (a chained scan with decoupled look-back; tiles
// are taken in order from a ticket, so a tile only waits on tiles whose CTAs
// are already running).  Thread q = 0..3 of each group of four owns 16 cells
// of one block key.  Per key: the first sorted position (exclusive prefix of
// the counts), and the counts re-zeroed.  Per block key: whether any of the
// blocks at -{0,1}^3 holds particles (then it is a grid block, id = prefix of
// such keys), its coordinates, and the work items of its particle run.
__global__ void __launch_bounds__(256) k_bins(const BatchDev b) {
  __shared__ unsigned long long s_warp[8];
  __shared__ unsigned long long s_prefix;
  __shared__ uint32_t s_items[8];
  __shared__ uint32_t s_tile, s_item_base;
  if (!bins_fit(b)) return;
  const int64_t K = b.ctr->key_blocks;
  const int64_t ntiles = (K * 64 + kBinTile - 1) / kBinTile;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, q = threadIdx.x & 3;
  volatile unsigned long long* state = b.bin_state;
  for (;;) {
    if (threadIdx.x == 0) s_tile = atomicAdd(&b.ctr->bin_ticket, 1u);
    __syncthreads();
    const int64_t tile = s_tile;
    if (tile >= ntiles) return;
    const int64_t bin0 = tile * kBinTile + threadIdx.x * 16;
    const int64_t bk = bin0 >> 6;
    const bool live = bk < K;
    // A block key without particles (occupancy 0) has zero counts: its counts
    // are neither read nor cleared, and its offsets are never looked up.
    const bool occupied = live && b.occ[bk] != 0;
    uint32_t c[16];
    uint32_t sum = 0;
    if (occupied) {
      const uint4* src = reinterpret_cast<const uint4*>(b.bins + bin0);
#pragma unroll
      for (int v = 0; v < 4; ++v) {
        const uint4 w = src[v];
        c[4 * v] = w.x;
        c[4 * v + 1] = w.y;
        c[4 * v + 2] = w.z;
        c[4 * v + 3] = w.w;
      }
    } else {
#pragma unroll
      for (int k = 0; k < 16; ++k) c[k] = 0;
    }
#pragma unroll
    for (int k = 0; k < 16; ++k) sum += c[k];
    uint32_t blk_count = sum + __shfl_xor_sync(0xffffffffu, sum, 1);
    blk_count += __shfl_xor_sync(0xffffffffu, blk_count, 2);
    int s = 0, cx = 0, cy = 0, cz = 0;
    bool need = false;
    if (live && q == 0) {
      s = scene_of_key(b, (uint32_t)bk);
      const SceneDev& sc = b.scenes[s];
      const uint32_t local = (uint32_t)bk - sc.key_base;
      const uint32_t d0 = (uint32_t)sc.dim[0], d01 = d0 * (uint32_t)sc.dim[1];
      cx = (int)(local % d0);
      cy = (int)((local / d0) % (uint32_t)sc.dim[1]);
      cz = (int)(local / d01);
#pragma unroll
      for (int d = 0; d < 8; ++d) {
        const int ox = d & 1, oy = (d >> 1) & 1, oz = d >> 2;
        if (cx >= ox && cy >= oy && cz >= oz) need |= b.occ[bk - (ox + oy * d0 + oz * d01)] != 0;
      }
    }
    const unsigned long long v = sum + (need ? (1ull << kBlkShift) : 0ull);
    // inclusive scan of v over the CTA
    unsigned long long x = v;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const unsigned long long y = __shfl_up_sync(0xffffffffu, x, o);
      if (lane >= o) x += y;
    }
    if (lane == 31) s_warp[warp] = x;
    // work items of the block's particle run (owned by q == 0)
    const uint32_t n_it = (q == 0 && blk_count > 0) ? (blk_count + b.chunk - 1) / b.chunk : 0u;
    uint32_t it_x = n_it;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const uint32_t y = __shfl_up_sync(0xffffffffu, it_x, o);
      if (lane >= o) it_x += y;
    }
    if (lane == 31) s_items[warp] = it_x;
    __syncthreads();
    unsigned long long before = 0;
    uint32_t it_before = 0;
    for (int w = 0; w < warp; ++w) {
      before += s_warp[w];
      it_before += s_items[w];
    }
    if (warp == 0) {
      unsigned long long agg = 0;
      uint32_t it_total = 0;
      for (int w = 0; w < 8; ++w) {
        agg += s_warp[w];
        it_total += s_items[w];
      }
      if (lane == 0) {
        state[tile] = (tile == 0 ? kTileIncl : kTileAgg) | agg;
        s_item_base = it_total ? atomicAdd(&b.ctr->n_items, it_total) : 0u;
      }
      unsigned long long excl = 0;
      if (tile > 0) {
        int64_t p = tile - 1;
        int spin = 0;
        for (;;) {
          const int64_t j = p - lane;
          unsigned long long st = 2ull << 62;  // before tile 0: an empty inclusive prefix
          if (j >= 0) st = state[j];
          if (__any_sync(0xffffffffu, (st >> 62) == 0)) {
            if (++spin > (1 << 22)) {
              if (lane == 0) flag(b, ST_SCAN_STALL);
              break;
            }
            __nanosleep(32);
            continue;
          }
          const unsigned incl = __ballot_sync(0xffffffffu, (st >> 62) == 2);
          if (incl) {
            const int first = __ffs(incl) - 1;
            excl += warp_sum64(lane <= first ? (st & kTileVal) : 0ull);
            break;
          }
          excl += warp_sum64(st & kTileVal);
          p -= 32;
        }
        if (lane == 0) state[tile] = kTileIncl | (excl + agg);
      }
      if (lane == 0) {
        s_prefix = excl;
        if (tile == ntiles - 1) b.ctr->n_blocks = (uint32_t)((excl + agg) >> kBlkShift);
      }
    }
    __syncthreads();
    const unsigned long long run = s_prefix + before + x - v;
    uint32_t pos = (uint32_t)(run & kPartMask);
    if (occupied) {
      uint4* off = reinterpret_cast<uint4*>(b.bin_off + bin0);
      uint4* zero = reinterpret_cast<uint4*>(b.bins + bin0);
#pragma unroll
      for (int w = 0; w < 4; ++w) {
        uint4 o;
        o.x = pos;
        pos += c[4 * w];
        o.y = pos;
        pos += c[4 * w + 1];
        o.z = pos;
        pos += c[4 * w + 2];
        o.w = pos;
        pos += c[4 * w + 3];
        off[w] = o;
        zero[w] = make_uint4(0, 0, 0, 0);
      }
    }
    if (live && q == 0) {
      const uint32_t id = (uint32_t)(run >> kBlkShift);
      int32_t mapped = -1;
      if (need) {
        if ((int64_t)id < b.cap_blocks) {
          const SceneDev& sc = b.scenes[s];
          b.blk[id] = make_int4(sc.lo[0] + cx, sc.lo[1] + cy, sc.lo[2] + cz, s);
          mapped = (int32_t)id;
        } else {
          flag(b, ST_BLOCK_OVERFLOW);
        }
      }
      b.idmap[bk] = mapped;
      const uint32_t start = (uint32_t)(run & kPartMask);
      if (n_it && (int64_t)start + blk_count > b.total) flag(b, ST_LOOKUP_MISS);
      else if (n_it) {
        const SceneDev& sc = b.scenes[s];
        uint32_t item = s_item_base + it_before + it_x - n_it;
        for (uint32_t k = 0; k < n_it; ++k, ++item) {
          if ((int64_t)item >= b.cap_items) {
            flag(b, ST_BLOCK_OVERFLOW);
            break;
          }
          BlockHeader* h = b.item_hdr + item;
          const uint32_t a = start + k * (uint32_t)b.chunk;
          h->start = (int32_t)a;
          h->end = (int32_t)min(a + (uint32_t)b.chunk, start + blk_count);
          h->scene = s;
          h->bx = sc.lo[0] + cx;
          h->by = sc.lo[1] + cy;
          h->bz = sc.lo[2] + cz;
          h->pad0 = h->pad1 = 0;
        }
      }
    }
    __syncthreads();  // s_tile, s_prefix and s_item_base are reused by the next tile
  }
}

// Counting-sort scatter (the order of particles with equal keys is that of
// the runs' atomics; within a run it follows the input), the occupancy
// bytes cleared for the next step, and the neighbour ids of every work item.
__global__ void __launch_bounds__(256) k_scatter(const BatchDev b) {
  if (!bins_fit(b)) return;
  const int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  // the scan's tile states are spent: clear every tile for the next step (whose
  // keys G2P may write before any other kernel runs)
  for (int64_t j = t; j < b.cap_bins / kBinTile + 1; j += (int64_t)gridDim.x * blockDim.x) b.bin_state[j] = 0;
  const int lane = threadIdx.x & 31;
  const bool valid = t < b.total;
  const uint32_t key = valid ? b.keys[0][t] : 0xFFFFFFFFu;
  int first, len;
  key_run(key, lane, first, len);
  uint32_t base = 0;
  if (valid && lane == first) {
    base = atomicAdd(&b.bin_off[key], (uint32_t)len);
    b.occ[key >> 6] = 0;
  }
  base = __shfl_sync(0xffffffffu, base, first);
  const uint32_t pos = base + (uint32_t)(lane - first);
  if (valid) {
    if (pos < b.total)
      b.vals[1][pos] = b.vals[0][t];
    else
      flag(b, ST_LOOKUP_MISS);
  }
  const int64_t work = (int64_t)min(b.ctr->n_items, (uint32_t)b.cap_items) * 8;
  for (int64_t e = t; e < work; e += (int64_t)gridDim.x * blockDim.x) {
    BlockHeader* h = b.item_hdr + (e >> 3);
    const int d = (int)(e & 7);
    const SceneDev& sc = b.scenes[h->scene];
    const int32_t id = b.idmap[block_key(sc, h->bx + (d & 1), h->by + ((d >> 1) & 1), h->bz + (d >> 2))];
    if (id < 0) flag(b, ST_LOOKUP_MISS);
    h->nbr[d] = id;
  }
}

// -------------------------------------------------------------------- blocks
// Id of block `key` (coordinates and scene in bc), inserting it if absent.
// Table entries hold (key << 32) | id.  The thread whose CAS claims an empty
// slot stores the key with a pending id, takes the next block id and publishes
// it; a thread that meets the key while its id is pending waits for it (the
// claiming thread is running, so the wait is short; it is bounded all the
// same and reports ST_HASH_FULL if it runs out).
constexpr uint32_t kPendingId = 0xFFFFFFFFu;
__device__ __forceinline__ int32_t block_id(const BatchDev& b, uint32_t key, int4 bc) {
  uint32_t slot = hash32(key) & b.hmask;
  volatile unsigned long long* tab = b.htab;
  const unsigned long long pending = ((unsigned long long)key << 32) | kPendingId;
  for (uint32_t probe = 0; probe <= b.hmask; ++probe) {
    unsigned long long e = tab[slot];
    if (e == kEmptyEntry) {
      e = atomicCAS(&b.htab[slot], kEmptyEntry, pending);
      if (e == kEmptyEntry) {
        const uint32_t id = atomicAdd(&b.ctr->n_blocks, 1u);
        if ((int64_t)id >= b.cap_blocks) {
          flag(b, ST_BLOCK_OVERFLOW);
          atomicExch(&b.htab[slot], ((unsigned long long)key << 32) | 0x7FFFFFFFu);
          return -1;
        }
        b.blk[id] = bc;
        __threadfence();
        atomicExch(&b.htab[slot], ((unsigned long long)key << 32) | id);
        return (int32_t)id;
      }
    }
    if ((uint32_t)(e >> 32) == key) {
      for (int spin = 0; (uint32_t)e == kPendingId; ++spin) {
        if (spin == (1 << 20)) {
          flag(b, ST_HASH_FULL);
          return -1;
        }
        __nanosleep(20);
        e = tab[slot];
      }
      const int32_t id = (int32_t)(uint32_t)e;
      return id < b.cap_blocks ? id : -1;
    }
    slot = (slot + 1) & b.hmask;
  }
  flag(b, ST_HASH_FULL);
  return -1;
}

__device__ __forceinline__ int4 decode_block(const SceneDev& sc, uint32_t bk, int s) {
  uint32_t local = bk - sc.key_base;
  const int bx = sc.lo[0] + (int)(local % (uint32_t)sc.dim[0]);
  local /= (uint32_t)sc.dim[0];
  const int by = sc.lo[1] + (int)(local % (uint32_t)sc.dim[1]);
  const int bz = sc.lo[2] + (int)(local / (uint32_t)sc.dim[1]);
  return make_int4(bx, by, bz, s);
}

// Block table and work items in one pass, one CTA per `chunk` sorted positions
// (blockDim.x == chunk).  A work item is a run of consecutive particles of one
// block inside one chunk: it starts at a chunk start or at the first particle of
// a block (a change of block key) and ends at the next such position.  The
// thread at an item's start inserts or finds the ids of the item's block and
// its +{0,1}^3 neighbours (the blocks its particles' stencils reach) and writes
// the item header the particle kernels read.
__global__ void __launch_bounds__(1024) k_blocks(const BatchDev b) {
  __shared__ unsigned s_mask[32];
  const int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nwarps = (blockDim.x + 31) >> 5;
  const bool valid = t < b.total;
  const uint32_t* K = sorted_keys(b);
  const uint32_t bk = valid ? K[t] >> 6 : 0;
  const bool start = valid && (threadIdx.x == 0 || t == 0 || (K[t - 1] >> 6) != bk);
  const unsigned m = __ballot_sync(0xffffffffu, start);
  if (lane == 0) s_mask[warp] = m;
  __syncthreads();
  if (!start) return;
  // the next item start inside this chunk (or the chunk's end)
  int next = blockDim.x;
  for (int w = warp; w < nwarps; ++w) {
    unsigned rest = s_mask[w];
    if (w == warp) rest = lane == 31 ? 0u : rest & (~0u << (lane + 1));
    if (rest) {
      next = w * 32 + __ffs(rest) - 1;
      break;
    }
  }
  const int s = scene_of(b, t);
  const SceneDev& sc = b.scenes[s];
  const int4 c = decode_block(sc, bk, s);
  BlockHeader h;
  h.start = (int32_t)t;
  h.end = (int32_t)min((int64_t)blockIdx.x * blockDim.x + next, b.total);
  h.scene = s;
  h.bx = c.x;
  h.by = c.y;
  h.bz = c.z;
  h.pad0 = h.pad1 = 0;
#pragma unroll
  for (int d = 0; d < 8; ++d) {
    const int nx = c.x + (d & 1), ny = c.y + ((d >> 1) & 1), nz = c.z + (d >> 2);
    h.nbr[d] = block_id(b, block_key(sc, nx, ny, nz), make_int4(nx, ny, nz, s));
  }
  const uint32_t item = atomicAdd(&b.ctr->n_items, 1u);
  if ((int64_t)item >= b.cap_items) {
    flag(b, ST_BLOCK_OVERFLOW);
    return;
  }
  b.item_hdr[item] = h;
}

// Number of grid blocks this step.
__device__ __forceinline__ uint32_t num_blocks(const BatchDev& b) {
  return min(b.ctr->n_blocks, (uint32_t)b.cap_blocks);
}

// Work-item queue of a persistent CTA.  Warp 0 claims the next item and loads
// its header into registers while the CTA works on the current one, so a claim
// costs no dependent global loads.  claim() stores the header in one shared
// buffer between two barriers; claim_buffered() stores it in the other of two
// buffers (the one of the item before, which nobody reads any more) and needs
// one barrier.
struct ItemQueue {
  int next;     // item claimed ahead (warp 0)
  int word;     // header word `lane` of that item (lanes 0..15 of warp 0)
  int cur = 0;  // header buffer of the current item
  __device__ void fetch(const BatchDev& b, uint32_t* counter, uint32_t items) {
    if (threadIdx.x >= 32) return;
    int n = 0;
    if (threadIdx.x == 0) n = (int)atomicAdd(counter, 1u);
    next = __shfl_sync(0xffffffffu, n, 0);
    if (threadIdx.x < 16 && (uint32_t)next < items) word = reinterpret_cast<const int*>(b.item_hdr + next)[threadIdx.x];
  }
  __device__ bool claim(const BatchDev& b, uint32_t* counter, BlockHeader& h, int& s_next) {
    const uint32_t items = min(b.ctr->n_items, (uint32_t)b.cap_items);
    __syncthreads();  // everyone is done with the previous item's header and tile
    if (threadIdx.x < 16) reinterpret_cast<int*>(&h)[threadIdx.x] = word;
    if (threadIdx.x == 0) s_next = next;
    __syncthreads();
    if ((uint32_t)s_next >= items) return false;
    fetch(b, counter, items);
    return true;
  }
  // The next item's header (hdr[2], s_next[2] in shared memory), or null when
  // the queue is empty.
  __device__ const BlockHeader* claim_buffered(const BatchDev& b, uint32_t* counter, BlockHeader* hdr,
                                               int* s_next) {
    const uint32_t items = min(b.ctr->n_items, (uint32_t)b.cap_items);
    const int nb = cur ^ 1;
    if (threadIdx.x < 16) reinterpret_cast<int*>(&hdr[nb])[threadIdx.x] = word;
    if (threadIdx.x == 0) s_next[nb] = next;
    __syncthreads();  // everyone is done with the previous item's tile; its successor's header is stored
    cur = nb;
    if ((uint32_t)s_next[cur] >= items) return nullptr;
    fetch(b, counter, items);
    return &hdr[cur];
  }
};

// Tile position of local node `node` (0..63) of neighbour d; false if outside
// the 7x7x7 region a particle block's stencils can reach.
template <typename R>
__device__ __forceinline__ bool tile_of(int d, int node, int& t) {
  const int x = 4 * (d & 1) + (node & 3);
  const int y = 4 * ((d >> 1) & 1) + ((node >> 2) & 3);
  const int z = 4 * (d >> 2) + (node >> 4);
  t = tile_index<R>(x, y, z);
  return x <= 6 && y <= 6 && z <= 6;
}

// -------------------------------------------------------------------- P2G
template <typename R, int MODE>
struct P2GChannels {
  static constexpr int n = MODE == P2G_MASS ? 1 : (MODE == P2G_MASS_MOMENTUM ? 4 : 7);
};

// Per-particle record staged in shared memory for the scatter: the stencil
// weights and slopes per axis, then m, m v, and the symmetric force matrix.
// y and z hold (weight, slope) pairs per stencil offset.  In double, x does
// too and the force matrix is (xx, yy, zz, xy, xz, yz).  In float the record
// is laid out for the packed two-wide arithmetic of the scatter: x holds
// (w_q, w_q+2, dw_q, dw_q+2) for q = 0, 1 (the two nodes of a lane) and the
// force matrix is (xx, xy, xy, yy, xz, yz, zz, 0), whose pairs are the rows
// M e_x, M e_y, M e_z as the scatter combines them.  Record strides (36
// floats, 34 doubles) make the 16-byte record stores of a warp conflict-free.
enum : int { RW_X = 0, RW_Y = 8, RW_Z = 16, R_M = 24, R_MV = 25, R_F = 28 };
constexpr int kP2GWarps = 8;

template <typename R>
constexpr int rec_stride() {
  return sizeof(R) == 4 ? 36 : 34;
}

template <typename R, int MODE>
constexpr size_t p2g_smem() {
  return sizeof(R) * (P2GChannels<R, MODE>::n * TileShape<R>::N + kP2GWarps * 32 * rec_stride<R>());
}

// Stores a record (36 floats, 34 doubles) with 16-byte stores.
__device__ __forceinline__ void store_record(float* rr, const float (&v)[36]) {
#pragma unroll
  for (int k = 0; k < 9; ++k)
    reinterpret_cast<float4*>(rr)[k] = make_float4(v[4 * k], v[4 * k + 1], v[4 * k + 2], v[4 * k + 3]);
}
__device__ __forceinline__ void store_record(double* rr, const double (&v)[34]) {
#pragma unroll
  for (int k = 0; k < 17; ++k) reinterpret_cast<double2*>(rr)[k] = make_double2(v[2 * k], v[2 * k + 1]);
}

__device__ __forceinline__ float2 splat2(float a) { return make_float2(a, a); }

// The record walk of the scatter below in float, with the packed two-wide
// arithmetic of sm_100 (__ffma2_rn / __fmul2_rn: two fmaf / fmul in one
// instruction, same rounding).  Per lane and particle: {A, B, C} from the y and
// z weights, P = A (m, m v) and U = A M e_x, V = B M e_y + C M e_z as channel
// pairs, then for each of the lane's two x nodes (w, dw): (m, m v) += w P and
// f += dw U + w V.
template <int MODE>
__device__ __forceinline__ void p2g_walk_f32(const float* wrec, float* tile, int my_cell, int cnt, int lane, int qi,
                                             int qj, int qk, int col) {
  constexpr int N = TileShape<float>::N, kRec = rec_stride<float>();
  constexpr bool kMom = MODE == P2G_FULL || MODE == P2G_PRE || MODE == P2G_MASS_MOMENTUM;
  constexpr bool kForce = MODE == P2G_FULL || MODE == P2G_PRE || MODE == P2G_FORCE;
  constexpr bool kMass = MODE != P2G_FORCE;
  const float2 zero = make_float2(0.f, 0.f);
  float2 am01[2] = {zero, zero}, am23[2] = {zero, zero}, af01[2] = {zero, zero};
  float af2[2] = {0.f, 0.f};
  auto add = [&](int qq) {
    const float* rr = wrec + qq * kRec;
    const float2 py = *reinterpret_cast<const float2*>(rr + RW_Y + 2 * qj);
    const float2 pz = *reinterpret_cast<const float2*>(rr + RW_Z + 2 * qk);
    const float4 xw = *reinterpret_cast<const float4*>(rr + RW_X + 4 * qi);
    const float A = py.x * pz.x;
    const float2 A2 = splat2(A);
    float2 P01 = zero, P23 = zero;
    if constexpr (kMass || kMom) {
      const float4 mm = *reinterpret_cast<const float4*>(rr + R_M);  // m, m v
      P01 = __fmul2_rn(A2, make_float2(mm.x, mm.y));
      P23 = __fmul2_rn(A2, make_float2(mm.z, mm.w));
    }
    float2 U01 = zero, V01 = zero;
    float U2 = 0.f, V2 = 0.f;
    if constexpr (kForce) {
      const float4 f0 = *reinterpret_cast<const float4*>(rr + R_F);      // xx, xy | xy, yy
      const float4 f1 = *reinterpret_cast<const float4*>(rr + R_F + 4);  // xz, yz | zz, -
      const float B = py.y * pz.x, C = py.x * pz.y;
      U01 = __fmul2_rn(A2, make_float2(f0.x, f0.y));
      U2 = A * f1.x;
      V01 = __ffma2_rn(splat2(C), make_float2(f1.x, f1.y), __fmul2_rn(splat2(B), make_float2(f0.z, f0.w)));
      V2 = fmaf(C, f1.z, B * f1.y);
    }
    const float w[2] = {xw.x, xw.y}, dw[2] = {xw.z, xw.w};
#pragma unroll
    for (int x = 0; x < 2; ++x) {
      const float2 w2 = splat2(w[x]);
      if constexpr (kMass || kMom) {
        am01[x] = __ffma2_rn(w2, P01, am01[x]);
        am23[x] = __ffma2_rn(w2, P23, am23[x]);
      }
      if constexpr (kForce) {
        af01[x] = __ffma2_rn(splat2(dw[x]), U01, __ffma2_rn(w2, V01, af01[x]));
        af2[x] = fmaf(dw[x], U2, fmaf(w[x], V2, af2[x]));
      }
    }
  };
  auto flush = [&](int at) {
#pragma unroll
    for (int x = 0; x < 2; ++x) {
      float* t = tile + at + col + qi + 2 * x;
      if constexpr (kMass) atomicAdd(t, am01[x].x);
      if constexpr (kMom) {
        atomicAdd(t + N, am01[x].y);
        atomicAdd(t + 2 * N, am23[x].x);
        atomicAdd(t + 3 * N, am23[x].y);
      }
      if constexpr (kForce) {
        atomicAdd(t + 4 * N, af01[x].x);
        atomicAdd(t + 5 * N, af01[x].y);
        atomicAdd(t + 6 * N, af2[x]);
      }
      am01[x] = am23[x] = af01[x] = zero;
      af2[x] = 0.f;
    }
  };
  // Walk the runs of equal cells (the particles arrive cell-sorted): the run
  // boundaries come from one ballot, so the inner loop carries no per-particle
  // cell test.
  const int prev = __shfl_up_sync(0xffffffffu, my_cell, 1);
  unsigned starts = __ballot_sync(0xffffffffu, lane < cnt && (lane == 0 || my_cell != prev));
  while (starts) {
    const int s0 = __ffs(starts) - 1;
    starts &= starts - 1;
    const int e0 = starts ? __ffs(starts) - 1 : cnt;
    const int cell = __shfl_sync(0xffffffffu, my_cell, s0);
    if (cell < 0) continue;  // particles outside the tile (flagged by the caller)
    int qq = s0;
    for (; qq + 1 < e0; qq += 2) {
      add(qq);
      add(qq + 1);
    }
    if (qq < e0) add(qq);
    flush(cell);
  }
}

// P2G with the lanes of a warp mapped to stencil nodes rather than particles.
//
// A warp takes 32 consecutive particles of the block's cell-sorted run.  First
// every lane evaluates one particle -- weights, m v, the force matrix -- into a
// shared-memory record.  Then the warp walks the 32 records in order; lane l
// owns the two stencil nodes (l>>4 + {0,2}, (l>>2)&3, l&3) of the current
// particle and adds that particle's mass, momentum and force into registers.
// Per (y, z) column the lane forms A = wy wz, B = dwy wz, C = wy dwz once,
// then U = A M e_x and V = B M e_y + C M e_z, so a node (wx, dwx) of the
// column takes wx (m, m v) A and dwx U + wx V: M grad w with grad w =
// (dwx A, wx B, wx C).  Consecutive particles share a cell, so the register sums only leave
// the warp (as shared-memory atomics into the block tile) when the cell
// changes.  The tile is flushed to the global grid with one atomic per node and
// channel.
template <typename R, int MODE>
__global__ void __launch_bounds__(256, sizeof(R) == 4 ? 4 : 2) k_p2g(const BatchDev b) {
  constexpr int NCH = P2GChannels<R, MODE>::n;
  constexpr int kRec = rec_stride<R>();
  constexpr bool kMom = MODE == P2G_FULL || MODE == P2G_PRE || MODE == P2G_MASS_MOMENTUM;
  constexpr bool kForce = MODE == P2G_FULL || MODE == P2G_PRE || MODE == P2G_FORCE;
  constexpr bool kMass = MODE != P2G_FORCE;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  R* tile = reinterpret_cast<R*>(smem_raw);  // [NCH][TileShape<R>::N]
  R* recs = tile + NCH * TileShape<R>::N;              // [warps][32][kRec]
  __shared__ BlockHeader hbuf[2];
  __shared__ int s_next[2];
  R* acc_g = (R*)b.acc;
  const int64_t plane = (int64_t)b.cap_blocks * 64;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  R* wrec = recs + warp * 32 * kRec;
  const int qi = lane >> 4, qj = (lane >> 2) & 3, qk = lane & 3;
  const int col = tile_index<R>(0, qj, qk);

  // The tile is zeroed once here; each item's flush clears what it adds (the
  // barrier at the next claim orders that before the next item's walk).
  for (int e = threadIdx.x; e < NCH * TileShape<R>::N; e += blockDim.x) tile[e] = R(0);
  ItemQueue q;
  q.fetch(b, &b.ctr->work_p2g, min(b.ctr->n_items, (uint32_t)b.cap_items));
  while (const BlockHeader* hp = q.claim_buffered(b, &b.ctr->work_p2g, hbuf, s_next)) {
    const BlockHeader& h = *hp;
    const SceneDev& sc = b.scenes[h.scene];
    const R dx = (R)sc.dx;
    const PlaneView<R> pv{(const R*)sc.r[sc.cur], sc.fp[sc.cur], sc.id[sc.cur], sc.stride};
    const uint32_t* vals = sorted_vals(b);
    const int n = h.end - h.start;
    for (int base = warp * 32; base < n; base += kP2GWarps * 32) {
      const int p = base + lane;
      int my_cell = -1;
      if (p < n) {
        const int64_t i = vals[h.start + p];
        const R x0 = pv.at(PX, i), x1 = pv.at(PX + 1, i), x2 = pv.at(PX + 2, i);
        const AxisWeights<R> wx = axis_weights(x0, dx), wy = axis_weights(x1, dx), wz = axis_weights(x2, dx);
        const int tx = wx.base - 4 * h.bx, ty = wy.base - 4 * h.by, tz = wz.base - 4 * h.bz;
        R v[kRec];
#pragma unroll
        for (int a = 0; a < 4; ++a) {
          if constexpr (sizeof(R) == 4) {
            v[RW_X + 4 * (a & 1) + (a >> 1)] = wx.w[a];
            v[RW_X + 4 * (a & 1) + 2 + (a >> 1)] = wx.dw[a];
          } else {
            v[RW_X + 2 * a] = wx.w[a];
            v[RW_X + 2 * a + 1] = wx.dw[a];
          }
          v[RW_Y + 2 * a] = wy.w[a];
          v[RW_Y + 2 * a + 1] = wy.dw[a];
          v[RW_Z + 2 * a] = wz.w[a];
          v[RW_Z + 2 * a + 1] = wz.dw[a];
        }
        const R m = pv.at(PM, i);
        v[R_M] = m;
        v[R_MV] = v[R_MV + 1] = v[R_MV + 2] = R(0);
        if constexpr (kMom) {
          v[R_MV] = m * pv.at(PV, i);
          v[R_MV + 1] = m * pv.at(PV + 1, i);
          v[R_MV + 2] = m * pv.at(PV + 2, i);
        }
#pragma unroll
        for (int e = R_F; e < kRec; ++e) v[e] = R(0);
        Sym3<R> M{R(0), R(0), R(0), R(0), R(0), R(0)};
        if constexpr (MODE == P2G_PRE) {
          // force matrix left by the previous step's G2P (or prepare_force)
          M = Sym3<R>{pv.at(PFM, i), pv.at(PFM + 1, i), pv.at(PFM + 2, i),
                      pv.at(PFM + 3, i), pv.at(PFM + 4, i), pv.at(PFM + 5, i)};
        } else if constexpr (kForce) {
          M3<R> FE;
#pragma unroll
          for (int e = 0; e < 9; ++e) FE.a[e] = pv.at(PFE + e, i);
          M3<double> FP;
#pragma unroll
          for (int e = 0; e < 9; ++e) FP.a[e] = pv.fp[e * pv.st + i];
          const double hard = exp(sc.xi * (1.0 - det3(FP)));
          M = force_matrix<R>(FE, pv.at(PVOL, i), (R)sc.mu0, (R)sc.lambda0, (R)hard);
        }
        if constexpr (sizeof(R) == 4) {
          v[R_F] = M.xx;
          v[R_F + 1] = M.xy;
          v[R_F + 2] = M.xy;
          v[R_F + 3] = M.yy;
          v[R_F + 4] = M.xz;
          v[R_F + 5] = M.yz;
          v[R_F + 6] = M.zz;
        } else {
          v[R_F] = M.xx;
          v[R_F + 1] = M.yy;
          v[R_F + 2] = M.zz;
          v[R_F + 3] = M.xy;
          v[R_F + 4] = M.xz;
          v[R_F + 5] = M.yz;
        }
        store_record(wrec + lane * kRec, v);
        const bool inside = (unsigned)tx <= 3u && (unsigned)ty <= 3u && (unsigned)tz <= 3u;
        if (!inside) flag(b, ST_OUT_OF_BOX);  // non-finite or mis-sorted: never index the tile with it
        my_cell = inside ? tile_index<R>(tx, ty, tz) : -1;
      }
      __syncwarp();
      const int cnt = min(32, n - base);
      if constexpr (sizeof(R) == 4) {
        p2g_walk_f32<MODE>(wrec, tile, my_cell, cnt, lane, qi, qj, qk, col);
      } else {
        R acc[2][NCH];
#pragma unroll
        for (int x = 0; x < 2; ++x)
#pragma unroll
          for (int c = 0; c < NCH; ++c) acc[x][c] = R(0);
        auto flush = [&](int at) {
#pragma unroll
          for (int x = 0; x < 2; ++x)
#pragma unroll
            for (int c = 0; c < NCH; ++c) {
              if (c == 0 && !kMass) continue;
              if (c >= 1 && c <= 3 && !kMom) continue;
              atomicAdd(&tile[c * TileShape<R>::N + at + col + qi + 2 * x], acc[x][c]);
              acc[x][c] = R(0);
            }
        };
        // Walk the runs of equal cells (the particles arrive cell-sorted): the
        // run boundaries come from one ballot, so the inner loop carries no
        // per-particle cell test.
        auto add = [&](int qq) {
          const R* rr = wrec + qq * kRec;
          using R2 = typename Vec<R>::two;
          const R2 py = *reinterpret_cast<const R2*>(rr + RW_Y + 2 * qj);
          const R2 pz = *reinterpret_cast<const R2*>(rr + RW_Z + 2 * qk);
          const R A = py.x * pz.x;
          R P[4], U[3], V[3];
          {
            const R2 mm0 = *reinterpret_cast<const R2*>(rr + R_M);      // m, m v_x
            const R2 mm1 = *reinterpret_cast<const R2*>(rr + R_M + 2);  // m v_y, m v_z
            P[0] = A * mm0.x;
            P[1] = A * mm0.y;
            P[2] = A * mm1.x;
            P[3] = A * mm1.y;
          }
          if constexpr (kForce) {
            const R2 f0 = *reinterpret_cast<const R2*>(rr + R_F);      // xx, yy
            const R2 f1 = *reinterpret_cast<const R2*>(rr + R_F + 2);  // zz, xy
            const R2 f2 = *reinterpret_cast<const R2*>(rr + R_F + 4);  // xz, yz
            const R B = py.y * pz.x, C = py.x * pz.y;
            const R mxx = f0.x, myy = f0.y, mzz = f1.x, mxy = f1.y, mxz = f2.x, myz = f2.y;
            U[0] = A * mxx;
            U[1] = A * mxy;
            U[2] = A * mxz;
            V[0] = B * mxy + C * mxz;
            V[1] = B * myy + C * myz;
            V[2] = B * myz + C * mzz;
          }
#pragma unroll
          for (int x = 0; x < 2; ++x) {
            const R2 px = *reinterpret_cast<const R2*>(rr + RW_X + 2 * (qi + 2 * x));
            const R wxv = px.x, dwx = px.y;
            if constexpr (kMass) acc[x][0] += wxv * P[0];
            if constexpr (kMom) {
              acc[x][1] += wxv * P[1];
              acc[x][2] += wxv * P[2];
              acc[x][3] += wxv * P[3];
            }
            if constexpr (kForce) {
              acc[x][4] += dwx * U[0] + wxv * V[0];
              acc[x][5] += dwx * U[1] + wxv * V[1];
              acc[x][6] += dwx * U[2] + wxv * V[2];
            }
          }
        };
        const int prev = __shfl_up_sync(0xffffffffu, my_cell, 1);
        unsigned starts = __ballot_sync(0xffffffffu, lane < cnt && (lane == 0 || my_cell != prev));
        while (starts) {
          const int s0 = __ffs(starts) - 1;
          starts &= starts - 1;
          const int e0 = starts ? __ffs(starts) - 1 : cnt;
          const int cell = __shfl_sync(0xffffffffu, my_cell, s0);
          if (cell < 0) continue;  // particles outside the tile (flagged above)
          int qq = s0;
          for (; qq + 1 < e0; qq += 2) {
            add(qq);
            add(qq + 1);
          }
          if (qq < e0) add(qq);
          flush(cell);
        }
      }
      __syncwarp();
    }
    __syncthreads();
    // Flush: one global atomic per touched node and channel, clearing the
    // tile as it goes.
    for (int e = threadIdx.x; e < 8 * 64; e += blockDim.x) {
      const int d = e >> 6, node = e & 63;
      int t;
      if (!tile_of<R>(d, node, t)) continue;
      const int32_t nb = h.nbr[d];
      R v[NCH];
      bool any = false;
#pragma unroll
      for (int ch = 0; ch < NCH; ++ch) {
        v[ch] = tile[ch * TileShape<R>::N + t];
        any |= v[ch] != R(0);
      }
      if (!any) continue;
#pragma unroll
      for (int ch = 0; ch < NCH; ++ch) tile[ch * TileShape<R>::N + t] = R(0);
      if (nb < 0) continue;
      const int64_t g = (int64_t)nb * 64 + node;
#pragma unroll
      for (int ch = 0; ch < NCH; ++ch)
        if (v[ch] != R(0)) atomicAdd(&acc_g[ch * plane + g], v[ch]);
    }
  }
}

// ------------------------------------------------------------- grid update
template <typename R>
__global__ void __launch_bounds__(256) k_grid_update(const BatchDev b) {
  R* acc = (R*)b.acc;
  R* vel = (R*)b.vel;
  const int64_t plane = (int64_t)b.cap_blocks * 64;
  const int64_t work = (int64_t)num_blocks(b) * 64;
  for (int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; e < work;
       e += (int64_t)gridDim.x * blockDim.x) {
    const int64_t blk = e >> 6;
    const int node = (int)(e & 63);
    const int4 bc = b.blk[blk];
    const SceneDev& sc = b.scenes[bc.w];
    const R m = acc[e];
    R v[3] = {R(0), R(0), R(0)}, pm[3] = {R(0), R(0), R(0)};
    {
      const R p[3] = {acc[plane + e], acc[2 * plane + e], acc[3 * plane + e]};
      const R f[3] = {acc[4 * plane + e], acc[5 * plane + e], acc[6 * plane + e]};
      const R g[3] = {(R)sc.g[0], (R)sc.g[1], (R)sc.g[2]};
      node_velocity(m, p, f, g, (R)sc.dt, v, pm);
    }
    const R dx = (R)sc.dx;
    const R px = dx * (R)(4 * bc.x + (node & 3));
    const R py = dx * (R)(4 * bc.y + ((node >> 2) & 3));
    const R pz = dx * (R)(4 * bc.z + (node >> 4));
    for (int c = 0; c < sc.coll_count; ++c) collide(b.colliders[sc.coll_begin + c], px, py, pz, v[0], v[1], v[2]);
    const bool later = b.imp_mass != nullptr;  // the implicit solve finishes the FLIP channels
    if (later) reinterpret_cast<R*>(b.imp_mass)[e] = m;
#pragma unroll
    for (int a = 0; a < 3; ++a) {
      vel[a * plane + e] = v[a];
      vel[(3 + a) * plane + e] = m > R(0) ? (later ? -pm[a] : v[a] - pm[a]) : R(0);
    }
#pragma unroll
    for (int ch = 0; ch < kAccCh; ++ch) acc[ch * plane + e] = R(0);
  }
}

template <typename R>
__global__ void __launch_bounds__(256) k_zero_grid(const BatchDev b) {
  R* acc = (R*)b.acc;
  const int64_t plane = (int64_t)b.cap_blocks * 64;
  const int64_t work = (int64_t)num_blocks(b) * 64;
  for (int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; e < work;
       e += (int64_t)gridDim.x * blockDim.x)
    for (int ch = 0; ch < kAccCh; ++ch) acc[ch * plane + e] = R(0);
}

// --------------------------------------------------------------------- G2P
template <int MODE>
struct G2PChannels {
  static constexpr int n = MODE == G2P_VOLUME ? 1 : (MODE == G2P_STRESS ? 3 : 6);
};

// Flushes a CTA's running block box of one scene (warp-reduced, then atomics
// that are skipped when they cannot improve the stored box).
__device__ __forceinline__ void flush_box(SceneDev& ps, int bmin[3], int bmax[3]) {
  int lo[3], hi[3];
  for (int a = 0; a < 3; ++a) {
    lo[a] = __reduce_min_sync(0xffffffffu, bmin[a]);
    hi[a] = __reduce_max_sync(0xffffffffu, bmax[a]);
    bmin[a] = INT_MAX;
    bmax[a] = INT_MIN;
  }
  if ((threadIdx.x & 31) == 0) box_update(ps, lo, hi);
}

// Next step's force matrix from the projected F_E, the square root returned by
// plastic_projection and the new F_P (hardening in double).
// Elastoplastic projection in the batch's precision.  In the mixed form the
// float eigensolve is redone in double when a singular value lies within
// kMixedTau of a clamp bound, or a clamp acts on two singular values within
// kMixedTau of each other (used_fp64 = true; see near_critical).
constexpr float kMixedTau = 1e-5f;

// Both precisions first try the elastic fast path (elastic_projection: no
// clamp within a margin, root from the polar factor); particles near or past a
// clamp bound take the eigensolve as before.
constexpr double kElasticMargin = 1e-12;

template <typename R>
__device__ __forceinline__ Plastic<R> project(M3<R>& FE, const SceneDev& sc, bool& used_fp64) {
  if constexpr (std::is_same<R, double>::value) {
    const double lo = 1.0 - sc.theta_c, hi = 1.0 + sc.theta_s;
    Plastic<double> fast;
    if (elastic_projection(FE, lo, hi, kElasticMargin, fast)) return fast;
    return plastic_projection(FE, lo, hi);
  } else {
    const M3<float> trial = FE;
    const float lo = 1.0f - (float)sc.theta_c, hi = 1.0f + (float)sc.theta_s;
    Plastic<float> fast;
    if (elastic_projection(FE, lo, hi, kMixedTau, fast)) return fast;
    Plastic<float> pl = plastic_projection(FE, lo, hi);
    if (!near_critical(pl.sigma, lo, hi, kMixedTau, pl.clamped)) return pl;
    used_fp64 = true;
    M3<double> Fd;
#pragma unroll
    for (int e = 0; e < 9; ++e) Fd.a[e] = (double)trial.a[e];
    const Plastic<double> pd = plastic_projection(Fd, 1.0 - sc.theta_c, 1.0 + sc.theta_s);
#pragma unroll
    for (int e = 0; e < 9; ++e) FE.a[e] = (float)Fd.a[e];
    pl.Dinv = Sym3<float>{(float)pd.Dinv.xx, (float)pd.Dinv.yy, (float)pd.Dinv.zz,
                          (float)pd.Dinv.xy, (float)pd.Dinv.xz, (float)pd.Dinv.yz};
    pl.root = Sym3<float>{(float)pd.root.xx, (float)pd.root.yy, (float)pd.root.zz,
                          (float)pd.root.xy, (float)pd.root.xz, (float)pd.root.yz};
#pragma unroll
    for (int i = 0; i < 3; ++i) pl.sigma[i] = (float)pd.sigma[i];
    pl.clamped = pd.clamped;
    pl.regular = pd.regular;
    return pl;
  }
}

template <typename R>
__device__ __forceinline__ Sym3<R> next_force(const M3<R>& FE, const Plastic<R>& pl, const M3<double>& FP,
                                              const SceneDev& sc, R V0) {
  const double hard = exp(sc.xi * (1.0 - det3(FP)));
  if (!pl.regular) return force_matrix<R>(FE, V0, (R)sc.mu0, (R)sc.lambda0, (R)hard);
  return assemble_force<R>(gram_rows(FE), pl.root, det3(FE), V0, (R)sc.mu0, (R)sc.lambda0, (R)hard);
}

// Node-major G2P tile: the channels of one node are adjacent, so a full-mode
// gather reads each node with two 16-byte loads in float (6 channels padded to
// 8) and three in double.
template <typename R, int MODE>
struct G2PTile {
  static constexpr int NCH = G2PChannels<MODE>::n;
  static constexpr int NS = NCH == 6 ? (sizeof(R) == 4 ? 8 : 6) : NCH;  // node stride
  static constexpr int size() { return TileShape<R>::N * NS; }
};

template <typename R, int MODE>
__device__ __forceinline__ void load_node(const R* tile, int t, R (&f)[G2PChannels<MODE>::n]) {
  using T = G2PTile<R, MODE>;
  const R* p = tile + t * T::NS;
  if constexpr (T::NCH == 6 && sizeof(R) == 4) {
    const float4 a = *reinterpret_cast<const float4*>(p);
    const float2 c = *reinterpret_cast<const float2*>(p + 4);
    f[0] = a.x, f[1] = a.y, f[2] = a.z, f[3] = a.w, f[4] = c.x, f[5] = c.y;
  } else if constexpr (T::NCH == 6) {
#pragma unroll
    for (int k = 0; k < 3; ++k) {
      const double2 a = *reinterpret_cast<const double2*>(p + 2 * k);
      f[2 * k] = a.x;
      f[2 * k + 1] = a.y;
    }
  } else {
#pragma unroll
    for (int ch = 0; ch < T::NCH; ++ch) f[ch] = p[ch];
  }
}

// Asynchronous global -> shared copies (cp.async): issued per thread, waited
// for by the same thread, so they need no barrier.
__device__ __forceinline__ void cp_async(void* sdst, const void* gsrc, int bytes_4_or_8) {
  const unsigned d = (unsigned)__cvta_generic_to_shared(sdst);
  if (bytes_4_or_8 == 8)
    asm volatile("cp.async.ca.shared.global [%0], [%1], 8;\n" ::"r"(d), "l"(gsrc) : "memory");
  else
    asm volatile("cp.async.ca.shared.global [%0], [%1], 4;\n" ::"r"(d), "l"(gsrc) : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::: "memory"); }
__device__ __forceinline__ void cp_async_wait_all() { asm volatile("cp.async.wait_all;\n" ::: "memory"); }

// Full-mode G2P: the particle state the update reads after the gather (F_E,
// F_P, v, m, V_p0, id) is copied into per-thread shared slots as soon as the
// particle's index is known, so its load latency overlaps the gather.
constexpr int kG2PThreads = 256;
template <typename R>
struct G2PSlots {
  double fp[9][kG2PThreads];
  R fe[9][kG2PThreads];
  R v[3][kG2PThreads];
  R m[kG2PThreads];
  R v0[kG2PThreads];
  int32_t id[kG2PThreads];
};

// Full-mode gather in float: a node's 6 channels as three pairs, accumulated
// with the packed two-wide FMA of sm_100 (__ffma2_rn: two fmaf in one
// instruction, same rounding), contracted z, then y, then x as in the generic
// path.  Outputs: grad v (column-major), v_pic, and the FLIP term.
__device__ __forceinline__ float2 splat(float a) { return make_float2(a, a); }

__device__ __forceinline__ void gather_f32(const float* tile, int t0, const AxisWeights<float>& wx,
                                           const AxisWeights<float>& wy, const AxisWeights<float>& wz,
                                           float gv[9], float vpic[3], float dflip[3]) {
  constexpr int Y = TileShape<float>::Y, Z = TileShape<float>::Z;
  float2 wz2[4], dwz2[4];
#pragma unroll
  for (int e = 0; e < 4; ++e) {
    wz2[e] = splat(wz.w[e]);
    dwz2[e] = splat(wz.dw[e]);
  }
  const float2 zero = make_float2(0.f, 0.f);
  float2 vp01 = zero, g01 = zero, gy01 = zero, gz01 = zero, df12 = zero;
  float vp2 = 0.f, df0 = 0.f, g2 = 0.f, gy2 = 0.f, gz2 = 0.f;
#pragma unroll
  for (int a = 0; a < 4; ++a) {
    float2 SS01 = zero, SS23 = zero, SS45 = zero, SD01 = zero, TS01 = zero;
    float SD2 = 0.f, TS2 = 0.f;
#pragma unroll
    for (int c = 0; c < 4; ++c) {
      float2 S01 = zero, S23 = zero, S45 = zero, T01 = zero;
      float T2 = 0.f;
#pragma unroll
      for (int e = 0; e < 4; ++e) {
        const float* p = tile + (t0 + a + Y * c + Z * e) * 8;
        const float4 q = *reinterpret_cast<const float4*>(p);
        const float2 f45 = *reinterpret_cast<const float2*>(p + 4);
        const float2 f01 = make_float2(q.x, q.y), f23 = make_float2(q.z, q.w);
        S01 = __ffma2_rn(wz2[e], f01, S01);
        S23 = __ffma2_rn(wz2[e], f23, S23);
        S45 = __ffma2_rn(wz2[e], f45, S45);
        T01 = __ffma2_rn(dwz2[e], f01, T01);
        T2 = fmaf(wz.dw[e], q.z, T2);
      }
      const float2 wy2 = splat(wy.w[c]), dwy2 = splat(wy.dw[c]);
      SS01 = __ffma2_rn(wy2, S01, SS01);
      SS23 = __ffma2_rn(wy2, S23, SS23);
      SS45 = __ffma2_rn(wy2, S45, SS45);
      SD01 = __ffma2_rn(dwy2, S01, SD01);
      SD2 = fmaf(wy.dw[c], S23.x, SD2);
      TS01 = __ffma2_rn(wy2, T01, TS01);
      TS2 = fmaf(wy.w[c], T2, TS2);
    }
    const float2 wx2 = splat(wx.w[a]), dwx2 = splat(wx.dw[a]);
    vp01 = __ffma2_rn(wx2, SS01, vp01);
    vp2 = fmaf(wx.w[a], SS23.x, vp2);
    df0 = fmaf(wx.w[a], SS23.y, df0);
    df12 = __ffma2_rn(wx2, SS45, df12);
    g01 = __ffma2_rn(dwx2, SS01, g01);
    g2 = fmaf(wx.dw[a], SS23.x, g2);
    gy01 = __ffma2_rn(wx2, SD01, gy01);
    gy2 = fmaf(wx.w[a], SD2, gy2);
    gz01 = __ffma2_rn(wx2, TS01, gz01);
    gz2 = fmaf(wx.w[a], TS2, gz2);
  }
  vpic[0] = vp01.x, vpic[1] = vp01.y, vpic[2] = vp2;
  dflip[0] = df0, dflip[1] = df12.x, dflip[2] = df12.y;
  gv[0] = g01.x, gv[1] = g01.y, gv[2] = g2;
  gv[3] = gy01.x, gv[4] = gy01.y, gv[5] = gy2;
  gv[6] = gz01.x, gv[7] = gz01.y, gv[8] = gz2;
}

template <typename R, int MODE>
__global__ void __launch_bounds__(256, sizeof(R) == 4 ? 3 : 2) k_g2p(const BatchDev b) {
  constexpr int NCH = G2PChannels<MODE>::n;
  constexpr int NS = G2PTile<R, MODE>::NS;
  constexpr bool kGrad = MODE == G2P_FULL || MODE == G2P_STRESS;
  constexpr bool kVel = MODE == G2P_FULL || MODE == G2P_VELOCITY;
  constexpr bool kDeferDouble = MODE == G2P_FULL && !std::is_same<R, double>::value;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  R* tile = reinterpret_cast<R*>(smem_raw);  // [TileShape<R>::N][NS]
  G2PSlots<R>* slot = reinterpret_cast<G2PSlots<R>*>(smem_raw + sizeof(R) * G2PTile<R, MODE>::size());
  const int me = threadIdx.x;
  __shared__ BlockHeader h;
  const R* vel = (const R*)b.vel;
  const R* acc = (const R*)b.acc;
  const int64_t plane = (int64_t)b.cap_blocks * 64;
  int bmin[3] = {INT_MAX, INT_MAX, INT_MAX}, bmax[3] = {INT_MIN, INT_MIN, INT_MIN};
  int last_scene = -1;
  // write the next step's sort keys and bin counts (see k_keyspace)
  const bool emit = MODE == G2P_FULL && b.dense && b.ctr->emit_ok;

  __shared__ int s_item;
  ItemQueue q;
  q.fetch(b, &b.ctr->work_g2p, min(b.ctr->n_items, (uint32_t)b.cap_items));
  while (q.claim(b, &b.ctr->work_g2p, h, s_item)) {
    // Stage the 7x7x7 nodes this block's stencils read.
    for (int e = threadIdx.x; e < 8 * 64; e += blockDim.x) {
      const int d = e >> 6, node = e & 63;
      int t;
      if (!tile_of<R>(d, node, t)) continue;
      const int32_t nb = h.nbr[d];
      const int64_t g = (int64_t)(nb < 0 ? 0 : nb) * 64 + node;
      R v[NCH];
#pragma unroll
      for (int ch = 0; ch < NCH; ++ch) {
        if constexpr (MODE == G2P_VOLUME) v[ch] = acc[g];
        else v[ch] = vel[ch * plane + g];
        if (nb < 0) v[ch] = R(0);
      }
      R* dst = tile + t * NS;
      if constexpr (NCH == 6 && sizeof(R) == 4) {
        reinterpret_cast<float4*>(dst)[0] = make_float4(v[0], v[1], v[2], v[3]);
        reinterpret_cast<float2*>(dst)[2] = make_float2(v[4], v[5]);
      } else if constexpr (NCH == 6) {
#pragma unroll
        for (int k = 0; k < 3; ++k) reinterpret_cast<double2*>(dst)[k] = make_double2(v[2 * k], v[2 * k + 1]);
      } else {
#pragma unroll
        for (int ch = 0; ch < NCH; ++ch) dst[ch] = v[ch];
      }
    }
    __syncthreads();
    const int s = h.scene;
    if (MODE == G2P_FULL && s != last_scene) {
      if (last_scene >= 0) flush_box(b.scenes[last_scene], bmin, bmax);
      last_scene = s;
    }
    const SceneDev& sc = b.scenes[s];
    const R dx = (R)sc.dx;
    const int cur = sc.cur;
    const PlaneView<R> pv{(const R*)sc.r[cur], sc.fp[cur], sc.id[cur], sc.stride};
    const uint32_t* vals = sorted_vals(b);
    const int n = h.end - h.start;
    for (int k = threadIdx.x; k < n; k += blockDim.x) {
      const int j = h.start + k;
      const int64_t i = vals[j];
      if constexpr (MODE == G2P_FULL) {
        cp_async_wait_all();  // this thread's slot is free again
        constexpr int rb = (int)sizeof(R);
#pragma unroll
        for (int e = 0; e < 9; ++e) {
          cp_async(&slot->fe[e][me], pv.r + (PFE + e) * pv.st + i, rb);
          cp_async(&slot->fp[e][me], pv.fp + e * pv.st + i, 8);
        }
#pragma unroll
        for (int a = 0; a < 3; ++a) cp_async(&slot->v[a][me], pv.r + (PV + a) * pv.st + i, rb);
        cp_async(&slot->m[me], pv.r + PM * pv.st + i, rb);
        cp_async(&slot->v0[me], pv.r + PVOL * pv.st + i, rb);
        cp_async(&slot->id[me], pv.id + i, 4);
        cp_async_commit();
      }
      R x[3];
#pragma unroll
      for (int a = 0; a < 3; ++a) x[a] = pv.at(PX + a, i);
      const AxisWeights<R> wx = axis_weights(x[0], dx), wy = axis_weights(x[1], dx), wz = axis_weights(x[2], dx);
      const int tx = wx.base - 4 * h.bx, ty = wy.base - 4 * h.by, tz = wz.base - 4 * h.bz;
      if ((unsigned)tx > 3u || (unsigned)ty > 3u || (unsigned)tz > 3u) {
        flag(b, ST_OUT_OF_BOX);  // non-finite or mis-sorted particle: never index the tile with it
        if (emit) atomicOr(&b.ctr->emit_fail, 1u);  // and no key of it for the next step
        continue;
      }

      if constexpr (MODE == G2P_VOLUME) {
        // calculate_volume (grid.cpp:138-160)
        const double dx3 = pow((double)sc.dx, 3.0);
        R density = R(0);
#pragma unroll
        for (int a = 0; a < 4; ++a)
#pragma unroll
          for (int c = 0; c < 4; ++c)
#pragma unroll
            for (int e = 0; e < 4; ++e) {
              const R w = wx.w[a] * wy.w[c] * wz.w[e];
              density += (tile[tile_index<R>(tx + a, ty + c, tz + e) * NS] * w) / (R)dx3;
            }
        R* rw = (R*)sc.r[cur];
        rw[PVOL * sc.stride + i] = pv.at(PM, i) / density;
        continue;
      } else {
        // grad v = sum_n v_n (grad w_n)^T, v_pic = sum_n w_n v_n, FLIP term = sum_n w_n dv_n
        // (grid.cpp:250-276, 295-319), contracted one axis at a time: z, then y, then x.
        R gv[9] = {R(0), R(0), R(0), R(0), R(0), R(0), R(0), R(0), R(0)};  // column-major
        R vpic[3] = {R(0), R(0), R(0)}, dflip[3] = {R(0), R(0), R(0)};
        if constexpr (std::is_same<R, float>::value && NCH == 6) {
          gather_f32(tile, tile_index<R>(tx, ty, tz), wx, wy, wz, gv, vpic, dflip);
        } else {
#pragma unroll
        for (int a = 0; a < 4; ++a) {
          R SS[NCH], SD[3], TS[3];
#pragma unroll
          for (int ch = 0; ch < NCH; ++ch) SS[ch] = R(0);
#pragma unroll
          for (int ch = 0; ch < 3; ++ch) SD[ch] = TS[ch] = R(0);
#pragma unroll
          for (int c = 0; c < 4; ++c) {
            R S[NCH], T[3];
#pragma unroll
            for (int ch = 0; ch < NCH; ++ch) S[ch] = R(0);
#pragma unroll
            for (int ch = 0; ch < 3; ++ch) T[ch] = R(0);
#pragma unroll
            for (int e = 0; e < 4; ++e) {
              R f[NCH];
              load_node<R, MODE>(tile, tile_index<R>(tx + a, ty + c, tz + e), f);
#pragma unroll
              for (int ch = 0; ch < NCH; ++ch) {
                S[ch] += wz.w[e] * f[ch];
                if (kGrad && ch < 3) T[ch] += wz.dw[e] * f[ch];
              }
            }
#pragma unroll
            for (int ch = 0; ch < NCH; ++ch) SS[ch] += wy.w[c] * S[ch];
            if constexpr (kGrad) {
#pragma unroll
              for (int ch = 0; ch < 3; ++ch) {
                SD[ch] += wy.dw[c] * S[ch];
                TS[ch] += wy.w[c] * T[ch];
              }
            }
          }
          if constexpr (kVel) {
#pragma unroll
            for (int ch = 0; ch < 3; ++ch) {
              vpic[ch] += wx.w[a] * SS[ch];
              dflip[ch] += wx.w[a] * SS[3 + ch];
            }
          }
          if constexpr (kGrad) {
#pragma unroll
            for (int r = 0; r < 3; ++r) {
              gv[r] += wx.dw[a] * SS[r];
              gv[3 + r] += wx.w[a] * SD[r];
              gv[6 + r] += wx.w[a] * TS[r];
            }
          }
        }
        }
        const R dt = (R)sc.dt;
        if constexpr (MODE == G2P_FULL) cp_async_wait_all();
        R vn[3];
        if constexpr (kVel) {
          // G2P (grid.cpp:321-324)
          const R alpha = (R)sc.alpha;
#pragma unroll
          for (int a = 0; a < 3; ++a) {
            const R vflip = (MODE == G2P_FULL ? slot->v[a][me] : pv.at(PV + a, i)) + dflip[a];
            vn[a] = (R(1) - alpha) * vpic[a] + alpha * vflip;
          }
        }
        if constexpr (MODE == G2P_VELOCITY) {
          R* rw = (R*)sc.r[cur];
#pragma unroll
          for (int a = 0; a < 3; ++a) rw[(PV + a) * sc.stride + i] = vn[a];
          continue;
        }
        const int64_t o = j - sc.begin;  // block-sorted slot in the other buffer
        const int64_t st = sc.stride;
        R V0 = R(0);
        if constexpr (MODE == G2P_FULL) {
          // particle_collisions (grid.cpp:327-333), position_update (grid.cpp:335-338);
          // the kinematic part of the new state is written before the stress
          // update so that its registers are free for the projection
          for (int c = 0; c < sc.coll_count; ++c)
            collide(b.colliders[sc.coll_begin + c], x[0], x[1], x[2], vn[0], vn[1], vn[2]);
          R* rw = (R*)sc.r[cur ^ 1];
          int nblk[3], ncell[3];
          bool finite = true;
#pragma unroll
          for (int a = 0; a < 3; ++a) {
            const R xn = x[a] + dt * vn[a];
            rw[(PX + a) * st + o] = xn;
            rw[(PV + a) * st + o] = vn[a];
            nblk[a] = ncell[a] = 0;
            if (isfinite((double)xn)) {
              nblk[a] = block_coord(xn, dx, ncell[a]);
              bmin[a] = min(bmin[a], nblk[a]);
              bmax[a] = max(bmax[a], nblk[a]);
            } else {
              finite = false;
              flag(b, ST_NONFINITE);
            }
          }
          if (emit) {
            // the next step's sort key against the scene's emission box, as
            // k_keys would compute it, and its bin count (one atomic per key
            // among the warp's lanes: neighbouring particles share cells)
            bool ok = finite;
#pragma unroll
            for (int a = 0; a < 3; ++a) ok &= nblk[a] >= sc.elo[a] && nblk[a] <= sc.elo[a] + sc.edim[a] - 2;
            uint32_t key = 0xFFFFFFFFu;
            if (ok) {
              const uint32_t bk =
                  sc.ekey_base + (uint32_t)(((int64_t)(nblk[2] - sc.elo[2]) * sc.edim[1] + (nblk[1] - sc.elo[1])) *
                                                sc.edim[0] +
                                            (nblk[0] - sc.elo[0]));
              key = (bk << 6) | (uint32_t)(ncell[0] + 4 * ncell[1] + 16 * ncell[2]);
              b.keys[0][j] = key;
              b.vals[0][j] = (uint32_t)o;
            } else {
              atomicOr(&b.ctr->emit_fail, 1u);
            }
            const unsigned same = __match_any_sync(__activemask(), key);
            if (ok && (threadIdx.x & 31) == __ffs(same) - 1) {
              atomicAdd(&b.bins[key], (uint32_t)__popc(same));
              b.occ[key >> 6] = 1;
            }
          }
          V0 = slot->v0[me];
          rw[PM * st + o] = slot->m[me];
          rw[PVOL * st + o] = V0;
          sc.id[cur ^ 1][o] = slot->id[me];
        }
        // stress_update (grid.cpp:277-285)
        M3<R> FEn, trial;
        M3<double> FPn;
        Plastic<R> pl;
        bool needs_double = false;
        (void)trial;
        {
          M3<R> FE, L;
#pragma unroll
          for (int e = 0; e < 9; ++e) {
            FE.a[e] = MODE == G2P_FULL ? slot->fe[e][me] : pv.at(PFE + e, i);
            L.a[e] = dt * gv[e];
          }
          L.a[0] += R(1);
          L.a[4] += R(1);
          L.a[8] += R(1);
          FEn = mat_mul(L, FE);
        }
        if constexpr (kDeferDouble) {
          // Mixed form: a projection that needs double is redone by k_fixup
          // from the trial F_E, which is kept for it in the output slot.
          trial = FEn;
          const R lo = R(1) - (R)sc.theta_c, hi = R(1) + (R)sc.theta_s;
          if (!elastic_projection(FEn, lo, hi, (R)kMixedTau, pl)) {
            pl = plastic_projection(FEn, lo, hi);
            needs_double = near_critical(pl.sigma, lo, hi, (R)kMixedTau, pl.clamped);
          }
        } else {
          bool used_fp64 = false;
          pl = project(FEn, sc, used_fp64);
          if constexpr (!std::is_same<R, double>::value) {
            const unsigned act = __activemask();
            const unsigned fb = __ballot_sync(act, used_fp64);
            if (fb && (threadIdx.x & 31) == __ffs(act) - 1) atomicAdd(&b.ctr->fp64_projections, (uint32_t)__popc(fb));
          }
        }
#pragma unroll
        for (int e = 0; e < 9; ++e) FPn.a[e] = MODE == G2P_FULL ? slot->fp[e][me] : pv.fp[e * pv.st + i];
        if (pl.clamped) sym_mul_inplace(pl.Dinv, FPn);
        if constexpr (MODE == G2P_STRESS) {
          R* rw = (R*)sc.r[cur];
          double* fw = sc.fp[cur];
#pragma unroll
          for (int e = 0; e < 9; ++e) {
            rw[(PFE + e) * sc.stride + i] = FEn.a[e];
            fw[e * sc.stride + i] = FPn.a[e];
          }
          continue;
        }
        if constexpr (MODE == G2P_FULL) {
          const Sym3<R> Mn = next_force(FEn, pl, FPn, sc, V0);
          R* rw = (R*)sc.r[cur ^ 1];
          double* fw = sc.fp[cur ^ 1];
#pragma unroll
          for (int e = 0; e < 9; ++e) {
            rw[(PFE + e) * st + o] = needs_double ? trial.a[e] : FEn.a[e];
            fw[e * st + o] = FPn.a[e];
          }
          if constexpr (kDeferDouble) {
            const unsigned act = __activemask();
            const unsigned fb = __ballot_sync(act, needs_double);
            if (fb) {
              const int lane = threadIdx.x & 31, leader = __ffs(act) - 1;
              uint32_t base = 0;
              if (lane == leader) base = atomicAdd(&b.ctr->fp64_projections, (uint32_t)__popc(fb));
              base = __shfl_sync(act, base, leader);
              if (needs_double) {
                const uint32_t slot = base + __popc(fb & ((1u << lane) - 1u));
                if (slot < (uint32_t)b.cap_fixups) b.fixups[slot] = make_int4(s, (int)o, (int)i, 0);
                else flag(b, ST_BLOCK_OVERFLOW);
              }
            }
          }
          rw[(PFM + 0) * st + o] = Mn.xx;
          rw[(PFM + 1) * st + o] = Mn.yy;
          rw[(PFM + 2) * st + o] = Mn.zz;
          rw[(PFM + 3) * st + o] = Mn.xy;
          rw[(PFM + 4) * st + o] = Mn.xz;
          rw[(PFM + 5) * st + o] = Mn.yz;
        }
      }
    }
  }
  if constexpr (MODE == G2P_FULL) cp_async_wait_all();
  if (MODE == G2P_FULL && last_scene >= 0) flush_box(b.scenes[last_scene], bmin, bmax);
}

// Mixed form: the plastic projections G2P flagged as near-critical, redone in
// double from the trial F_E it left in the output slot, with the new F_P and
// the next force matrix (runs after G2P, before the buffers swap).
__global__ void __launch_bounds__(256) k_fixup(const BatchDev b) {
  const uint32_t n = min(b.ctr->fp64_projections, (uint32_t)b.cap_fixups);
  for (uint32_t e = blockIdx.x * blockDim.x + threadIdx.x; e < n; e += gridDim.x * blockDim.x) {
    const int4 f = b.fixups[e];
    const SceneDev& sc = b.scenes[f.x];
    const int cur = sc.cur;
    float* rw = (float*)sc.r[cur ^ 1];
    double* fw = sc.fp[cur ^ 1];
    const double* fp_old = sc.fp[cur];
    const int64_t st = sc.stride, o = f.y, i = f.z;
    M3<double> F, FP;
#pragma unroll
    for (int k = 0; k < 9; ++k) {
      F.a[k] = (double)rw[(PFE + k) * st + o];
      FP.a[k] = fp_old[k * st + i];
    }
    const Plastic<double> pl = plastic_projection(F, 1.0 - sc.theta_c, 1.0 + sc.theta_s);
    if (pl.clamped) sym_mul_inplace(pl.Dinv, FP);
    const double hard = exp(sc.xi * (1.0 - det3(FP)));
    const double V0 = (double)rw[PVOL * st + o];
    const Sym3<double> M = pl.regular
                               ? assemble_force(gram_rows(F), pl.root, det3(F), V0, sc.mu0, sc.lambda0, hard)
                               : force_matrix(F, V0, sc.mu0, sc.lambda0, hard);
#pragma unroll
    for (int k = 0; k < 9; ++k) {
      rw[(PFE + k) * st + o] = (float)F.a[k];
      fw[k * st + o] = FP.a[k];
    }
    rw[(PFM + 0) * st + o] = (float)M.xx;
    rw[(PFM + 1) * st + o] = (float)M.yy;
    rw[(PFM + 2) * st + o] = (float)M.zz;
    rw[(PFM + 3) * st + o] = (float)M.xy;
    rw[(PFM + 4) * st + o] = (float)M.xz;
    rw[(PFM + 5) * st + o] = (float)M.yz;
  }
}

// Force matrix of every particle from its F_E, F_P and V_p0 (after an upload,
// setup() or a parameter change; afterwards G2P keeps it current).
template <typename R>
__global__ void __launch_bounds__(256) k_prepare_force(const BatchDev b) {
  const int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= b.total) return;
  const SceneDev& sc = b.scenes[scene_of(b, t)];
  const int64_t i = t - sc.begin;
  R* r = (R*)sc.r[sc.cur];
  const double* fp = sc.fp[sc.cur];
  const int64_t st = sc.stride;
  M3<R> FE;
#pragma unroll
  for (int e = 0; e < 9; ++e) FE.a[e] = r[(PFE + e) * st + i];
  M3<double> FP;
#pragma unroll
  for (int e = 0; e < 9; ++e) FP.a[e] = fp[e * st + i];
  const double hard = exp(sc.xi * (1.0 - det3(FP)));
  const Sym3<R> M = force_matrix<R>(FE, r[PVOL * st + i], (R)sc.mu0, (R)sc.lambda0, (R)hard);
  r[(PFM + 0) * st + i] = M.xx;
  r[(PFM + 1) * st + i] = M.yy;
  r[(PFM + 2) * st + i] = M.zz;
  r[(PFM + 3) * st + i] = M.xy;
  r[(PFM + 4) * st + i] = M.xz;
  r[(PFM + 5) * st + i] = M.yz;
}

__global__ void k_finish(const BatchDev b) {
  for (int s = threadIdx.x; s < b.num_scenes; s += blockDim.x) b.scenes[s].cur ^= 1;
}

// ------------------------------------------------------------ launch helpers
// Launch settings that depend on the device (SM count, the occupancy of a
// persistent kernel, a kernel's shared-memory attribute) are set up once per
// device and kept per device: a process may drive several GPUs, from several
// host threads.
constexpr int kMaxDevices = 64;

int current_device() {
  int dev = 0;
  check_cuda(cudaGetDevice(&dev), "cudaGetDevice");
  if (dev < 0 || dev >= kMaxDevices) throw Error(SNOW_E_ARG, "device index out of range");
  return dev;
}

struct PerDevice {
  std::atomic<int> v[kMaxDevices];
  PerDevice() {
    for (auto& x : v) x.store(0);
  }
  // The value for the current device, computed by `make` the first time
  // (two threads may both compute it; they store the same value).
  template <typename F>
  int get(F&& make) {
    std::atomic<int>& x = v[current_device()];
    int r = x.load(std::memory_order_acquire);
    if (!r) {
      r = make();
      x.store(r, std::memory_order_release);
    }
    return r;
  }
};

template <typename K>
int persistent_grid(K kernel, int threads, size_t smem) {
  int per_sm = 0;
  check_cuda(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kernel, threads, smem), "occupancy");
  if (per_sm < 1) per_sm = 1;
  return per_sm * sm_count();
}

template <typename K>
void set_smem(K kernel, size_t smem) {
  // always: without it static + dynamic shared memory is held to 48 KB
  if (smem > 0)
    check_cuda(cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem),
               "shared memory size");
}

}  // namespace

int sm_count() {
  static PerDevice count;
  return count.get([] {
    int n = 0;
    check_cuda(cudaDeviceGetAttribute(&n, cudaDevAttrMultiProcessorCount, current_device()), "SM count");
    return n > 0 ? n : 1;
  });
}

template <typename R>
void StepLaunch<R>::bbox_init(const BatchDev& b, cudaStream_t s) {
  if (b.total <= 0) return;
  k_bbox_init<R><<<(unsigned)((b.total + 255) / 256), 256, 0, s>>>(b);
}
template <typename R>
void StepLaunch<R>::keyspace(const BatchDev& b, cudaStream_t s, bool) {
  k_keyspace<false><<<1, kKeyspaceThreads, 0, s>>>(b);
}
template <typename R>
void StepLaunch<R>::keys(const BatchDev& b, cudaStream_t s) {
  if (b.total <= 0) return;
  // grid-stride: a few waves at most, so that the launch is short when the
  // previous step's G2P already wrote the keys
  const int64_t want = (b.total + 255) / 256;
  k_keys<R><<<(unsigned)std::min<int64_t>(want, 8 * (int64_t)sm_count()), 256, 0, s>>>(b);
}
template <typename R>
void StepLaunch<R>::blocks(const BatchDev& b, cudaStream_t s) {
  if (b.total <= 0) return;
  if (b.dense) {
    static PerDevice bins_grid;
    const int grid = bins_grid.get([] { return persistent_grid(k_bins, 256, 0); });
    const int64_t tiles = b.cap_bins / kBinTile;
    k_bins<<<(unsigned)std::min<int64_t>(grid, std::max<int64_t>(tiles, 1)), 256, 0, s>>>(b);
    k_scatter<<<(unsigned)((b.total + 255) / 256), 256, 0, s>>>(b);
    return;
  }
  check_cuda(cudaMemsetAsync(b.htab, 0xFF, sizeof(unsigned long long) * ((size_t)b.hmask + 1), s),
             "clear block table");
  k_blocks<<<(unsigned)((b.total + b.chunk - 1) / b.chunk), b.chunk, 0, s>>>(b);
}

template <typename R, int MODE>
static void launch_p2g(const BatchDev& b, cudaStream_t s) {
  const size_t smem = p2g_smem<R, MODE>();
  static PerDevice grids;
  const int grid = grids.get([&] {
    set_smem(k_p2g<R, MODE>, smem);
    return persistent_grid(k_p2g<R, MODE>, 256, smem);
  });
  k_p2g<R, MODE><<<grid, 256, smem, s>>>(b);
}
template <typename R>
void StepLaunch<R>::p2g(const BatchDev& b, int mode, cudaStream_t s) {
  if (b.total <= 0) return;
  switch (mode) {
    case P2G_FULL: launch_p2g<R, P2G_FULL>(b, s); break;
    case P2G_MASS: launch_p2g<R, P2G_MASS>(b, s); break;
    case P2G_MASS_MOMENTUM: launch_p2g<R, P2G_MASS_MOMENTUM>(b, s); break;
    case P2G_FORCE: launch_p2g<R, P2G_FORCE>(b, s); break;
    case P2G_PRE: launch_p2g<R, P2G_PRE>(b, s); break;
  }
}
template <typename R>
void StepLaunch<R>::grid_update(const BatchDev& b, cudaStream_t s) {
  if (b.total <= 0) return;
  static PerDevice grids;
  const int grid = grids.get([] { return persistent_grid(k_grid_update<R>, 256, 0); });
  k_grid_update<R><<<grid, 256, 0, s>>>(b);
}
template <typename R>
void StepLaunch<R>::zero_grid(const BatchDev& b, cudaStream_t s) {
  if (b.total <= 0) return;
  k_zero_grid<R><<<4 * sm_count(), 256, 0, s>>>(b);
}
template <typename R, int MODE>
static void launch_g2p(const BatchDev& b, cudaStream_t s) {
  const size_t smem = sizeof(R) * G2PTile<R, MODE>::size() + (MODE == G2P_FULL ? sizeof(G2PSlots<R>) : 0);
  static PerDevice grids;
  const int grid = grids.get([&] {
    set_smem(k_g2p<R, MODE>, smem);
    return persistent_grid(k_g2p<R, MODE>, 256, smem);
  });
  k_g2p<R, MODE><<<grid, 256, smem, s>>>(b);
}
template <typename R>
void StepLaunch<R>::g2p(const BatchDev& b, int mode, cudaStream_t s) {
  if (b.total <= 0) return;
  switch (mode) {
    case G2P_FULL: launch_g2p<R, G2P_FULL>(b, s); break;
    case G2P_VOLUME: launch_g2p<R, G2P_VOLUME>(b, s); break;
    case G2P_STRESS: launch_g2p<R, G2P_STRESS>(b, s); break;
    case G2P_VELOCITY: launch_g2p<R, G2P_VELOCITY>(b, s); break;
  }
}
template <typename R>
void StepLaunch<R>::fixup(const BatchDev& b, cudaStream_t s) {
  if (std::is_same<R, double>::value || b.total <= 0) return;
  k_fixup<<<2 * sm_count(), 256, 0, s>>>(b);
}
template <typename R>
void StepLaunch<R>::prepare_force(const BatchDev& b, cudaStream_t s) {
  if (b.total <= 0) return;
  k_prepare_force<R><<<(unsigned)((b.total + 255) / 256), 256, 0, s>>>(b);
}
template <typename R>
void StepLaunch<R>::finish(const BatchDev& b, cudaStream_t s) {
  k_finish<<<1, 256, 0, s>>>(b);
}
template <typename R>
void StepLaunch<R>::finish_and_keyspace(const BatchDev& b, cudaStream_t s) {
  k_keyspace<true><<<1, kKeyspaceThreads, 0, s>>>(b);
}

template struct StepLaunch<double>;
template struct StepLaunch<float>;

}  // namespace snow
