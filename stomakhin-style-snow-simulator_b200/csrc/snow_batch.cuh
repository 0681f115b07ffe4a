// Device-side data layout of a batch of independent snow scenes.
//
// Particles (per scene, double-buffered, structure of arrays):
//   real planes  r[k * stride + i], k = 0..22: x0 x1 x2, v0 v1 v2, m, V_p0,
//                F_E (9, column-major), the force matrix (6, see PFM);
//                element type R (double, or float in the mixed-precision form)
//   F_P planes   fp[k * stride + i], k = 0..8, always double
//   id           original index of the particle within its scene
// G2P writes each step's output in block-sorted order into the other buffer,
// so the particle arrays follow the grid blocks and stay coalesced.
//
// Grid: 4x4x4-node blocks, rebuilt every step.  Block b holds nodes
// (4*bx + lx, 4*by + ly, 4*bz + lz), local index lx + 4*ly + 16*lz.  Channels
// are planes of cap_blocks*64 values:
//   acc  [0] mass, [1..3] momentum, [4..6] force   (P2G output, zeroed after use)
//   vel  [0..2] velocity after collisions, [3..5] velocity - momentum/mass
//        (the FLIP increment; 0 at massless nodes)
// A block is found through an open-addressing hash table keyed by the block's
// 32-bit "block key" (see below); a slot holds the key and the block id in one
// 64-bit word.
//
// Sort key of a particle: the block key (the linear index of its block in its
// scene's bounding box of blocks, offset by the scene's key base) shifted left
// by 6, plus its cell within the block (cx + 4 cy + 16 cz).  The bounding box
// (one block of margin on the high side, so the +{0,1}^3 neighbours used by
// P2G/G2P are addressable) is measured by G2P for the next step.
//
// While the key boxes fit the dense bins (the usual case: their size is the
// boxes' volume in cells), particles are ordered by a counting sort over the
// keys, and grid block ids are a prefix sum over the block keys whose
// +{0,1}^3 neighbourhood holds particles, looked up directly by key.  Larger
// boxes fall back to the radix sort and the block hash table.
#pragma once

#include <cstdint>

#include "snow_math.cuh"

namespace snow {

// One P2G/G2P work item: a run of particles [start, end) of the block
// (bx, by, bz) of `scene`, and the ids of the block's +{0,1}^3 neighbours.
struct BlockHeader {
  int32_t start, end, scene, bx, by, bz, pad0, pad1;
  int32_t nbr[8];
};
static_assert(sizeof(BlockHeader) == 64, "item header is 16 words");

constexpr int kRealPlanes = 23;
constexpr int kFPPlanes = 9;
// PFM: the force matrix -V_p0 P F_E^T of the particle's current state (symmetric:
// xx, yy, zz, xy, xz, yz), written by G2P for the next step's P2G.
enum : int { PX = 0, PV = 3, PM = 6, PVOL = 7, PFE = 8, PFM = 17 };
constexpr int kRadixBits = 9;  // sort digit width (radix_sort.cu)
constexpr int kAccCh = 7;
constexpr int kVelCh = 6;
constexpr unsigned long long kEmptyEntry = ~0ull;
constexpr int kBinTile = 4096;  // keys per tile of the dense-bin scan (64 blocks)

// Status bits reported back to the host (snow_gpu_status).
enum : uint32_t {
  ST_BLOCK_OVERFLOW = 1u << 0,   // more grid blocks than allocated
  ST_HASH_FULL = 1u << 1,        // hash table probe exhausted
  ST_KEY_OVERFLOW = 1u << 2,     // bounding boxes too large for 32-bit sort keys
  ST_NONFINITE = 1u << 3,        // a particle position became NaN/Inf
  ST_OUT_OF_BOX = 1u << 4,       // a particle fell outside its scene's key box
  ST_LOOKUP_MISS = 1u << 5,      // a block expected in the table was not found
  ST_BIN_OVERFLOW = 1u << 6,     // key boxes larger than the dense bins
  ST_SCAN_STALL = 1u << 7,       // a bin-scan tile waited too long for its predecessor
};

struct SceneDev {
  void* r[2];        // real planes, buffers 0/1
  double* fp[2];     // F_P planes
  int32_t* id[2];    // original index
  int64_t stride;    // plane stride (elements)
  int64_t n;         // particles
  int64_t begin;     // offset of this scene in the batch's sorted index space
  int32_t cur;       // buffer holding the current state
  int32_t active;    // stepped by batch steps
  // step parameters (src/grid.cpp:359 arguments)
  double dx, dt, g[3], mu0, lambda0, xi, theta_c, theta_s, alpha;
  int32_t coll_begin, coll_count;
  // key box (written by the keyspace kernel each step)
  int32_t lo[3], dim[3];
  uint32_t key_base;
  uint32_t key_count;
  // bounding box of particle blocks measured for the next step (atomics)
  int32_t nb_lo[3], nb_hi[3];
  // emission box: the key box G2P writes the next step's sort keys against,
  // the blocks of this step's particles grown by one block on every side (a
  // particle moves less than a block per step); the next step sorts in it
  int32_t elo[3], edim[3];
  uint32_t ekey_base;
};

struct Counters {
  uint32_t n_blocks;    // grid blocks
  uint32_t key_blocks;  // block keys over all scenes' key boxes this step
  uint32_t sort_bits;   // significant key bits this step
  uint32_t work_p2g, work_grid, work_g2p, work_aux;
  uint32_t status;
  uint32_t n_items;     // (block, chunk) work items of the particle kernels
  uint32_t fp64_projections;  // mixed form: plastic projections redone in double
  uint32_t bin_ticket;  // next tile of the dense-bin scan
  uint32_t last_blocks, last_fp64;  // n_blocks and fp64_projections of the previous step
  // next-step keys written by G2P (dense bins only): emit_ok when the emission
  // boxes fit the bins, emit_fail when a particle fell outside its emission
  // box; keys_ready when this step's keys and bin counts are G2P's (the keys
  // kernel then has nothing to do)
  uint32_t emit_ok, emit_fail, keys_ready;
  uint32_t emit_blocks;  // block keys of the emission boxes G2P writes against
};

struct BatchDev {
  SceneDev* scenes;
  int32_t num_scenes;
  int64_t total;            // particles over all active scenes (sorted index space)
  const Collider* colliders;
  // sort
  uint32_t* keys[2];
  uint32_t* vals[2];
  uint32_t* hist;
  uint32_t* digit_total;
  int32_t ntiles;
  // dense key bins (counting sort by key, used when `dense` is set; otherwise
  // the radix sort and the block hash table): per key (block key << 6 | cell)
  // a particle count (zero between steps) and the first sorted position, and
  // per block key an occupancy byte (zero between steps) and the grid block id
  int32_t dense;
  int64_t cap_bins;         // keys (a multiple of kBinTile)
  uint32_t* bins;
  uint32_t* bin_off;
  uint8_t* occ;
  int32_t* idmap;
  unsigned long long* bin_state;  // chained-scan state of each bin tile
  // blocks: hash table of (block key << 32) | block id, empty slots all ones
  unsigned long long* htab;
  uint32_t hmask;
  int32_t cap_blocks;
  int4* blk;                // (bx, by, bz, scene)
  // work items of P2G/G2P: runs of at most `chunk` consecutive sorted particles
  // of one block, so that large blocks spread over CTAs
  BlockHeader* item_hdr;
  int32_t cap_items;
  int32_t chunk;
  // mixed form: (scene, output slot, input index) of projections to redo in double
  int4* fixups;
  int64_t cap_fixups;
  // grid
  void* acc;                // R[kAccCh][cap_blocks * 64]
  void* vel;                // R[kVelCh][cap_blocks * 64]
  Counters* ctr;
  // semi-implicit update (null when off): the grid update also writes each
  // node's mass here and leaves -momentum/mass in the FLIP channels, which the
  // solve completes once the velocities are final
  void* imp_mass;           // R[cap_blocks * 64]
};

// 32-bit mixer (finaliser of MurmurHash3) for the block table.
SNOW_HD uint32_t hash32(uint32_t k) {
  k ^= k >> 16;
  k *= 0x85ebca6bu;
  k ^= k >> 13;
  k *= 0xc2b2ae35u;
  k ^= k >> 16;
  return k;
}

// Block key of block (bx,by,bz) in scene s; the caller guarantees the block
// lies inside the key box.
SNOW_HD uint32_t block_key(const SceneDev& s, int bx, int by, int bz) {
  return s.key_base +
         (uint32_t)(((int64_t)(bz - s.lo[2]) * s.dim[1] + (by - s.lo[1])) * s.dim[0] + (bx - s.lo[0]));
}

__device__ __forceinline__ int32_t hash_find(const BatchDev& b, uint32_t key) {
  uint32_t slot = hash32(key) & b.hmask;
  for (uint32_t probe = 0; probe <= b.hmask; ++probe) {
    const unsigned long long e = b.htab[slot];
    if (e == kEmptyEntry) return -1;
    if ((uint32_t)(e >> 32) == key) {
      const uint32_t id = (uint32_t)e;
      return id < (uint32_t)b.cap_blocks ? (int32_t)id : -1;
    }
    slot = (slot + 1) & b.hmask;
  }
  return -1;
}

// Index of the scene owning sorted position j (scenes occupy consecutive ranges).
__device__ __forceinline__ int scene_of(const BatchDev& b, int64_t j) {
  int lo = 0, hi = b.num_scenes - 1;
  while (lo < hi) {
    const int mid = (lo + hi + 1) >> 1;
    if (b.scenes[mid].begin <= j) lo = mid; else hi = mid - 1;
  }
  return lo;
}

// ---------------------------------------------------------------- launchers
// Host-side launch functions (snow_kernels.cu, radix_sort.cu).
template <typename R>
struct StepLaunch {
  static void keyspace(const BatchDev& b, cudaStream_t s, bool init_box);
  static void keys(const BatchDev& b, cudaStream_t s);
  static void blocks(const BatchDev& b, cudaStream_t s);
  static void p2g(const BatchDev& b, int mode, cudaStream_t s);
  static void grid_update(const BatchDev& b, cudaStream_t s);
  static void g2p(const BatchDev& b, int mode, cudaStream_t s);
  static void zero_grid(const BatchDev& b, cudaStream_t s);
  static void finish(const BatchDev& b, cudaStream_t s);
  // finish, then keyspace for the next step, in one launch
  static void finish_and_keyspace(const BatchDev& b, cudaStream_t s);
  static void bbox_init(const BatchDev& b, cudaStream_t s);
  static void prepare_force(const BatchDev& b, cudaStream_t s);
  static void fixup(const BatchDev& b, cudaStream_t s);
};

enum P2GMode : int { P2G_FULL = 0, P2G_MASS = 1, P2G_MASS_MOMENTUM = 2, P2G_FORCE = 3, P2G_PRE = 4 };
enum G2PMode : int { G2P_FULL = 0, G2P_VOLUME = 1, G2P_STRESS = 2, G2P_VELOCITY = 3 };

void radix_sort(const BatchDev& b, cudaStream_t s);
int sm_count();

}  // namespace snow
