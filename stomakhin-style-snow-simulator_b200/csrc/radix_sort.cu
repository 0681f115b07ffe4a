// Stable LSD radix sort of the batch's (key, particle index) pairs, 9 bits per
// pass, reduce-then-scan:
//   upsweep    per 2048-key tile, a 512-bin digit histogram
//   scan       per digit, an exclusive scan over the tiles (digit-major order)
//   downsweep  per tile, the stable rank of every key among equal digits
//              (warp match + per-warp counts), then a scatter to
//              digit_base + tile_offset + rank
// The number of passes depends on the key bits of the current step, which
// only the device knows (Counters::sort_bits); every kernel of a pass that is
// not needed returns at once, so the host launches a fixed 4 passes and the
// sequence can be captured in a CUDA graph.  Pass p reads buffer p & 1 and
// writes buffer (p + 1) & 1; the sorted result is in buffer passes & 1.
// Nine-bit digits sort the 18-bit keys of a 650k-particle scene in two passes.
#include <cuda_runtime.h>

#include "snow_batch.cuh"

namespace snow {
namespace {

constexpr int kBits = kRadixBits;
constexpr int kDigits = 1 << kBits;
constexpr int kThreads = 256;
constexpr int kPerThread = kDigits / kThreads;  // digits owned by each thread
constexpr int kItems = 8;
constexpr int kTile = kThreads * kItems;
constexpr int kWarps = kThreads / 32;
constexpr int kMaxPasses = (32 + kBits - 1) / kBits;
static_assert(kDigits % kThreads == 0, "digits must be a multiple of the block size");

__device__ __forceinline__ bool pass_needed(const BatchDev& b, int pass) {
  return (uint32_t)(pass * kBits) < b.ctr->sort_bits;
}

// Exclusive scan over the 256 threads of a block; returns the block total.
__device__ __forceinline__ uint32_t block_exclusive_scan(uint32_t v, uint32_t& total,
                                                         uint32_t* s_warp) {
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  uint32_t x = v;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    const uint32_t y = __shfl_up_sync(0xffffffffu, x, o);
    if (lane >= o) x += y;
  }
  if (lane == 31) s_warp[warp] = x;
  __syncthreads();
  if (warp == 0) {
    uint32_t w = lane < kWarps ? s_warp[lane] : 0;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const uint32_t y = __shfl_up_sync(0xffffffffu, w, o);
      if (lane >= o) w += y;
    }
    if (lane < kWarps) s_warp[lane] = w;
  }
  __syncthreads();
  const uint32_t before = warp > 0 ? s_warp[warp - 1] : 0;
  total = s_warp[kWarps - 1];
  __syncthreads();
  return before + x - v;
}

__global__ void __launch_bounds__(kThreads) k_upsweep(const BatchDev b, int pass) {
  if (!pass_needed(b, pass)) return;
  __shared__ uint32_t h[kDigits];
  const uint32_t* keys = b.keys[pass & 1];
  const int shift = pass * kBits;
  for (int d = threadIdx.x; d < kDigits; d += kThreads) h[d] = 0;
  __syncthreads();
  const int64_t base = (int64_t)blockIdx.x * kTile;
  const int lane = threadIdx.x & 31;
#pragma unroll
  for (int k = 0; k < kItems; ++k) {
    const int64_t j = base + k * kThreads + threadIdx.x;
    const bool valid = j < b.total;
    const uint32_t d = valid ? (keys[j] >> shift) & (kDigits - 1) : kDigits;
    const uint32_t peers = __match_any_sync(0xffffffffu, d);
    if (valid && lane == __ffs(peers) - 1) atomicAdd(&h[d], (uint32_t)__popc(peers));
  }
  __syncthreads();
  for (int d = threadIdx.x; d < kDigits; d += kThreads) b.hist[(int64_t)d * b.ntiles + blockIdx.x] = h[d];
}

// One block per digit: exclusive scan of that digit's per-tile counts.
__global__ void __launch_bounds__(kThreads) k_scan(const BatchDev b, int pass) {
  if (!pass_needed(b, pass)) return;
  __shared__ uint32_t s_warp[kWarps];
  uint32_t* row = b.hist + (int64_t)blockIdx.x * b.ntiles;
  uint32_t carry = 0;
  for (int base = 0; base < b.ntiles; base += kThreads) {
    const int t = base + threadIdx.x;
    const uint32_t v = t < b.ntiles ? row[t] : 0;
    uint32_t total;
    const uint32_t ex = block_exclusive_scan(v, total, s_warp);
    if (t < b.ntiles) row[t] = carry + ex;
    carry += total;
  }
  if (threadIdx.x == 0) b.digit_total[blockIdx.x] = carry;
}

__global__ void __launch_bounds__(kThreads) k_downsweep(const BatchDev b, int pass) {
  if (!pass_needed(b, pass)) return;
  __shared__ uint32_t s_off[kDigits];
  __shared__ uint32_t s_run[kDigits];
  __shared__ uint32_t s_cnt[kWarps][kDigits];
  __shared__ uint32_t s_warp[kWarps];
  const uint32_t* kin = b.keys[pass & 1];
  const uint32_t* vin = b.vals[pass & 1];
  uint32_t* kout = b.keys[(pass + 1) & 1];
  uint32_t* vout = b.vals[(pass + 1) & 1];
  const int shift = pass * kBits;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;

  {  // digit bases: exclusive scan of digit totals (thread t owns digits t*kPerThread...),
     // plus this tile's offset within each digit
    uint32_t tot[kPerThread], sum = 0;
#pragma unroll
    for (int q = 0; q < kPerThread; ++q) {
      tot[q] = b.digit_total[threadIdx.x * kPerThread + q];
      sum += tot[q];
    }
    uint32_t all;
    uint32_t ex = block_exclusive_scan(sum, all, s_warp);
#pragma unroll
    for (int q = 0; q < kPerThread; ++q) {
      const int d = threadIdx.x * kPerThread + q;
      s_off[d] = ex + b.hist[(int64_t)d * b.ntiles + blockIdx.x];
      s_run[d] = 0;
      ex += tot[q];
    }
  }
  const int64_t base = (int64_t)blockIdx.x * kTile;
  const unsigned lt_mask = (1u << lane) - 1u;
  for (int round = 0; round < kItems; ++round) {
    const int64_t j = base + round * kThreads + threadIdx.x;
    const bool valid = j < b.total;
    uint32_t key = 0, val = 0;
    if (valid) {
      key = kin[j];
      val = vin[j];
    }
    const uint32_t d = valid ? (key >> shift) & (kDigits - 1) : kDigits;
    for (int e = threadIdx.x; e < kWarps * kDigits; e += kThreads) (&s_cnt[0][0])[e] = 0;
    __syncthreads();
    const uint32_t peers = __match_any_sync(0xffffffffu, d);
    const uint32_t rank = __popc(peers & lt_mask);
    if (valid && rank == 0) s_cnt[warp][d] = __popc(peers);
    __syncthreads();
#pragma unroll
    for (int q = 0; q < kPerThread; ++q) {  // per digit: prefix over warps, continuing from earlier rounds
      const int dd = threadIdx.x * kPerThread + q;
      uint32_t run = s_run[dd];
#pragma unroll
      for (int w = 0; w < kWarps; ++w) {
        const uint32_t c = s_cnt[w][dd];
        s_cnt[w][dd] = run;
        run += c;
      }
      s_run[dd] = run;
    }
    __syncthreads();
    if (valid) {
      const uint32_t pos = s_off[d] + s_cnt[warp][d] + rank;
      kout[pos] = key;
      vout[pos] = val;
    }
    __syncthreads();
  }
}

}  // namespace

void radix_sort(const BatchDev& b, cudaStream_t s) {
  if (b.total <= 0 || b.dense) return;  // dense bins: counting sort in StepLaunch::blocks
  for (int pass = 0; pass < kMaxPasses; ++pass) {
    k_upsweep<<<b.ntiles, kThreads, 0, s>>>(b, pass);
    k_scan<<<kDigits, kThreads, 0, s>>>(b, pass);
    k_downsweep<<<b.ntiles, kThreads, 0, s>>>(b, pass);
  }
}

int radix_tiles(int64_t n) { return (int)((n + kTile - 1) / kTile); }
int radix_digits() { return kDigits; }

}  // namespace snow
