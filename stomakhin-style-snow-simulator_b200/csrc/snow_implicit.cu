// Semi-implicit grid velocity update (Stomakhin et al., "A material point
// method for snow simulation", SIGGRAPH 2013, Section 4, eq. 9), the update
// the reference declares (include/snow/grid.hpp:76,80,88-92:
// constitutive_differential, index_nodes, deformation_differential,
// force_differential, apply_A, Conjugate_residual) and never defines.
//
// After the explicit grid update v* (collisions applied), the velocities of
// the nodes with mass solve
//   (I + beta dt^2 M^-1 H) v = v*,   H u = -delta f(u),
//   delta F_p = dt (sum_i u_i grad w_ip^T) F_Ep,
//   delta f_i = -sum_p V_p0 A_p(delta F_p) F_Ep^T grad w_ip,
// A_p the differential of the fixed-corotated stress at F_Ep (its F_P, and so
// the hardening, held fixed; corotated_differential).  The operator is
// self-adjoint in <a, b>_M = sum_i m_i a_i . b_i, in which conjugate residuals
// run from v = v* until <r, r>_M <= tol^2 <v*, v*>_M.
//
// Device work per iteration: one apply of the operator -- a persistent kernel
// over the P2G/G2P work items that stages u of the item's 7x7x7 nodes in
// shared memory, gathers each particle's delta F, forms G = -V0 dP F_E^T and
// scatters G grad w back into a shared tile, flushed with one global atomic
// per node and channel -- and node kernels for the vector updates with their
// M-weighted dot products.  The host reads the dot products between launches
// (the solve is not captured into the step graph).
#include <cuda_runtime.h>

#include <algorithm>
#include <climits>
#include <cmath>
#include <string>

#include "snow_batch.cuh"
#include "snow_engine.hpp"

namespace snow {
namespace {

constexpr int kImpThreads = 256;
constexpr int kTileSide = 7, kTileNodes = kTileSide * kTileSide * kTileSide;

template <typename R>
struct ImpDev {
  R* mass;                  // [plane]
  R *r, *p, *Ar, *Ap, *df;  // [3][plane] each
  R *rot, *sym, *lame;      // by sorted position: [9][cap_p], [6][cap_p], [2][cap_p]
  int64_t plane, cap_p;
  double* dots;             // [4] accumulators the host reads
  uint32_t* work;           // item counter of the apply kernel
};

__device__ __forceinline__ int tile_at(int x, int y, int z) { return x + kTileSide * (y + kTileSide * z); }

__device__ __forceinline__ int scene_of_pos(const BatchDev& b, int64_t j) {
  int lo = 0, hi = b.num_scenes - 1;
  while (lo < hi) {
    const int mid = (lo + hi + 1) >> 1;
    if (b.scenes[mid].begin <= j) lo = mid; else hi = mid - 1;
  }
  return lo;
}

__device__ __forceinline__ const uint32_t* sorted_index(const BatchDev& b) {
  if (b.dense) return b.vals[1];
  const uint32_t passes = (b.ctr->sort_bits + kRadixBits - 1) / kRadixBits;
  return b.vals[passes & 1];
}

// Adds v0 (and v1) of every thread of the block into dst[0] (and dst[1]).
__device__ void block_add(double* dst, double v0, double v1, bool two) {
  __shared__ double s[2][kImpThreads / 32];
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    v0 += __shfl_xor_sync(0xffffffffu, v0, o);
    v1 += __shfl_xor_sync(0xffffffffu, v1, o);
  }
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  if (lane == 0) {
    s[0][warp] = v0;
    s[1][warp] = v1;
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    double a = 0.0, c = 0.0;
    for (int w = 0; w < kImpThreads / 32; ++w) {
      a += s[0][w];
      c += s[1][w];
    }
    atomicAdd(dst, a);
    if (two) atomicAdd(dst + 1, c);
  }
}

// Per particle, by sorted position: the polar factors of F_E (fixed during the
// solve) and the hardened Lame parameters.
template <typename R>
__global__ void __launch_bounds__(kImpThreads) k_imp_prep(const BatchDev b, const ImpDev<R> d) {
  const uint32_t* vals = sorted_index(b);
  for (int64_t j = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; j < b.total;
       j += (int64_t)gridDim.x * blockDim.x) {
    const SceneDev& sc = b.scenes[scene_of_pos(b, j)];
    const int64_t i = vals[j];
    const R* r = (const R*)sc.r[sc.cur];
    const double* fp = sc.fp[sc.cur];
    M3<R> F;
#pragma unroll
    for (int e = 0; e < 9; ++e) F.a[e] = r[(PFE + e) * sc.stride + i];
    M3<double> FP;
#pragma unroll
    for (int e = 0; e < 9; ++e) FP.a[e] = fp[e * sc.stride + i];
    M3<R> Rm;
    Sym3<R> S;
    if (!polar_factors(F, Rm, S)) {  // a singular F_E: reported, and no stiffness from it
      atomicOr(&b.ctr->status, ST_NONFINITE);
#pragma unroll
      for (int e = 0; e < 9; ++e) Rm.a[e] = R(e % 4 == 0 ? 1 : 0);
      S = Sym3<R>{R(1), R(1), R(1), R(0), R(0), R(0)};
    }
    const double h = exp(sc.xi * (1.0 - det3(FP)));
#pragma unroll
    for (int e = 0; e < 9; ++e) d.rot[e * d.cap_p + j] = Rm.a[e];
    const R sv[6] = {S.xx, S.yy, S.zz, S.xy, S.xz, S.yz};
#pragma unroll
    for (int e = 0; e < 6; ++e) d.sym[e * d.cap_p + j] = sv[e];
    d.lame[j] = (R)(sc.mu0 * h);
    d.lame[d.cap_p + j] = (R)(sc.lambda0 * h);
  }
}

// df += delta f(u): the force differential of the node field u (3 planes).
template <typename R>
__global__ void __launch_bounds__(kImpThreads) k_imp_apply(const BatchDev b, const ImpDev<R> d, const R* u) {
  __shared__ R tu[3][kTileNodes];
  __shared__ R tf[3][kTileNodes];
  __shared__ BlockHeader h;
  __shared__ int s_item;
  const uint32_t items = min(b.ctr->n_items, (uint32_t)b.cap_items);
  const uint32_t* vals = sorted_index(b);
  const int64_t plane = d.plane;
  for (;;) {
    if (threadIdx.x == 0) s_item = (int)atomicAdd(d.work, 1u);
    __syncthreads();
    if ((uint32_t)s_item >= items) return;
    if (threadIdx.x < 16)
      reinterpret_cast<int*>(&h)[threadIdx.x] = reinterpret_cast<const int*>(b.item_hdr + s_item)[threadIdx.x];
    __syncthreads();
    for (int e = threadIdx.x; e < 8 * 64; e += blockDim.x) {
      const int nd = e >> 6, node = e & 63;
      const int x = 4 * (nd & 1) + (node & 3), y = 4 * ((nd >> 1) & 1) + ((node >> 2) & 3),
                z = 4 * (nd >> 2) + (node >> 4);
      if (x >= kTileSide || y >= kTileSide || z >= kTileSide) continue;
      const int t = tile_at(x, y, z);
      const int32_t nb = h.nbr[nd];
      const int64_t g = (int64_t)(nb < 0 ? 0 : nb) * 64 + node;
#pragma unroll
      for (int c = 0; c < 3; ++c) {
        tu[c][t] = nb < 0 ? R(0) : u[c * plane + g];
        tf[c][t] = R(0);
      }
    }
    __syncthreads();
    const SceneDev& sc = b.scenes[h.scene];
    const R dx = (R)sc.dx, dt = (R)sc.dt;
    const R* pr = (const R*)sc.r[sc.cur];
    const int n = h.end - h.start;
    for (int k = threadIdx.x; k < n; k += blockDim.x) {
      const int64_t j = h.start + k;
      const int64_t i = vals[j];
      const AxisWeights<R> wx = axis_weights(pr[(PX + 0) * sc.stride + i], dx);
      const AxisWeights<R> wy = axis_weights(pr[(PX + 1) * sc.stride + i], dx);
      const AxisWeights<R> wz = axis_weights(pr[(PX + 2) * sc.stride + i], dx);
      const int tx = wx.base - 4 * h.bx, ty = wy.base - 4 * h.by, tz = wz.base - 4 * h.bz;
      if ((unsigned)tx > 3u || (unsigned)ty > 3u || (unsigned)tz > 3u) {
        atomicOr(&b.ctr->status, ST_OUT_OF_BOX);
        continue;
      }
      // grad u = sum_n u_n grad w_n^T
      R gu[9] = {R(0), R(0), R(0), R(0), R(0), R(0), R(0), R(0), R(0)};  // column-major
      for (int a = 0; a < 4; ++a)
        for (int c = 0; c < 4; ++c)
#pragma unroll
          for (int e = 0; e < 4; ++e) {
            const int t = tile_at(tx + a, ty + c, tz + e);
            const R gw[3] = {wx.dw[a] * wy.w[c] * wz.w[e], wx.w[a] * wy.dw[c] * wz.w[e],
                             wx.w[a] * wy.w[c] * wz.dw[e]};
#pragma unroll
            for (int rr = 0; rr < 3; ++rr) {
              const R un = tu[rr][t];
#pragma unroll
              for (int cc = 0; cc < 3; ++cc) gu[cc * 3 + rr] += un * gw[cc];
            }
          }
      M3<R> F, G, dF;
#pragma unroll
      for (int e = 0; e < 9; ++e) F.a[e] = pr[(PFE + e) * sc.stride + i];
#pragma unroll
      for (int cc = 0; cc < 3; ++cc)
#pragma unroll
        for (int rr = 0; rr < 3; ++rr)
          dF(rr, cc) = dt * (gu[rr] * F(0, cc) + gu[3 + rr] * F(1, cc) + gu[6 + rr] * F(2, cc));
      M3<R> Rm;
#pragma unroll
      for (int e = 0; e < 9; ++e) Rm.a[e] = d.rot[e * d.cap_p + j];
      const Sym3<R> S{d.sym[j], d.sym[d.cap_p + j], d.sym[2 * d.cap_p + j], d.sym[3 * d.cap_p + j],
                      d.sym[4 * d.cap_p + j], d.sym[5 * d.cap_p + j]};
      const M3<R> dP = corotated_differential(F, Rm, S, d.lame[j], d.lame[d.cap_p + j], dF);
      const R V0 = pr[PVOL * sc.stride + i];
      // G = -V0 dP F^T
#pragma unroll
      for (int cc = 0; cc < 3; ++cc)
#pragma unroll
        for (int rr = 0; rr < 3; ++rr)
          G(rr, cc) = -V0 * (dP(rr, 0) * F(cc, 0) + dP(rr, 1) * F(cc, 1) + dP(rr, 2) * F(cc, 2));
      for (int a = 0; a < 4; ++a)
        for (int c = 0; c < 4; ++c)
#pragma unroll
          for (int e = 0; e < 4; ++e) {
            const int t = tile_at(tx + a, ty + c, tz + e);
            const R gw[3] = {wx.dw[a] * wy.w[c] * wz.w[e], wx.w[a] * wy.dw[c] * wz.w[e],
                             wx.w[a] * wy.w[c] * wz.dw[e]};
#pragma unroll
            for (int rr = 0; rr < 3; ++rr)
              atomicAdd(&tf[rr][t], G(rr, 0) * gw[0] + G(rr, 1) * gw[1] + G(rr, 2) * gw[2]);
          }
    }
    __syncthreads();
    for (int e = threadIdx.x; e < 8 * 64; e += blockDim.x) {
      const int nd = e >> 6, node = e & 63;
      const int x = 4 * (nd & 1) + (node & 3), y = 4 * ((nd >> 1) & 1) + ((node >> 2) & 3),
                z = 4 * (nd >> 2) + (node >> 4);
      if (x >= kTileSide || y >= kTileSide || z >= kTileSide) continue;
      const int32_t nb = h.nbr[nd];
      if (nb < 0) continue;
      const int t = tile_at(x, y, z);
      const int64_t g = (int64_t)nb * 64 + node;
#pragma unroll
      for (int c = 0; c < 3; ++c)
        if (tf[c][t] != R(0)) atomicAdd(&d.df[c * plane + g], tf[c][t]);
    }
    __syncthreads();
  }
}

__device__ __forceinline__ int64_t node_count(const BatchDev& b) {
  return (int64_t)min(b.ctr->n_blocks, (uint32_t)b.cap_blocks) * 64;
}

// beta dt of the scene node e belongs to.
__device__ __forceinline__ double node_bdt(const BatchDev& b, int64_t e, double beta) {
  return beta * b.scenes[b.blk[e >> 6].w].dt;
}

// r = b - A b for the start x = b = v*: r = beta dt df / m; p = r.
// dots += (<r, r>_M, <x, x>_M).
template <typename R>
__global__ void __launch_bounds__(kImpThreads) k_imp_start(const BatchDev b, const ImpDev<R> d, double beta) {
  const R* x = (const R*)b.vel;
  double rr = 0.0, xx = 0.0;
  const int64_t work = node_count(b);
  for (int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; e < work; e += (int64_t)gridDim.x * blockDim.x) {
    const R m = d.mass[e];
    const R bdt = (R)node_bdt(b, e, beta);
#pragma unroll
    for (int c = 0; c < 3; ++c) {
      const int64_t k = c * d.plane + e;
      const R rv = m > R(0) ? bdt * d.df[k] / m : R(0);
      d.r[k] = d.p[k] = rv;
      if (m > R(0)) {
        rr += (double)m * rv * rv;
        xx += (double)m * x[k] * x[k];
      }
    }
  }
  block_add(d.dots, rr, xx, true);
}

// Ar = r - beta dt df / m (the operator on r, from df = delta f(r)); with
// `first`, also Ap = Ar.  dots += (<r, Ar>_M, <Ar, Ar>_M when first).
template <typename R>
__global__ void __launch_bounds__(kImpThreads) k_imp_ar(const BatchDev b, const ImpDev<R> d, double beta, int first) {
  double rAr = 0.0, ArAr = 0.0;
  const int64_t work = node_count(b);
  for (int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; e < work; e += (int64_t)gridDim.x * blockDim.x) {
    const R m = d.mass[e];
    const R bdt = (R)node_bdt(b, e, beta);
#pragma unroll
    for (int c = 0; c < 3; ++c) {
      const int64_t k = c * d.plane + e;
      const R a = m > R(0) ? d.r[k] - bdt * d.df[k] / m : R(0);
      d.Ar[k] = a;
      if (first) d.Ap[k] = a;
      if (m > R(0)) {
        rAr += (double)m * d.r[k] * a;
        ArAr += (double)m * a * a;
      }
    }
  }
  block_add(d.dots, rAr, ArAr, first != 0);
}

// x += alpha p; r -= alpha Ap.  dots += <r, r>_M.
template <typename R>
__global__ void __launch_bounds__(kImpThreads) k_imp_update(const BatchDev b, const ImpDev<R> d, double alpha) {
  R* x = (R*)b.vel;
  double rr = 0.0;
  const int64_t work = node_count(b);
  for (int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; e < work; e += (int64_t)gridDim.x * blockDim.x) {
    const R m = d.mass[e];
    if (!(m > R(0))) continue;
#pragma unroll
    for (int c = 0; c < 3; ++c) {
      const int64_t k = c * d.plane + e;
      x[k] += (R)alpha * d.p[k];
      const R rv = d.r[k] - (R)alpha * d.Ap[k];
      d.r[k] = rv;
      rr += (double)m * rv * rv;
    }
  }
  block_add(d.dots, rr, 0.0, false);
}

// p = r + beta_k p; Ap = Ar + beta_k Ap.  dots += <Ap, Ap>_M.
template <typename R>
__global__ void __launch_bounds__(kImpThreads) k_imp_direction(const BatchDev b, const ImpDev<R> d, double beta_k) {
  double apap = 0.0;
  const int64_t work = node_count(b);
  for (int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; e < work; e += (int64_t)gridDim.x * blockDim.x) {
    const R m = d.mass[e];
    if (!(m > R(0))) continue;
#pragma unroll
    for (int c = 0; c < 3; ++c) {
      const int64_t k = c * d.plane + e;
      d.p[k] = d.r[k] + (R)beta_k * d.p[k];
      const R a = d.Ar[k] + (R)beta_k * d.Ap[k];
      d.Ap[k] = a;
      apap += (double)m * a * a;
    }
  }
  block_add(d.dots, apap, 0.0, false);
}

// vel[0..2] <- A vel[0..2] = u - beta dt df / m at nodes with mass (df =
// delta f(u)); massless nodes keep u.
template <typename R>
__global__ void __launch_bounds__(kImpThreads) k_imp_apply_out(const BatchDev b, const ImpDev<R> d, double beta) {
  R* u = (R*)b.vel;
  const int64_t work = node_count(b);
  for (int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; e < work; e += (int64_t)gridDim.x * blockDim.x) {
    const R m = d.mass[e];
    if (!(m > R(0))) continue;
    const R bdt = (R)node_bdt(b, e, beta);
#pragma unroll
    for (int c = 0; c < 3; ++c) u[c * d.plane + e] -= bdt * d.df[c * d.plane + e] / m;
  }
}

// The FLIP channels: v - momentum / mass now that v is final (they hold
// -momentum / mass at nodes with mass since the grid update).
template <typename R>
__global__ void __launch_bounds__(kImpThreads) k_imp_finish(const BatchDev b, const ImpDev<R> d) {
  R* v = (R*)b.vel;
  const int64_t work = node_count(b);
  for (int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; e < work; e += (int64_t)gridDim.x * blockDim.x) {
    if (!(d.mass[e] > R(0))) continue;
#pragma unroll
    for (int c = 0; c < 3; ++c) v[(3 + c) * d.plane + e] += v[c * d.plane + e];
  }
}

// Host node lists <-> the grid of a one-scene batch built with the block hash
// table: node k (ijk[k]) lives at grid entry e(k), or nowhere when no particle
// stencil reaches it (e = -1).
__global__ void k_imp_node_entries(const BatchDev b, const int32_t* ijk, int64_t n_nodes, int64_t* entry) {
  const int64_t k = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= n_nodes) return;
  const SceneDev& sc = b.scenes[0];
  int bc[3], loc[3];
  entry[k] = -1;
  for (int a = 0; a < 3; ++a) {
    const int v = ijk[3 * k + a];
    bc[a] = v >> 2;
    loc[a] = v & 3;
    if (bc[a] < sc.lo[a] || bc[a] >= sc.lo[a] + sc.dim[a]) return;
  }
  const int32_t id = hash_find(b, block_key(sc, bc[0], bc[1], bc[2]));
  if (id >= 0) entry[k] = (int64_t)id * 64 + loc[0] + 4 * loc[1] + 16 * loc[2];
}

// mass and the vector (q if given, else the node velocity) into the grid.
__global__ void k_imp_load(const BatchDev b, const int64_t* entry, const double* fields, const double* q,
                           int64_t n_nodes, double* mass) {
  const int64_t k = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= n_nodes || entry[k] < 0) return;
  const int64_t e = entry[k], plane = (int64_t)b.cap_blocks * 64;
  double* v = (double*)b.vel;
  mass[e] = fields[10 * k];
  for (int a = 0; a < 3; ++a) v[a * plane + e] = q ? q[3 * k + a] : fields[10 * k + 4 + a];
}

__global__ void k_imp_store(const BatchDev b, const int64_t* entry, const double* fields, const double* q,
                            int64_t n_nodes, double* out) {
  const int64_t k = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= n_nodes) return;
  const int64_t e = entry[k], plane = (int64_t)b.cap_blocks * 64;
  const double* v = (const double*)b.vel;
  for (int a = 0; a < 3; ++a)
    out[3 * k + a] = e >= 0 ? v[a * plane + e] : (q ? q[3 * k + a] : fields[10 * k + 4 + a]);
}

}  // namespace

void Batch::ensure_implicit() {
  const size_t rs = rsize_;
  const int64_t plane = (int64_t)cap_blocks_ * 64;
  if (plane > imp_cap_nodes_) {
    if (imp_nodes_) cudaFree(imp_nodes_);
    imp_nodes_ = nullptr;
    check_cuda(cudaMalloc(&imp_nodes_, (size_t)plane * 16 * rs), "cudaMalloc implicit nodes");
    imp_cap_nodes_ = plane;
  }
  if (cap_p_ > imp_cap_p_) {
    if (imp_parts_) cudaFree(imp_parts_);
    imp_parts_ = nullptr;
    check_cuda(cudaMalloc(&imp_parts_, (size_t)cap_p_ * 17 * rs), "cudaMalloc implicit particles");
    imp_cap_p_ = cap_p_;
  }
  if (!imp_dots_) {
    check_cuda(cudaMalloc((void**)&imp_dots_, 4 * sizeof(double) + 64), "cudaMalloc implicit scalars");
    check_cuda(cudaMallocHost((void**)&imp_host_, 4 * sizeof(double)), "cudaMallocHost implicit scalars");
  }
}

void Batch::free_implicit() {
  if (imp_nodes_) cudaFree(imp_nodes_);
  if (imp_parts_) cudaFree(imp_parts_);
  if (imp_dots_) cudaFree(imp_dots_);
  if (imp_host_) cudaFreeHost(imp_host_);
  imp_nodes_ = imp_parts_ = nullptr;
  imp_dots_ = nullptr;
  imp_host_ = nullptr;
  imp_cap_nodes_ = imp_cap_p_ = 0;
}

template <typename R>
void Batch::implicit_solve(const BatchDev& b, cudaStream_t s, bool apply_only) {
  ImpDev<R> d{};
  const int64_t plane = (int64_t)cap_blocks_ * 64;  // the grid's channel stride, as for vel
  if (plane > imp_cap_nodes_ || total_ > imp_cap_p_) throw Error(SNOW_E_STATE, "implicit buffers not sized");
  R* nodes = static_cast<R*>(imp_nodes_);
  d.mass = nodes;
  d.r = nodes + plane;
  d.p = nodes + 4 * plane;
  d.Ar = nodes + 7 * plane;
  d.Ap = nodes + 10 * plane;
  d.df = nodes + 13 * plane;
  d.plane = plane;
  R* parts = static_cast<R*>(imp_parts_);
  d.cap_p = imp_cap_p_;
  d.rot = parts;
  d.sym = parts + 9 * imp_cap_p_;
  d.lame = parts + 15 * imp_cap_p_;
  d.dots = imp_dots_;
  d.work = reinterpret_cast<uint32_t*>(imp_dots_ + 4);
  const double beta = imp_beta_;  // the batch's setting; dt is each scene's own
  const int sms = sm_count();
  const int node_grid = 4 * sms, apply_grid = 2 * sms;
  auto zero_df = [&] {
    check_cuda(cudaMemsetAsync(d.df, 0, (size_t)3 * plane * sizeof(R), s), "implicit df");
    check_cuda(cudaMemsetAsync(d.work, 0, sizeof(uint32_t), s), "implicit work");
  };
  auto dots = [&](int k) {
    check_cuda(cudaMemcpyAsync(imp_host_, imp_dots_, 4 * sizeof(double), cudaMemcpyDeviceToHost, s), "dots");
    check_cuda(cudaStreamSynchronize(s), "implicit solve");
    for (int q = 0; q < k; ++q) imp_read_[q] = imp_host_[q];
    check_cuda(cudaMemsetAsync(imp_dots_, 0, 4 * sizeof(double), s), "dots");
  };
  check_cuda(cudaMemsetAsync(imp_dots_, 0, 4 * sizeof(double), s), "dots");
  k_imp_prep<R><<<std::max<int64_t>(1, std::min<int64_t>((b.total + 255) / 256, 8 * sms)), kImpThreads, 0, s>>>(b, d);
  if (apply_only) {
    zero_df();
    k_imp_apply<R><<<apply_grid, kImpThreads, 0, s>>>(b, d, (const R*)b.vel);
    k_imp_apply_out<R><<<node_grid, kImpThreads, 0, s>>>(b, d, beta);
    check_cuda(cudaGetLastError(), "implicit apply");
    return;
  }
  // r = v* - A v*, p = r
  zero_df();
  k_imp_apply<R><<<apply_grid, kImpThreads, 0, s>>>(b, d, (const R*)b.vel);
  k_imp_start<R><<<node_grid, kImpThreads, 0, s>>>(b, d, beta);
  dots(2);
  double rr = imp_read_[0];
  const double bb = imp_read_[1];
  // Ar = A r, Ap = Ar
  zero_df();
  k_imp_apply<R><<<apply_grid, kImpThreads, 0, s>>>(b, d, d.r);
  k_imp_ar<R><<<node_grid, kImpThreads, 0, s>>>(b, d, beta, 1);
  dots(2);
  double gamma = imp_read_[0], apap = imp_read_[1];
  int it = 0;
  while (it < imp_max_iter_ && rr > imp_tol2_ * bb && apap > 0.0) {
    const double alpha = gamma / apap;
    k_imp_update<R><<<node_grid, kImpThreads, 0, s>>>(b, d, alpha);
    dots(1);
    rr = imp_read_[0];
    ++it;
    if (!(rr > imp_tol2_ * bb)) break;
    zero_df();
    k_imp_apply<R><<<apply_grid, kImpThreads, 0, s>>>(b, d, d.r);
    k_imp_ar<R><<<node_grid, kImpThreads, 0, s>>>(b, d, beta, 0);
    dots(1);
    const double gamma_next = imp_read_[0];
    if (gamma == 0.0) break;
    const double beta_k = gamma_next / gamma;
    gamma = gamma_next;
    k_imp_direction<R><<<node_grid, kImpThreads, 0, s>>>(b, d, beta_k);
    dots(1);
    apap = imp_read_[0];
  }
  k_imp_finish<R><<<node_grid, kImpThreads, 0, s>>>(b, d);
  check_cuda(cudaGetLastError(), "implicit solve");
  last_imp_iters_ = it;
  last_imp_res_ = bb > 0.0 ? std::sqrt(std::max(rr, 0.0) / bb) : 0.0;
}

template void Batch::implicit_solve<double>(const BatchDev&, cudaStream_t, bool);
template void Batch::implicit_solve<float>(const BatchDev&, cudaStream_t, bool);

}  // namespace snow

// ------------------------------------------------------------ stage entry
using namespace snow;

extern "C" int snow_gpu_stage_implicit(const int32_t* ijk, const double* fields, int64_t n_nodes,
                                       const double* records, int64_t n, double grid_spacing, double time_step,
                                       double mu_0, double lambda_0, double hardening_coefficient, double beta,
                                       double squared_tolerance, int max_iterations, const double* q, double* out,
                                       int* iterations) {
  try {
    if (n < 0 || (n > 0 && !records)) throw Error(SNOW_E_ARG, "bad particle array");
    if (n_nodes < 0 || (n_nodes > 0 && (!ijk || !fields || !out))) throw Error(SNOW_E_ARG, "bad node list");
    if (!(grid_spacing > 0.0) || !(beta >= 0.0 && beta <= 1.0) || !(squared_tolerance > 0.0) || max_iterations < 1)
      throw Error(SNOW_E_ARG, "bad implicit parameters");
    if (iterations) *iterations = 0;
    if (n_nodes == 0) return SNOW_OK;
    if (n == 0 || beta == 0.0) {  // no particles or no implicit term: A is the identity
      for (int64_t k = 0; k < n_nodes; ++k)
        for (int a = 0; a < 3; ++a) out[3 * k + a] = q ? q[3 * k + a] : fields[10 * k + 4 + a];
      return SNOW_OK;
    }
    snow_step_params p{};
    p.grid_spacing = grid_spacing;
    p.time_step = time_step;
    p.mu_0 = mu_0;
    p.lambda_0 = lambda_0;
    p.hardening_coefficient = hardening_coefficient;
    p.max_compression = 0.5;
    p.max_stretch = 0.5;
    Batch batch(SNOW_FP64);
    batch.add_scene(records, n, &p, nullptr, 0, nullptr);
    batch.set_dense(false);  // node lookups through the block hash table
    batch.set_implicit(beta, std::sqrt(squared_tolerance), max_iterations);
    batch.prepare(nullptr);
    batch.ensure_implicit();
    const BatchDev b = batch.dev(batch.device_scenes(), 1, n);
    StepLaunch<double>::keyspace(b, nullptr, true);
    StepLaunch<double>::keys(b, nullptr);
    radix_sort(b, nullptr);
    StepLaunch<double>::blocks(b, nullptr);
    const int64_t plane = (int64_t)b.cap_blocks * 64;
    check_cuda(cudaMemset(b.vel, 0, (size_t)plane * kVelCh * sizeof(double)), "velocities");
    check_cuda(cudaMemset(b.imp_mass, 0, (size_t)plane * sizeof(double)), "masses");
    int64_t* entry = nullptr;
    double *dfields = nullptr, *dq = nullptr, *dout = nullptr;
    int32_t* dijk = nullptr;
    auto release = [&] {
      cudaFree(entry);
      cudaFree(dfields);
      cudaFree(dq);
      cudaFree(dout);
      cudaFree(dijk);
    };
    try {
      check_cuda(cudaMalloc((void**)&entry, n_nodes * sizeof(int64_t)), "cudaMalloc");
      check_cuda(cudaMalloc((void**)&dfields, n_nodes * 10 * sizeof(double)), "cudaMalloc");
      check_cuda(cudaMalloc((void**)&dout, n_nodes * 3 * sizeof(double)), "cudaMalloc");
      check_cuda(cudaMalloc((void**)&dijk, n_nodes * 3 * sizeof(int32_t)), "cudaMalloc");
      check_cuda(cudaMemcpy(dijk, ijk, n_nodes * 3 * sizeof(int32_t), cudaMemcpyHostToDevice), "nodes");
      check_cuda(cudaMemcpy(dfields, fields, n_nodes * 10 * sizeof(double), cudaMemcpyHostToDevice), "nodes");
      if (q) {
        check_cuda(cudaMalloc((void**)&dq, n_nodes * 3 * sizeof(double)), "cudaMalloc");
        check_cuda(cudaMemcpy(dq, q, n_nodes * 3 * sizeof(double), cudaMemcpyHostToDevice), "q");
      }
      const unsigned g = (unsigned)((n_nodes + 255) / 256);
      k_imp_node_entries<<<g, 256>>>(b, dijk, n_nodes, entry);
      k_imp_load<<<g, 256>>>(b, entry, dfields, dq, n_nodes, (double*)b.imp_mass);
      check_cuda(cudaGetLastError(), "load nodes");
      batch.implicit_solve<double>(b, nullptr, q != nullptr);
      k_imp_store<<<g, 256>>>(b, entry, dfields, dq, n_nodes, dout);
      check_cuda(cudaGetLastError(), "store nodes");
      check_cuda(cudaMemcpy(out, dout, n_nodes * 3 * sizeof(double), cudaMemcpyDeviceToHost), "out");
      Counters c{};
      check_cuda(cudaMemcpy(&c, b.ctr, sizeof c, cudaMemcpyDeviceToHost), "status");
      if (c.status) throw Error(SNOW_E_STATE, "implicit stage: grid status " + std::to_string(c.status));
    } catch (...) {
      release();
      throw;
    }
    release();
    if (iterations && !q) batch.implicit_stats(iterations, nullptr);
    return SNOW_OK;
  } catch (const Error& e) {
    return set_error(e.code, e.what());
  } catch (const std::exception& e) {
    return set_error(SNOW_E_ARG, e.what());
  }
}
