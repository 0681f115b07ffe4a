// Single-stage entry points: the reference's per-stage functions
// (include/snow/grid.hpp:75-95 of the reference tree) on host node lists and
// particle records, run through the same device code as the fused step.
// They build a private FP64 batch per call; they exist for the stage-level
// API and its tests, not for speed.
#include <cuda_runtime.h>

#include <algorithm>
#include <cstring>
#include <vector>

#include "snow_batch.cuh"
#include "snow_engine.hpp"
#include "snow_gpu.h"

namespace snow {
namespace {

static_assert(sizeof(snow_collider) == sizeof(Collider), "collider layouts must agree");

template <typename T>
struct DBuf {
  T* p = nullptr;
  explicit DBuf(size_t n) { check_cuda(cudaMalloc((void**)&p, (n ? n : 1) * sizeof(T)), "cudaMalloc"); }
  ~DBuf() { cudaFree(p); }
  DBuf(const DBuf&) = delete;
};

// A private batch holding the stage particles as one scene, with the block
// grid built for them (keyspace, keys, sort, blocks) but no P2G yet.
struct StageGrid {
  Batch batch{SNOW_FP64};
  int32_t id = -1;
  int64_t n = 0;
  BatchDev b{};
  StageGrid(const double* rec, int64_t n_, const snow_step_params& p) : n(n_) {
    id = batch.add_scene(rec, n, &p, nullptr, 0, nullptr);
    batch.set_dense(false);  // the node export reads the block hash table
    batch.prepare(nullptr);
    b = batch.dev(batch.device_scenes(), 1, n);
    StepLaunch<double>::keyspace(b, nullptr, true);
    StepLaunch<double>::keys(b, nullptr);
    radix_sort(b, nullptr);
    StepLaunch<double>::blocks(b, nullptr);
    check_cuda(cudaGetLastError(), "stage grid");
  }
  void finish_checked() {
    check_cuda(cudaMemcpy(batch.host_counters(), b.ctr, sizeof(Counters), cudaMemcpyDeviceToHost), "status");
    batch.set_last_status(batch.host_counters()->status);
    batch.check_status();
  }
  int64_t blocks() const {
    const Counters* c = const_cast<StageGrid*>(this)->batch.host_counters();
    return std::min<int64_t>(c->n_blocks, b.cap_blocks);
  }
  // Every node of every block, with the channels of acc.
  void export_nodes(int32_t* ijk, double* fields, int64_t cap, int64_t* n_nodes) {
    finish_checked();
    const int64_t nb = blocks();
    std::vector<int4> blk((size_t)nb);
    check_cuda(cudaMemcpy(blk.data(), b.blk, nb * sizeof(int4), cudaMemcpyDeviceToHost), "blocks");
    // ids that lost an insertion race hold no nodes: keep only the ids in the table
    std::vector<unsigned long long> tab((size_t)b.hmask + 1);
    check_cuda(cudaMemcpy(tab.data(), b.htab, tab.size() * sizeof(unsigned long long), cudaMemcpyDeviceToHost),
               "block table");
    std::vector<char> live((size_t)nb, 0);
    int64_t n_live = 0;
    for (const unsigned long long e : tab)
      if (e != kEmptyEntry && (int64_t)(uint32_t)e < nb && !live[(uint32_t)e]) {
        live[(uint32_t)e] = 1;
        ++n_live;
      }
    const int64_t nn = n_live * 64;
    if (n_nodes) *n_nodes = nn;
    if (nn > cap) throw Error(SNOW_E_ARG, "node capacity too small: need " + std::to_string(nn));
    const int64_t plane = (int64_t)b.cap_blocks * 64;
    std::vector<std::vector<double>> ch(kAccCh);
    for (int c = 0; c < kAccCh; ++c) {
      ch[c].resize((size_t)(nb * 64));
      check_cuda(cudaMemcpy(ch[c].data(), (const double*)b.acc + c * plane, nb * 64 * sizeof(double),
                            cudaMemcpyDeviceToHost),
                 "grid");
    }
    int64_t k = 0;
    for (int64_t id = 0; id < nb; ++id) {
      if (!live[(size_t)id]) continue;
      const int4 bc = blk[(size_t)id];
      for (int node = 0; node < 64; ++node, ++k) {
        const int64_t e = id * 64 + node;
        ijk[3 * k] = 4 * bc.x + (node & 3);
        ijk[3 * k + 1] = 4 * bc.y + ((node >> 2) & 3);
        ijk[3 * k + 2] = 4 * bc.z + (node >> 4);
        double* f = fields + 10 * k;
        f[0] = ch[0][(size_t)e];
        for (int a = 0; a < 3; ++a) {
          f[1 + a] = ch[1 + a][(size_t)e];
          f[4 + a] = 0.0;
          f[7 + a] = ch[4 + a][(size_t)e];
        }
      }
    }
    StepLaunch<double>::zero_grid(b, nullptr);
  }
};

// Loads host nodes into the stage grid (nodes outside its blocks are dropped:
// no stencil of the stage particles reaches them).  mode: 0 mass into acc,
// 1 velocity into vel[0..2], 2 velocity and FLIP increment into vel[0..5].
__global__ void k_load_nodes(const BatchDev b, const int32_t* ijk, const double* fields,
                             int64_t n_nodes, int mode) {
  const int64_t k = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= n_nodes) return;
  const SceneDev& sc = b.scenes[0];
  int bc[3], loc[3];
  for (int a = 0; a < 3; ++a) {
    const int v = ijk[3 * k + a];
    bc[a] = v >> 2;
    loc[a] = v & 3;
    if (bc[a] < sc.lo[a] || bc[a] >= sc.lo[a] + sc.dim[a]) return;
  }
  const int32_t id = hash_find(b, block_key(sc, bc[0], bc[1], bc[2]));
  if (id < 0) return;
  const int64_t e = (int64_t)id * 64 + loc[0] + 4 * loc[1] + 16 * loc[2];
  const int64_t plane = (int64_t)b.cap_blocks * 64;
  const double* f = fields + 10 * k;
  double* acc = (double*)b.acc;
  double* vel = (double*)b.vel;
  if (mode == 0) {
    acc[e] = f[0];
    return;
  }
  for (int a = 0; a < 3; ++a) vel[a * plane + e] = f[4 + a];
  if (mode == 2)
    for (int a = 0; a < 3; ++a) vel[(3 + a) * plane + e] = f[0] > 0.0 ? f[4 + a] - f[1 + a] / f[0] : 0.0;
}

__global__ void k_zero_vel(const BatchDev b) {
  const int64_t plane = (int64_t)b.cap_blocks * 64;
  const int64_t work = (int64_t)min(b.ctr->n_blocks, (uint32_t)b.cap_blocks) * 64;
  double* vel = (double*)b.vel;
  for (int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; e < work; e += (int64_t)gridDim.x * blockDim.x)
    for (int c = 0; c < kVelCh; ++c) vel[c * plane + e] = 0.0;
}

__global__ void k_grid_velocity_nodes(double* fields, int64_t n, double gx, double gy, double gz, double dt) {
  const int64_t k = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= n) return;
  double* f = fields + 10 * k;
  const double p[3] = {f[1], f[2], f[3]}, fo[3] = {f[7], f[8], f[9]}, g[3] = {gx, gy, gz};
  double v[3], pm[3];
  if (node_velocity(f[0], p, fo, g, dt, v, pm))
    for (int a = 0; a < 3; ++a) f[4 + a] = v[a];
}

__global__ void k_grid_collide_nodes(const int32_t* ijk, double* fields, int64_t n, const Collider* c,
                                     int nc, double dx) {
  const int64_t k = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= n) return;
  double* f = fields + 10 * k;
  const double x = dx * ijk[3 * k], y = dx * ijk[3 * k + 1], z = dx * ijk[3 * k + 2];
  for (int q = 0; q < nc; ++q) collide(c[q], x, y, z, f[4], f[5], f[6]);
}

// P = (P F^T) F^-T with P F^T = 2 mu (F F^T - sqrt(F F^T)) + lambda J (J-1) I
// (force_matrix with V_p0 = -1), F^-T from the transposed cofactors.
__global__ void k_stress(const double* rec, int64_t n, double mu0, double lambda0, double xi, double* P) {
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const double* p = rec + 26 * i;
  M3<double> F, FP;
  for (int e = 0; e < 9; ++e) {
    FP.a[e] = p[8 + e];
    F.a[e] = p[17 + e];
  }
  const double h = exp(xi * (1.0 - det3(FP)));
  const Sym3<double> S = force_matrix<double>(F, -1.0, mu0, lambda0, h);
  // cofactor matrix C: F^-T = C / det F
  M3<double> C;
  C(0, 0) = F(1, 1) * F(2, 2) - F(1, 2) * F(2, 1);
  C(0, 1) = F(1, 2) * F(2, 0) - F(1, 0) * F(2, 2);
  C(0, 2) = F(1, 0) * F(2, 1) - F(1, 1) * F(2, 0);
  C(1, 0) = F(0, 2) * F(2, 1) - F(0, 1) * F(2, 2);
  C(1, 1) = F(0, 0) * F(2, 2) - F(0, 2) * F(2, 0);
  C(1, 2) = F(0, 1) * F(2, 0) - F(0, 0) * F(2, 1);
  C(2, 0) = F(0, 1) * F(1, 2) - F(0, 2) * F(1, 1);
  C(2, 1) = F(0, 2) * F(1, 0) - F(0, 0) * F(1, 2);
  C(2, 2) = F(0, 0) * F(1, 1) - F(0, 1) * F(1, 0);
  const double inv_det = 1.0 / (F(0, 0) * C(0, 0) + F(0, 1) * C(0, 1) + F(0, 2) * C(0, 2));
  const double s[3][3] = {{S.xx, S.xy, S.xz}, {S.xy, S.yy, S.yz}, {S.xz, S.yz, S.zz}};
  double* out = P + 9 * i;
  for (int r = 0; r < 3; ++r)
    for (int c = 0; c < 3; ++c)
      out[c * 3 + r] = (s[r][0] * C(0, c) + s[r][1] * C(1, c) + s[r][2] * C(2, c)) * inv_det;
}

// forces[i][e] = (-V_p0 P F_E^T) gradient[i][e] (grid.cpp:176-180).
__global__ void k_force_scatter(const double* rec, int64_t n, const double* P, const double* grad, double* force) {
  const int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= n * 64) return;
  const int64_t i = t / 64;
  const double* p = rec + 26 * i;
  const double* Pi = P + 9 * i;
  const double V0 = p[7];
  double M[3][3];
  for (int r = 0; r < 3; ++r)
    for (int c = 0; c < 3; ++c) {
      double acc = 0.0;
      for (int k = 0; k < 3; ++k) acc += Pi[k * 3 + r] * p[17 + k * 3 + c];  // P(r,k) F_E(c,k)
      M[r][c] = -V0 * acc;
    }
  const double* g = grad + 3 * t;
  for (int r = 0; r < 3; ++r) force[3 * t + r] = M[r][0] * g[0] + M[r][1] * g[1] + M[r][2] * g[2];
}

// dP[i] = the differential of the fixed-corotated stress at F_E of particle
// i for dF[i] (corotated_differential; polar factors of F_E, hardening from
// F_P), matrices column-major.
__global__ void k_constitutive_differential(const double* rec, int64_t n, const double* dF, double mu0,
                                            double lambda0, double xi, double* dP, uint32_t* bad) {
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const double* p = rec + 26 * i;
  M3<double> F, FP, D;
  for (int e = 0; e < 9; ++e) {
    FP.a[e] = p[8 + e];
    F.a[e] = p[17 + e];
    D.a[e] = dF[9 * i + e];
  }
  M3<double> R;
  Sym3<double> S;
  if (!polar_factors(F, R, S)) {
    atomicOr(bad, 1u);
    return;
  }
  const double h = exp(xi * (1.0 - det3(FP)));
  const M3<double> out = corotated_differential(F, R, S, mu0 * h, lambda0 * h, D);
  for (int e = 0; e < 9; ++e) dP[9 * i + e] = out.a[e];
}

// dF[i] = dt (sum_e dv[i][e] grad[i][e]^T) F_E of particle i, over its 64
// stencil entries (the implicit update's deformation differential).
__global__ void k_deformation_differential(const double* rec, int64_t n, double dt, const double* grad,
                                           const double* dv, double* dF) {
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  double G[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0};  // column-major sum of dv grad^T
  for (int e = 0; e < 64; ++e) {
    const double* g = grad + 192 * i + 3 * e;
    const double* u = dv + 192 * i + 3 * e;
    for (int c = 0; c < 3; ++c)
      for (int r = 0; r < 3; ++r) G[c * 3 + r] += u[r] * g[c];
  }
  const double* F = rec + 26 * i + 17;
  for (int c = 0; c < 3; ++c)
    for (int r = 0; r < 3; ++r)
      dF[9 * i + c * 3 + r] = dt * (G[r] * F[c * 3] + G[3 + r] * F[c * 3 + 1] + G[6 + r] * F[c * 3 + 2]);
}

// axis_weights of every coordinate, in precision R (widened to double).
template <typename R>
__global__ void k_axis_weights(const double* x, int64_t n, double dx, int32_t* base, double* w, double* dw) {
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const AxisWeights<R> a = axis_weights((R)x[i], (R)dx);
  base[i] = a.base;
#pragma unroll
  for (int k = 0; k < 4; ++k) {
    w[4 * i + k] = (double)a.w[k];
    dw[4 * i + k] = (double)a.dw[k];
  }
}

// out[i][e] = (m w, m v w) for stencil weight w = weights[i][e] (grid.cpp:121-127).
__global__ void k_p2g_stencil(const double* rec, int64_t n, const double* weights, double* out) {
  const int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= n * 64) return;
  const double* p = rec + 26 * (t / 64);
  const double w = weights[t], m = p[6];
  out[4 * t] = w * m;
  for (int a = 0; a < 3; ++a) out[4 * t + 1 + a] = w * (m * p[3 + a]);
}

__global__ void k_particle_collide(double* rec, int64_t n, const Collider* c, int nc) {
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  double* p = rec + 26 * i;
  for (int q = 0; q < nc; ++q) collide(c[q], p[0], p[1], p[2], p[3], p[4], p[5]);
}

__global__ void k_advect(double* rec, int64_t n, double dt) {
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  double* p = rec + 26 * i;
  for (int a = 0; a < 3; ++a) p[a] = p[a] + dt * p[3 + a];
}

unsigned blocks_for(int64_t n) { return (unsigned)((n + 255) / 256); }

template <typename F>
int guarded(F&& f) {
  try {
    f();
    return SNOW_OK;
  } catch (const Error& e) {
    return set_error(e.code, e.what());
  } catch (const std::exception& e) {
    return set_error(SNOW_E_ARG, e.what());
  }
}

void check_records(const double* rec, int64_t n) {
  if (n < 0 || (n > 0 && !rec)) throw Error(SNOW_E_ARG, "bad particle array");
}

snow_step_params stage_params(double dx) {
  if (!(dx > 0.0)) throw Error(SNOW_E_ARG, "grid_spacing must be positive");
  snow_step_params p{};
  p.grid_spacing = dx;
  return p;
}

// calculate_volume / stress_update / G2P against a host grid.
void gather_stage(const int32_t* ijk, const double* fields, int64_t n_nodes, double* rec, int64_t n,
                  const snow_step_params& p, int load_mode, int g2p_mode) {
  check_records(rec, n);
  if (n == 0) return;
  if (n_nodes < 0 || (n_nodes > 0 && (!ijk || !fields))) throw Error(SNOW_E_ARG, "bad node list");
  StageGrid sg(rec, n, p);
  StepLaunch<double>::zero_grid(sg.b, nullptr);
  k_zero_vel<<<4 * sm_count(), 256>>>(sg.b);
  if (n_nodes > 0) {
    DBuf<int32_t> dijk((size_t)n_nodes * 3);
    DBuf<double> df((size_t)n_nodes * 10);
    check_cuda(cudaMemcpy(dijk.p, ijk, n_nodes * 3 * sizeof(int32_t), cudaMemcpyHostToDevice), "nodes");
    check_cuda(cudaMemcpy(df.p, fields, n_nodes * 10 * sizeof(double), cudaMemcpyHostToDevice), "nodes");
    k_load_nodes<<<blocks_for(n_nodes), 256>>>(sg.b, dijk.p, df.p, n_nodes, load_mode);
    check_cuda(cudaDeviceSynchronize(), "load nodes");
  }
  StepLaunch<double>::g2p(sg.b, g2p_mode, nullptr);
  StepLaunch<double>::zero_grid(sg.b, nullptr);
  check_cuda(cudaGetLastError(), "stage g2p");
  sg.finish_checked();
  sg.batch.download(sg.id, rec, n, nullptr);
}

std::vector<Collider> to_colliders(const snow_collider* c, int nc) { return device_colliders(c, nc); }

}  // namespace
}  // namespace snow

using namespace snow;

extern "C" {

int snow_gpu_stage_p2g(const double* records, int64_t n, double grid_spacing, int32_t* ijk,
                       double* fields, int64_t cap_nodes, int64_t* n_nodes) {
  return guarded([&] {
    check_records(records, n);
    if (n_nodes) *n_nodes = 0;
    if (n == 0) return;
    StageGrid sg(records, n, stage_params(grid_spacing));
    StepLaunch<double>::p2g(sg.b, P2G_MASS_MOMENTUM, nullptr);
    check_cuda(cudaDeviceSynchronize(), "stage p2g");
    sg.export_nodes(ijk, fields, cap_nodes, n_nodes);
  });
}

int snow_gpu_stage_force(const double* records, int64_t n, double grid_spacing, double mu_0,
                         double lambda_0, double hardening_coefficient, int32_t* ijk,
                         double* fields, int64_t cap_nodes, int64_t* n_nodes) {
  return guarded([&] {
    check_records(records, n);
    if (n_nodes) *n_nodes = 0;
    if (n == 0) return;
    snow_step_params p = stage_params(grid_spacing);
    p.mu_0 = mu_0;
    p.lambda_0 = lambda_0;
    p.hardening_coefficient = hardening_coefficient;
    StageGrid sg(records, n, p);
    StepLaunch<double>::p2g(sg.b, P2G_FORCE, nullptr);
    check_cuda(cudaDeviceSynchronize(), "stage force");
    sg.export_nodes(ijk, fields, cap_nodes, n_nodes);
  });
}

int snow_gpu_stage_p2g_stencil(const double* records, int64_t n, const double* weights, double* out) {
  return guarded([&] {
    check_records(records, n);
    if (n > 0 && (!weights || !out)) throw Error(SNOW_E_ARG, "NULL argument");
    if (n == 0) return;
    DBuf<double> d((size_t)n * 26), dw((size_t)n * 64), dout((size_t)n * 256);
    check_cuda(cudaMemcpy(d.p, records, n * 208, cudaMemcpyHostToDevice), "records");
    check_cuda(cudaMemcpy(dw.p, weights, n * 64 * 8, cudaMemcpyHostToDevice), "weights");
    k_p2g_stencil<<<blocks_for(n * 64), 256>>>(d.p, n, dw.p, dout.p);
    check_cuda(cudaGetLastError(), "p2g stencil");
    check_cuda(cudaMemcpy(out, dout.p, n * 256 * 8, cudaMemcpyDeviceToHost), "contributions");
  });
}

int snow_gpu_stage_stress(const double* records, int64_t n, double mu_0, double lambda_0,
                          double hardening_coefficient, double* P_out) {
  return guarded([&] {
    check_records(records, n);
    if (n > 0 && !P_out) throw Error(SNOW_E_ARG, "P_out is NULL");
    if (n == 0) return;
    DBuf<double> d((size_t)n * 26), dp((size_t)n * 9);
    check_cuda(cudaMemcpy(d.p, records, n * 208, cudaMemcpyHostToDevice), "records");
    k_stress<<<blocks_for(n), 256>>>(d.p, n, mu_0, lambda_0, hardening_coefficient, dp.p);
    check_cuda(cudaGetLastError(), "stress");
    check_cuda(cudaMemcpy(P_out, dp.p, n * 72, cudaMemcpyDeviceToHost), "stress out");
  });
}

int snow_gpu_stage_constitutive_differential(const double* records, int64_t n, const double* dF, double mu_0,
                                             double lambda_0, double hardening_coefficient, double* dP) {
  return guarded([&] {
    check_records(records, n);
    if (n > 0 && (!dF || !dP)) throw Error(SNOW_E_ARG, "NULL argument");
    if (n == 0) return;
    DBuf<double> d((size_t)n * 26), din((size_t)n * 9), dout((size_t)n * 9);
    DBuf<uint32_t> bad(1);
    check_cuda(cudaMemset(bad.p, 0, sizeof(uint32_t)), "flag");
    check_cuda(cudaMemcpy(d.p, records, n * 208, cudaMemcpyHostToDevice), "records");
    check_cuda(cudaMemcpy(din.p, dF, n * 72, cudaMemcpyHostToDevice), "dF");
    k_constitutive_differential<<<blocks_for(n), 256>>>(d.p, n, din.p, mu_0, lambda_0, hardening_coefficient,
                                                         dout.p, bad.p);
    check_cuda(cudaGetLastError(), "constitutive differential");
    uint32_t flag = 0;
    check_cuda(cudaMemcpy(&flag, bad.p, sizeof flag, cudaMemcpyDeviceToHost), "flag");
    if (flag) throw Error(SNOW_E_ARG, "constitutive_differential: a singular F_E");
    check_cuda(cudaMemcpy(dP, dout.p, n * 72, cudaMemcpyDeviceToHost), "dP");
  });
}

int snow_gpu_stage_deformation_differential(const double* records, int64_t n, double time_step,
                                            const double* gradients, const double* delta_v, double* dF) {
  return guarded([&] {
    check_records(records, n);
    if (n > 0 && (!gradients || !delta_v || !dF)) throw Error(SNOW_E_ARG, "NULL argument");
    if (n == 0) return;
    DBuf<double> d((size_t)n * 26), dg((size_t)n * 192), du((size_t)n * 192), dout((size_t)n * 9);
    check_cuda(cudaMemcpy(d.p, records, n * 208, cudaMemcpyHostToDevice), "records");
    check_cuda(cudaMemcpy(dg.p, gradients, n * 192 * 8, cudaMemcpyHostToDevice), "gradients");
    check_cuda(cudaMemcpy(du.p, delta_v, n * 192 * 8, cudaMemcpyHostToDevice), "delta_v");
    k_deformation_differential<<<blocks_for(n), 256>>>(d.p, n, time_step, dg.p, du.p, dout.p);
    check_cuda(cudaGetLastError(), "deformation differential");
    check_cuda(cudaMemcpy(dF, dout.p, n * 72, cudaMemcpyDeviceToHost), "dF");
  });
}

int snow_gpu_stage_force_scatter(const double* records, int64_t n, const double* P, const double* gradients,
                                 double* forces) {
  return guarded([&] {
    check_records(records, n);
    if (n > 0 && (!P || !gradients || !forces)) throw Error(SNOW_E_ARG, "NULL argument");
    if (n == 0) return;
    DBuf<double> d((size_t)n * 26), dp((size_t)n * 9), dg((size_t)n * 192), df((size_t)n * 192);
    check_cuda(cudaMemcpy(d.p, records, n * 208, cudaMemcpyHostToDevice), "records");
    check_cuda(cudaMemcpy(dp.p, P, n * 72, cudaMemcpyHostToDevice), "P");
    check_cuda(cudaMemcpy(dg.p, gradients, n * 192 * 8, cudaMemcpyHostToDevice), "gradients");
    k_force_scatter<<<blocks_for(n * 64), 256>>>(d.p, n, dp.p, dg.p, df.p);
    check_cuda(cudaGetLastError(), "force scatter");
    check_cuda(cudaMemcpy(forces, df.p, n * 192 * 8, cudaMemcpyDeviceToHost), "forces");
  });
}

int snow_gpu_stage_grid_velocity(double* fields, int64_t n_nodes, const double gravity[3], double time_step) {
  return guarded([&] {
    if (n_nodes < 0 || (n_nodes > 0 && !fields) || !gravity) throw Error(SNOW_E_ARG, "bad node list");
    if (n_nodes == 0) return;
    DBuf<double> df((size_t)n_nodes * 10);
    check_cuda(cudaMemcpy(df.p, fields, n_nodes * 80, cudaMemcpyHostToDevice), "nodes");
    k_grid_velocity_nodes<<<blocks_for(n_nodes), 256>>>(df.p, n_nodes, gravity[0], gravity[1], gravity[2], time_step);
    check_cuda(cudaGetLastError(), "grid velocity");
    check_cuda(cudaMemcpy(fields, df.p, n_nodes * 80, cudaMemcpyDeviceToHost), "nodes");
  });
}

int snow_gpu_stage_grid_collisions(const int32_t* ijk, double* fields, int64_t n_nodes,
                                   const snow_collider* colliders, int n_colliders, double grid_spacing) {
  return guarded([&] {
    if (n_nodes < 0 || (n_nodes > 0 && (!fields || !ijk))) throw Error(SNOW_E_ARG, "bad node list");
    auto c = to_colliders(colliders, n_colliders);
    if (n_nodes == 0 || c.empty()) return;
    DBuf<double> df((size_t)n_nodes * 10);
    DBuf<int32_t> dijk((size_t)n_nodes * 3);
    DBuf<Collider> dc(c.size());
    check_cuda(cudaMemcpy(df.p, fields, n_nodes * 80, cudaMemcpyHostToDevice), "nodes");
    check_cuda(cudaMemcpy(dijk.p, ijk, n_nodes * 12, cudaMemcpyHostToDevice), "nodes");
    check_cuda(cudaMemcpy(dc.p, c.data(), c.size() * sizeof(Collider), cudaMemcpyHostToDevice), "colliders");
    k_grid_collide_nodes<<<blocks_for(n_nodes), 256>>>(dijk.p, df.p, n_nodes, dc.p, (int)c.size(), grid_spacing);
    check_cuda(cudaGetLastError(), "grid collisions");
    check_cuda(cudaMemcpy(fields, df.p, n_nodes * 80, cudaMemcpyDeviceToHost), "nodes");
  });
}

int snow_gpu_stage_volume(const int32_t* ijk, const double* fields, int64_t n_nodes, double* records,
                          int64_t n, double grid_spacing) {
  return guarded([&] {
    gather_stage(ijk, fields, n_nodes, records, n, stage_params(grid_spacing), 0, G2P_VOLUME);
  });
}

int snow_gpu_stage_stress_update(const int32_t* ijk, const double* fields, int64_t n_nodes,
                                 double* records, int64_t n, double grid_spacing, double time_step,
                                 double max_compression, double max_stretch) {
  return guarded([&] {
    snow_step_params p = stage_params(grid_spacing);
    p.time_step = time_step;
    p.max_compression = max_compression;
    p.max_stretch = max_stretch;
    gather_stage(ijk, fields, n_nodes, records, n, p, 1, G2P_STRESS);
  });
}

int snow_gpu_stage_g2p(const int32_t* ijk, const double* fields, int64_t n_nodes, double* records,
                       int64_t n, double grid_spacing, double alpha) {
  return guarded([&] {
    snow_step_params p = stage_params(grid_spacing);
    p.alpha = alpha;
    gather_stage(ijk, fields, n_nodes, records, n, p, 2, G2P_VELOCITY);
  });
}

int snow_gpu_stage_particle_collisions(double* records, int64_t n, const snow_collider* colliders,
                                       int n_colliders) {
  return guarded([&] {
    check_records(records, n);
    auto c = to_colliders(colliders, n_colliders);
    if (n == 0 || c.empty()) return;
    DBuf<double> d((size_t)n * 26);
    DBuf<Collider> dc(c.size());
    check_cuda(cudaMemcpy(d.p, records, n * 208, cudaMemcpyHostToDevice), "records");
    check_cuda(cudaMemcpy(dc.p, c.data(), c.size() * sizeof(Collider), cudaMemcpyHostToDevice), "colliders");
    k_particle_collide<<<blocks_for(n), 256>>>(d.p, n, dc.p, (int)c.size());
    check_cuda(cudaGetLastError(), "particle collisions");
    check_cuda(cudaMemcpy(records, d.p, n * 208, cudaMemcpyDeviceToHost), "records");
  });
}

int snow_gpu_stage_weights(const double* x, int64_t n, double grid_spacing, int precision, int32_t* base,
                           double* w, double* dw) {
  return guarded([&] {
    if (n < 0 || (n > 0 && (!x || !base || !w || !dw))) throw Error(SNOW_E_ARG, "NULL argument");
    if (!(grid_spacing > 0.0)) throw Error(SNOW_E_ARG, "grid_spacing must be positive");
    if (precision != SNOW_FP64 && precision != SNOW_MIXED) throw Error(SNOW_E_ARG, "unknown precision");
    if (n == 0) return;
    DBuf<double> dx_((size_t)n), dw_((size_t)n * 4), ddw((size_t)n * 4);
    DBuf<int32_t> db((size_t)n);
    check_cuda(cudaMemcpy(dx_.p, x, n * sizeof(double), cudaMemcpyHostToDevice), "x");
    if (precision == SNOW_FP64)
      k_axis_weights<double><<<blocks_for(n), 256>>>(dx_.p, n, grid_spacing, db.p, dw_.p, ddw.p);
    else
      k_axis_weights<float><<<blocks_for(n), 256>>>(dx_.p, n, grid_spacing, db.p, dw_.p, ddw.p);
    check_cuda(cudaGetLastError(), "weights");
    check_cuda(cudaMemcpy(base, db.p, n * sizeof(int32_t), cudaMemcpyDeviceToHost), "base");
    check_cuda(cudaMemcpy(w, dw_.p, n * 4 * sizeof(double), cudaMemcpyDeviceToHost), "w");
    check_cuda(cudaMemcpy(dw, ddw.p, n * 4 * sizeof(double), cudaMemcpyDeviceToHost), "dw");
  });
}

int snow_gpu_stage_position_update(double* records, int64_t n, double time_step) {
  return guarded([&] {
    check_records(records, n);
    if (n == 0) return;
    DBuf<double> d((size_t)n * 26);
    check_cuda(cudaMemcpy(d.p, records, n * 208, cudaMemcpyHostToDevice), "records");
    k_advect<<<blocks_for(n), 256>>>(d.p, n, time_step);
    check_cuda(cudaGetLastError(), "position update");
    check_cuda(cudaMemcpy(records, d.p, n * 208, cudaMemcpyDeviceToHost), "records");
  });
}

}  // extern "C"
