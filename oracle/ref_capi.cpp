// ORACLE (reference build) -- test infrastructure only.
// Flat C entry points over the REFERENCE solver's own functions (src/grid.cpp,
// src/collision.cpp, src/import.cpp, src/export.cpp compiled unmodified from the
// reference tree by oracle/Makefile, against the project's Eigen-subset shim in
// place of Eigen3, which is not installed on this image).  Used by the tests to
// pin the oracle restatement and by bench.py's reference arm as the CPU baseline.
// Particles travel as 26-double records in the reference's struct Particle order.
// Step calls report the ten StepTimings stages and, in slot 10, the wall time
// of the step loop (milliseconds).
#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <stdexcept>
#include <string>
#include <vector>

#include "snow/collision.hpp"
#include "snow/debug.hpp"
#include "snow/export.hpp"
#include "snow/grid.hpp"
#include "snow/import.hpp"
#include "snow/particle.hpp"

static_assert(sizeof(Particle) == 208, "reference Particle must be 26 packed doubles");

namespace {
std::vector<Particle> to_vec(const double* rec, int64_t n) {
  std::vector<Particle> v;
  v.reserve((std::size_t)n);
  for (int64_t i = 0; i < n; ++i) {
    v.emplace_back(Eigen::Vector3d::Zero(), Eigen::Vector3d::Zero(), 0.0, 0.0);
    std::memcpy(static_cast<void*>(&v.back()), rec + 26 * i, sizeof(Particle));
  }
  return v;
}
void from_vec(const std::vector<Particle>& v, double* rec) {
  for (std::size_t i = 0; i < v.size(); ++i)
    std::memcpy(rec + 26 * i, static_cast<const void*>(&v[i]), sizeof(Particle));
}
std::vector<CollisionBody> planes(const double* q, int n) {
  std::vector<CollisionBody> b;
  for (int i = 0; i < n; ++i, q += 7)
    b.push_back(make_plane({q[0], q[1], q[2]}, {q[3], q[4], q[5]}, q[6]));
  return b;
}
// Solid oriented box (centre p, axes u, w, u x w, half extents h) as a user of
// the reference would write it: the point in the box's axes l, q_k = |l_k| -
// h_k; phi = |max(q, 0)| + min(max q, 0); normal inside = outward normal of
// the face with the largest q_k (first on a tie, + side at l_k = 0), outside =
// the normalised gradient of phi.
struct BoxFrame {
  Eigen::Vector3d p, ax[3], h;
  void local(const Eigen::Vector3d& x, double l[3], double q[3]) const {
    for (int k = 0; k < 3; ++k) {
      l[k] = ax[k].dot(x - p);
      q[k] = std::abs(l[k]) - h[k];
    }
  }
};
CollisionBody box_body(const BoxFrame& f, const Eigen::Vector3d& v, double mu) {
  return CollisionBody{[f](const Eigen::Vector3d& x) {
                         double l[3], q[3], out2 = 0.0;
                         f.local(x, l, q);
                         for (double e : q) out2 += e > 0.0 ? e * e : 0.0;
                         return std::sqrt(out2) + std::min(std::max(q[0], std::max(q[1], q[2])), 0.0);
                       },
                       [f](const Eigen::Vector3d& x) {
                         double l[3], q[3];
                         f.local(x, l, q);
                         int k = 0;
                         for (int a = 1; a < 3; ++a)
                           if (q[a] > q[k]) k = a;
                         if (q[k] <= 0.0) return Eigen::Vector3d((l[k] < 0.0 ? -1.0 : 1.0) * f.ax[k]);
                         Eigen::Vector3d g = Eigen::Vector3d::Zero();
                         for (int a = 0; a < 3; ++a)
                           if (q[a] > 0.0) g = g + (l[a] < 0.0 ? -q[a] : q[a]) * f.ax[a];
                         return Eigen::Vector3d(g.normalized());
                       },
                       [v](const Eigen::Vector3d&) { return v; }, mu};
}

// Bodies as n x 18 rows: kind, point[3], normal[3], velocity[3], friction,
// radius, axis[3], half extents[3].  A resting plane is the reference's own
// make_plane; a moving plane, a solid sphere and an oriented box are
// CollisionBody values with their phi / normal / velocity functions written
// out, as a user of the reference would.
std::vector<CollisionBody> bodies(const double* q, int n) {
  std::vector<CollisionBody> b;
  for (int i = 0; i < n; ++i, q += 18) {
    const Eigen::Vector3d p{q[1], q[2], q[3]}, nrm{q[4], q[5], q[6]}, v{q[7], q[8], q[9]};
    const double mu = q[10], r = q[11];
    if (q[0] == 2.0) {
      BoxFrame f;
      f.p = p;
      f.ax[0] = nrm;
      f.ax[1] = Eigen::Vector3d{q[12], q[13], q[14]};
      f.ax[2] = Eigen::Vector3d{nrm[1] * q[14] - nrm[2] * q[13], nrm[2] * q[12] - nrm[0] * q[14],
                                nrm[0] * q[13] - nrm[1] * q[12]};
      f.h = Eigen::Vector3d{q[15], q[16], q[17]};
      b.push_back(box_body(f, v, mu));
    } else if (q[0] == 1.0) {
      b.push_back(CollisionBody{[p, r](const Eigen::Vector3d& x) { return (x - p).norm() - r; },
                                [p](const Eigen::Vector3d& x) { return Eigen::Vector3d((x - p).normalized()); },
                                [v](const Eigen::Vector3d&) { return v; }, mu});
    } else if (v[0] == 0.0 && v[1] == 0.0 && v[2] == 0.0) {
      b.push_back(make_plane(p, nrm, mu));
    } else {
      const Eigen::Vector3d u = nrm.normalized();
      b.push_back(CollisionBody{[p, u](const Eigen::Vector3d& x) { return u.dot(x - p); },
                                [u](const Eigen::Vector3d&) { return u; },
                                [v](const Eigen::Vector3d&) { return v; }, mu});
    }
  }
  return b;
}
thread_local std::string g_err;
}  // namespace

extern "C" {

void ref_setup(double* rec, int64_t n, double dx) {
  auto v = to_vec(rec, n);
  setup(v, dx);
  from_vec(v, rec);
}

// params: gravity[3], dt, dx, mu0, lambda0, xi, theta_c, theta_s, alpha
static void run(double* rec, int64_t n, const double* p, const std::vector<CollisionBody>& bodies, int steps,
                double* stage_ms) {
  auto v = to_vec(rec, n);
  std::vector<ParticleStencil> stencils(v.size());
  StepTimings t;
  const auto t0 = std::chrono::steady_clock::now();
  for (int s = 0; s < steps; ++s)
    step(v, bodies, stencils, Eigen::Vector3d{p[0], p[1], p[2]}, p[3], p[4], p[5], p[6], p[7],
         p[8], p[9], p[10], t);
  const double wall = std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
  if (stage_ms) {
    stage_ms[10] = wall;
    const double ms[10] = {t.stencil, t.p2g, t.forces_constitutive, t.forces_accumulative,
                           t.grid_velocity, t.grid_collisions, t.stress_update, t.g2p,
                           t.particle_collisions, t.position_update};
    std::memcpy(stage_ms, ms, sizeof ms);
  }
  from_vec(v, rec);
}

void ref_step(double* rec, int64_t n, const double* p, const double* plane_data, int n_planes,
              int steps, double* stage_ms) {
  run(rec, n, p, planes(plane_data, n_planes), steps, stage_ms);
}
void ref_step_bodies(double* rec, int64_t n, const double* p, const double* body_rows, int n_bodies,
                     int steps, double* stage_ms) {
  run(rec, n, p, bodies(body_rows, n_bodies), steps, stage_ms);
}

// Two calls: with out == nullptr returns the particle count, else fills `out`
// (capacity records).  Returns -1 and keeps the exception text on error.
int64_t ref_import(const char* groups, const char* particles, double* out, int64_t capacity) {
  try {
    auto v = import_particles(groups, particles);
    if (out) {
      if ((int64_t)v.size() > capacity) return -2;
      from_vec(v, out);
    }
    return (int64_t)v.size();
  } catch (const std::exception& e) {
    g_err = e.what();
    return -1;
  }
}
const char* ref_last_error(void) { return g_err.c_str(); }

void ref_export(const double* rec, int64_t n, int frame) { export_particles(to_vec(rec, n), frame); }

}  // extern "C"
