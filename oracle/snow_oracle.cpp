// ORACLE -- test infrastructure only.  Nothing in the product links, loads or calls
// this file: it is the CPU checker that tests/, __graft_entry__.smoke() and the
// cpu_baseline leg of bench.py compare the CUDA path against.
//
// A plain C++20 restatement (no Eigen) of the explicit MPM snow step of the
// reference solver, src/grid.cpp, src/collision.cpp.  Every function cites the
// reference lines it follows.  Data structures mirror the reference on purpose:
// a fresh std::unordered_map grid per step, a 64-entry stencil per particle with
// cached node pointers, the same stage order and the same three OpenMP loops
// (stencil build, stress update, G2P; the rest serial), so that the oracle also
// serves as the "port" CPU baseline.
//
// Own linear algebra: column-major Vec3/Mat3 and a two-sided Jacobi SVD
// (Forsythe-Henrici / Brent-Luk-Van Loan: each 2x2 pivot block is first made
// symmetric by a left plane rotation, then diagonalised by a symmetric Jacobi
// rotation; Golub & Van Loan, Matrix Computations, 4th ed., 8.6.3).  Singular
// values are made non-negative (sign moved into U), matching what Eigen's
// JacobiSVD reports; R = U V^T and U clamp(S) V^T are then unique for
// non-singular input, which is all the step uses.
//
// Parity is pinned by (a) the reference's 24 known-answer unit tests
// (tests/snow_tests.cpp), restated in oracle/oracle_tests.cpp, and (b) the
// reference's own sources compiled against the project's Eigen-subset shim
// (oracle/_ref, built by oracle/Makefile) run on the same inputs.
#include <algorithm>
#include <array>
#include <chrono>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <limits>
#include <unordered_map>
#include <vector>

namespace oracle {

struct Vec3 {
  double v[3] = {0.0, 0.0, 0.0};
  Vec3() = default;
  Vec3(double a, double b, double c) : v{a, b, c} {}
  double& operator[](int i) { return v[i]; }
  double operator[](int i) const { return v[i]; }
};
inline Vec3 operator+(const Vec3& a, const Vec3& b) { return {a[0] + b[0], a[1] + b[1], a[2] + b[2]}; }
inline Vec3 operator-(const Vec3& a, const Vec3& b) { return {a[0] - b[0], a[1] - b[1], a[2] - b[2]}; }
inline Vec3 operator*(double s, const Vec3& a) { return {s * a[0], s * a[1], s * a[2]}; }
inline Vec3 operator/(const Vec3& a, double s) { return {a[0] / s, a[1] / s, a[2] / s}; }
inline Vec3& operator+=(Vec3& a, const Vec3& b) {
  a[0] += b[0];
  a[1] += b[1];
  a[2] += b[2];
  return a;
}
inline double dot(const Vec3& a, const Vec3& b) { return a[0] * b[0] + a[1] * b[1] + a[2] * b[2]; }
inline double norm(const Vec3& a) { return std::sqrt(dot(a, a)); }

// Column-major 3x3: element (r, c) is a[c * 3 + r] (the layout of the reference's
// Eigen::Matrix3d inside a Particle record).
struct Mat3 {
  double a[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0};
  double& operator()(int r, int c) { return a[c * 3 + r]; }
  double operator()(int r, int c) const { return a[c * 3 + r]; }
  static Mat3 identity() {
    Mat3 m;
    m(0, 0) = m(1, 1) = m(2, 2) = 1.0;
    return m;
  }
};
inline Mat3 operator*(const Mat3& x, const Mat3& y) {
  Mat3 m;
  for (int r = 0; r < 3; ++r)
    for (int c = 0; c < 3; ++c) {
      double s = 0.0;
      for (int k = 0; k < 3; ++k) s += x(r, k) * y(k, c);
      m(r, c) = s;
    }
  return m;
}
inline Vec3 operator*(const Mat3& x, const Vec3& y) {
  Vec3 o;
  for (int r = 0; r < 3; ++r) o[r] = x(r, 0) * y[0] + x(r, 1) * y[1] + x(r, 2) * y[2];
  return o;
}
inline Mat3 operator*(double s, const Mat3& x) {
  Mat3 m;
  for (int i = 0; i < 9; ++i) m.a[i] = s * x.a[i];
  return m;
}
inline Mat3 operator+(const Mat3& x, const Mat3& y) {
  Mat3 m;
  for (int i = 0; i < 9; ++i) m.a[i] = x.a[i] + y.a[i];
  return m;
}
inline Mat3 operator-(const Mat3& x, const Mat3& y) {
  Mat3 m;
  for (int i = 0; i < 9; ++i) m.a[i] = x.a[i] - y.a[i];
  return m;
}
inline Mat3 transpose(const Mat3& x) {
  Mat3 m;
  for (int r = 0; r < 3; ++r)
    for (int c = 0; c < 3; ++c) m(c, r) = x(r, c);
  return m;
}
inline Mat3 outer(const Vec3& a, const Vec3& b) {
  Mat3 m;
  for (int r = 0; r < 3; ++r)
    for (int c = 0; c < 3; ++c) m(r, c) = a[r] * b[c];
  return m;
}
inline Mat3 diag(const Vec3& d) {
  Mat3 m;
  m(0, 0) = d[0];
  m(1, 1) = d[1];
  m(2, 2) = d[2];
  return m;
}
// Cofactor expansion along the first row.
inline double det(const Mat3& m) {
  return m(0, 0) * (m(1, 1) * m(2, 2) - m(1, 2) * m(2, 1)) -
         m(0, 1) * (m(1, 0) * m(2, 2) - m(1, 2) * m(2, 0)) +
         m(0, 2) * (m(1, 0) * m(2, 1) - m(1, 1) * m(2, 0));
}
// Transposed cofactor matrix over the determinant.
inline Mat3 inverse(const Mat3& m) {
  Mat3 c;
  c(0, 0) = m(1, 1) * m(2, 2) - m(1, 2) * m(2, 1);
  c(1, 0) = m(1, 2) * m(2, 0) - m(1, 0) * m(2, 2);
  c(2, 0) = m(1, 0) * m(2, 1) - m(1, 1) * m(2, 0);
  c(0, 1) = m(0, 2) * m(2, 1) - m(0, 1) * m(2, 2);
  c(1, 1) = m(0, 0) * m(2, 2) - m(0, 2) * m(2, 0);
  c(2, 1) = m(0, 1) * m(2, 0) - m(0, 0) * m(2, 1);
  c(0, 2) = m(0, 1) * m(1, 2) - m(0, 2) * m(1, 1);
  c(1, 2) = m(0, 2) * m(1, 0) - m(0, 0) * m(1, 2);
  c(2, 2) = m(0, 0) * m(1, 1) - m(0, 1) * m(1, 0);
  const double d = m(0, 0) * c(0, 0) + m(0, 1) * c(1, 0) + m(0, 2) * c(2, 0);
  return (1.0 / d) * c;
}
inline double frob(const Mat3& m) {
  double s = 0.0;
  for (double x : m.a) s += x * x;
  return std::sqrt(s);
}

// Two-sided Jacobi SVD of a 3x3 matrix: F = U diag(s) V^T with s >= 0, sorted
// in decreasing order.  Stands in for Eigen::JacobiSVD (reference grid.cpp:168,279).
void svd3(const Mat3& F, Mat3& U, Vec3& s, Mat3& V) {
  Mat3 A = F;
  U = Mat3::identity();
  V = Mat3::identity();
  const double eps = std::numeric_limits<double>::epsilon();
  const double tiny = std::numeric_limits<double>::min();
  static const int pairs[3][2] = {{0, 1}, {0, 2}, {1, 2}};
  for (int sweep = 0; sweep < 64; ++sweep) {
    bool changed = false;
    for (const auto& pq : pairs) {
      const int p = pq[0], q = pq[1];
      const double dmax = std::max(std::abs(A(p, p)), std::abs(A(q, q)));
      const double thresh = std::max(tiny, 2.0 * eps * dmax);
      if (std::abs(A(p, q)) <= thresh && std::abs(A(q, p)) <= thresh) continue;
      changed = true;
      // 1) left rotation G1 = [c1 -s1; s1 c1] with G1^T B symmetric.
      const double a = A(p, p), b = A(p, q), c = A(q, p), d = A(q, q);
      const double theta = std::atan2(c - b, a + d);
      const double c1 = std::cos(theta), s1 = std::sin(theta);
      const double m00 = c1 * a + s1 * c;
      const double m01 = c1 * b + s1 * d;
      const double m11 = -s1 * b + c1 * d;
      // 2) symmetric Jacobi rotation J = [c2 s2; -s2 c2] with J^T M J diagonal.
      double c2 = 1.0, s2 = 0.0;
      if (m01 != 0.0) {
        const double tau = (m11 - m00) / (2.0 * m01);
        double t;
        if (std::abs(tau) > 1e150)
          t = 1.0 / (2.0 * tau);
        else
          t = std::copysign(1.0, tau) / (std::abs(tau) + std::sqrt(1.0 + tau * tau));
        c2 = 1.0 / std::sqrt(1.0 + t * t);
        s2 = t * c2;
      }
      // B = G1 J D J^T: left factor L = G1 J, right factor J.
      double L[2][2], Rr[2][2];
      // G1 = [[c1, -s1],[s1, c1]], J = [[c2, s2],[-s2, c2]]
      L[0][0] = c1 * c2 + s1 * s2;
      L[0][1] = c1 * s2 - s1 * c2;
      L[1][0] = s1 * c2 - c1 * s2;
      L[1][1] = s1 * s2 + c1 * c2;
      Rr[0][0] = c2;
      Rr[0][1] = s2;
      Rr[1][0] = -s2;
      Rr[1][1] = c2;
      // A <- L^T A (rows p, q) ; U <- U L (cols p, q)
      for (int k = 0; k < 3; ++k) {
        const double ap = A(p, k), aq = A(q, k);
        A(p, k) = L[0][0] * ap + L[1][0] * aq;
        A(q, k) = L[0][1] * ap + L[1][1] * aq;
        const double up = U(k, p), uq = U(k, q);
        U(k, p) = up * L[0][0] + uq * L[1][0];
        U(k, q) = up * L[0][1] + uq * L[1][1];
      }
      // A <- A R (cols p, q) ; V <- V R (cols p, q)
      for (int k = 0; k < 3; ++k) {
        const double ap = A(k, p), aq = A(k, q);
        A(k, p) = ap * Rr[0][0] + aq * Rr[1][0];
        A(k, q) = ap * Rr[0][1] + aq * Rr[1][1];
        const double vp = V(k, p), vq = V(k, q);
        V(k, p) = vp * Rr[0][0] + vq * Rr[1][0];
        V(k, q) = vp * Rr[0][1] + vq * Rr[1][1];
      }
      A(p, q) = 0.0;
      A(q, p) = 0.0;
    }
    if (!changed) break;
  }
  // Non-negative singular values: move signs into U.
  double sv[3];
  for (int i = 0; i < 3; ++i) {
    sv[i] = A(i, i);
    if (sv[i] < 0.0) {
      sv[i] = -sv[i];
      for (int k = 0; k < 3; ++k) U(k, i) = -U(k, i);
    }
  }
  int order[3] = {0, 1, 2};
  std::sort(order, order + 3, [&](int i, int j) { return sv[i] > sv[j]; });
  Mat3 U2, V2;
  for (int c = 0; c < 3; ++c) {
    s[c] = sv[order[c]];
    for (int k = 0; k < 3; ++k) {
      U2(k, c) = U(k, order[c]);
      V2(k, c) = V(k, order[c]);
    }
  }
  U = U2;
  V = V2;
}

// ---------------------------------------------------------------- grid types
// GridIndex / GridNode / Grid: include/snow/grid.hpp:11-72 (the unused node
// fields density, delta_v, delta_force and colision_constrained are dropped).
struct NodeIdx {
  int i, j, k;
  bool operator==(const NodeIdx& o) const { return i == o.i && j == o.j && k == o.k; }
};
struct NodeIdxHash {
  std::size_t operator()(const NodeIdx& n) const noexcept {
    uint64_t h = (uint64_t)(uint32_t)n.i * 0x9E3779B185EBCA87ull;
    h ^= (uint64_t)(uint32_t)n.j * 0xC2B2AE3D27D4EB4Full + (h << 7) + (h >> 3);
    h ^= (uint64_t)(uint32_t)n.k * 0x165667B19E3779F9ull + (h << 11) + (h >> 5);
    return (std::size_t)(h ^ (h >> 29));
  }
};
struct Node {
  double mass = 0.0;
  Vec3 momentum, velocity, force;
  Vec3 delta_v, delta_force;  // the implicit update's Krylov vector and its force differential
};
using Grid = std::unordered_map<NodeIdx, Node, NodeIdxHash>;

// Particle record, 26 doubles / 208 bytes in the order of the reference's
// struct Particle (include/snow/particle.hpp:5-28): x_p, v_p, m_p, V_p0, F_P, F_E.
struct Particle {
  Vec3 x, v;
  double m, V0;
  Mat3 FP, FE;
};
static_assert(sizeof(Particle) == 208, "particle record layout");

struct StencilEntry {
  NodeIdx index;
  double weight = 0.0;
  Vec3 gradient;
  Node* node = nullptr;
};
using Stencil = std::array<StencilEntry, 64>;

// Analytic colliders standing for the reference's CollisionBody (phi, normal,
// velocity functions and a friction coefficient, include/snow/collision.hpp):
// make_plane (src/collision.cpp:5-27) stores the unit normal, phi(x) = n.(x - p)
// and zero velocity; the same plane may move with a constant velocity; a solid
// sphere has phi(x) = |x - c| - r and normal (x - c)/|x - c|.
struct Plane {
  int kind = 0;        // 0 plane, 1 sphere, 2 oriented box
  Vec3 point, normal;  // plane: point, unit normal; sphere and box: centre in `point`
  double friction = 0.0;
  Vec3 velocity{0.0, 0.0, 0.0};
  double radius = 0.0;
  Vec3 axis{0.0, 0.0, 0.0}, half{0.0, 0.0, 0.0};  // box: axes normal, axis, normal x axis; half extents
};
inline Vec3 unit(const Vec3& n) {
  const double len = norm(n);
  return len > 0.0 ? n / len : n;  // Eigen normalized() leaves a zero vector as is
}
inline Plane make_plane(const Vec3& p, const Vec3& n, double mu) {
  Plane b;
  b.point = p;
  b.normal = unit(n);
  b.friction = mu;
  return b;
}
// A solid oriented box as a user of the reference would write its CollisionBody:
// l = the point in the box's axes (u, w, u x w), q_k = |l_k| - h_k; phi is the
// signed distance |max(q, 0)| + min(max q, 0); the normal is, inside, the
// outward normal of the face with the largest q_k (first on a tie, + side at
// l_k = 0) and, outside, the normalised gradient of phi.
inline Vec3 cross(const Vec3& a, const Vec3& b) {
  return Vec3{a[1] * b[2] - a[2] * b[1], a[2] * b[0] - a[0] * b[2], a[0] * b[1] - a[1] * b[0]};
}
inline void box_frame(const Plane& b, const Vec3& x, Vec3 ax[3], double l[3], double q[3]) {
  ax[0] = b.normal;
  ax[1] = b.axis;
  ax[2] = cross(b.normal, b.axis);
  const Vec3 d = x - b.point;
  for (int k = 0; k < 3; ++k) {
    l[k] = dot(ax[k], d);
    q[k] = std::abs(l[k]) - b.half[k];
  }
}
inline double box_phi(const Plane& b, const Vec3& x) {
  Vec3 ax[3];
  double l[3], q[3];
  box_frame(b, x, ax, l, q);
  double out2 = 0.0;
  for (double v : q) out2 += v > 0.0 ? v * v : 0.0;
  return std::sqrt(out2) + std::min(std::max(q[0], std::max(q[1], q[2])), 0.0);
}
inline Vec3 box_normal(const Plane& b, const Vec3& x) {
  Vec3 ax[3];
  double l[3], q[3];
  box_frame(b, x, ax, l, q);
  int k = 0;
  for (int a = 1; a < 3; ++a)
    if (q[a] > q[k]) k = a;
  if (q[k] <= 0.0) return (l[k] < 0.0 ? -1.0 : 1.0) * ax[k];
  Vec3 g{0.0, 0.0, 0.0};
  for (int a = 0; a < 3; ++a)
    if (q[a] > 0.0) g = g + (l[a] < 0.0 ? -q[a] : q[a]) * ax[a];
  return unit(g);
}
inline double body_phi(const Plane& b, const Vec3& x) {
  if (b.kind == 2) return box_phi(b, x);
  return b.kind == 1 ? norm(x - b.point) - b.radius : dot(b.normal, x - b.point);
}
inline Vec3 body_normal(const Plane& b, const Vec3& x) {
  if (b.kind == 2) return box_normal(b, x);
  return b.kind == 1 ? unit(x - b.point) : b.normal;
}

// ------------------------------------------------------------------ kernels
// N(a, b): cubic B-spline of |a - b| (grid.cpp:24-40).
double N(double a, double b) {
  const double d = std::abs(a - b);
  if (d >= 0.0 && d < 1.0) return 0.5 * d * d * d - d * d + 2.0 / 3.0;
  if (d >= 1.0 && d < 2.0) return -1.0 / 6.0 * d * d * d + d * d - 2.0 * d + 4.0 / 3.0;
  return 0.0;
}
inline double signum(double x) { return x > 0.0 ? 1.0 : (x < 0.0 ? -1.0 : 0.0); }
// N_dash(node, x): derivative of N w.r.t. x (grid.cpp:42-58).
double N_dash(double node, double x) {
  const double d = std::abs(node - x);
  if (d >= 0.0 && d < 1.0) return (1.5 * d * d - 2 * d) * signum(x - node);
  if (d >= 1.0 && d < 2.0) return (-1.0 / 2.0 * d * d + 2 * d - 2.0) * signum(x - node);
  return 0.0;
}

inline void base_of(const Vec3& gp, int base[3]) {
  for (int a = 0; a < 3; ++a) base[a] = (int)std::floor(gp[a]) - 1;
}

// build_stencil (grid.cpp:60-117): 64 nodes from base = floor(x/dx) - 1, i-major.
Stencil build_stencil(const Particle& p, double dx) {
  Stencil st;
  const Vec3 gp = p.x / dx;
  int base[3];
  base_of(gp, base);
  double w[3][4], dw[3][4];
  for (int a = 0; a < 3; ++a)
    for (int i = 0; i < 4; ++i) {
      w[a][i] = N(base[a] + i, gp[a]);
      dw[a][i] = N_dash(base[a] + i, gp[a]) / dx;
    }
  int n = 0;
  for (int i = 0; i < 4; ++i)
    for (int j = 0; j < 4; ++j)
      for (int k = 0; k < 4; ++k) {
        StencilEntry& e = st[n++];
        e.index = {base[0] + i, base[1] + j, base[2] + k};
        e.weight = w[0][i] * w[1][j] * w[2][k];
        e.gradient = {dw[0][i] * w[1][j] * w[2][k], w[0][i] * dw[1][j] * w[2][k],
                      w[0][i] * w[1][j] * dw[2][k]};
      }
  return st;
}

// P2G (grid.cpp:119-136): inserts all 64 nodes, caches node pointers.
void p2g(Grid& grid, const Particle& p, Stencil& st) {
  const Vec3 mom = p.m * p.v;
  for (StencilEntry& e : st) {
    Node& node = grid[e.index];
    e.node = &node;
    node.mass += e.weight * p.m;
    node.momentum += e.weight * mom;
  }
}
void p2g(Grid& grid, const Particle& p, double dx) {
  Stencil st = build_stencil(p, dx);
  p2g(grid, p, st);
}

// calculate_volume (grid.cpp:138-160): V_p0 = m_p / sum_i(m_i w_ip / dx^3).
void calculate_volume(Grid& grid, Particle& p, double dx) {
  const Vec3 gp = p.x / dx;
  int base[3];
  base_of(gp, base);
  double density = 0.0;
  for (int i = 0; i < 4; ++i)
    for (int j = 0; j < 4; ++j)
      for (int k = 0; k < 4; ++k) {
        const NodeIdx idx{i + base[0], j + base[1], k + base[2]};
        const Node& node = grid[idx];
        const double wp = N(idx.i, gp[0]) * N(idx.j, gp[1]) * N(idx.k, gp[2]);
        density += (node.mass * wp) / std::pow(dx, 3.0);
      }
  p.V0 = p.m / density;
}

// force_constitutive (grid.cpp:162-172): fixed-corotated stress with
// exponential hardening, P = 2 mu (F_E - R_E) + lambda (J_E - 1) J_E F_E^-T.
Mat3 force_constitutive(const Particle& p, double mu0, double lambda0, double xi) {
  const double h = std::exp(xi * (1.0 - det(p.FP)));
  const double mu = mu0 * h, lambda = lambda0 * h;
  const double J = det(p.FE);
  Mat3 U, V;
  Vec3 s;
  svd3(p.FE, U, s, V);
  const Mat3 R = U * transpose(V);
  return (2 * mu) * (p.FE - R) + (lambda * (J - 1) * J) * transpose(inverse(p.FE));
}

// force_grid_accumulation (grid.cpp:174-182): node f += (-V_p0 P F_E^T) grad w.
void force_grid_accumulation(const Mat3& P, const Particle& p, const Stencil& st) {
  const Mat3 M = (-p.V0) * (P * transpose(p.FE));
  for (const StencilEntry& e : st) e.node->force += M * e.gradient;
}
// force_calculation (grid.cpp:184-193): test helper, stencil + lookup + scatter.
void force_calculation(Grid& grid, const Particle& p, double dx, double mu0, double lambda0,
                       double xi) {
  const Mat3 P = force_constitutive(p, mu0, lambda0, xi);
  Stencil st = build_stencil(p, dx);
  for (StencilEntry& e : st) e.node = &grid[e.index];
  force_grid_accumulation(P, p, st);
}

// grid_velocity (grid.cpp:195-204): massless nodes keep their velocity.
void grid_velocity(Grid& grid, const Vec3& g, double dt) {
  for (auto& [idx, node] : grid)
    if (node.mass > 0)
      node.velocity = (node.momentum / node.mass) + dt * ((node.force / node.mass) + g);
}

// collision_helper (grid.cpp:206-231): Coulomb friction against a collider.
Vec3 collide(const Vec3& x, const Vec3& v, const Plane& b) {
  const double phi = body_phi(b, x);
  if (phi <= 0) {
    const Vec3 n = body_normal(b, x);
    const Vec3 vc = b.velocity;
    const Vec3 vrel = v - vc;
    const double vn = dot(vrel, n);
    if (vn < 0) {
      const Vec3 vt = vrel - vn * n;
      Vec3 out;
      if (norm(vt) <= -1 * b.friction * vn)
        out = {0.0, 0.0, 0.0};
      else
        out = vt + (b.friction * vn) * (vt / norm(vt));
      return out + vc;
    }
  }
  return v;
}

// grid_collisions (grid.cpp:233-243): at the node position dx * index.
void grid_collisions(Grid& grid, const std::vector<Plane>& bodies, double dx) {
  for (auto& [idx, node] : grid) {
    const Vec3 xn{dx * idx.i, dx * idx.j, dx * idx.k};
    for (const Plane& b : bodies) node.velocity = collide(xn, node.velocity, b);
  }
}

// stress_update (grid.cpp:245-286): grad v, trial F_E, SVD clamp, F_P.
void stress_update(const Grid& grid, Particle& p, double dx, double dt, double theta_c,
                   double theta_s) {
  const Vec3 gp = p.x / dx;
  int base[3];
  base_of(gp, base);
  Mat3 gradv;
  for (int i = 0; i < 4; ++i)
    for (int j = 0; j < 4; ++j)
      for (int k = 0; k < 4; ++k) {
        const NodeIdx idx{i + base[0], j + base[1], k + base[2]};
        auto it = grid.find(idx);
        if (it == grid.end()) continue;
        const Node& node = it->second;
        const double Nx = N(idx.i, gp[0]), Ny = N(idx.j, gp[1]), Nz = N(idx.k, gp[2]);
        const double dNx = N_dash(idx.i, gp[0]), dNy = N_dash(idx.j, gp[1]),
                     dNz = N_dash(idx.k, gp[2]);
        const Vec3 gw{dNx * Ny * Nz * (1 / dx), Nx * dNy * Nz * (1 / dx), Nx * Ny * dNz * (1 / dx)};
        gradv = gradv + outer(node.velocity, gw);
      }
  const Mat3 FEt = (Mat3::identity() + dt * gradv) * p.FE;
  const Mat3 Ft = FEt * p.FP;
  Mat3 U, V;
  Vec3 s;
  svd3(FEt, U, s, V);
  for (int a = 0; a < 3; ++a) s[a] = std::clamp(s[a], 1 - theta_c, 1 + theta_s);
  p.FE = U * diag(s) * transpose(V);
  p.FP = inverse(p.FE) * Ft;
}

// G2P (grid.cpp:288-325): PIC/FLIP blend; FLIP skips massless nodes.
void g2p(const Grid& grid, Particle& p, double dx, double alpha) {
  Vec3 vpic, vtemp;
  const Vec3 gp = p.x / dx;
  int base[3];
  base_of(gp, base);
  for (int i = 0; i < 4; ++i)
    for (int j = 0; j < 4; ++j)
      for (int k = 0; k < 4; ++k) {
        const NodeIdx idx{i + base[0], j + base[1], k + base[2]};
        auto it = grid.find(idx);
        if (it == grid.end()) continue;
        const Node& node = it->second;
        const double wp = N(idx.i, gp[0]) * N(idx.j, gp[1]) * N(idx.k, gp[2]);
        vpic += wp * node.velocity;
        if (node.mass > 0) vtemp += wp * (node.velocity - (node.momentum / node.mass));
      }
  const Vec3 vflip = p.v + vtemp;
  p.v = (1 - alpha) * vpic + alpha * vflip;
}

// particle_collisions (grid.cpp:327-333) and position_update (grid.cpp:335-338).
void particle_collisions(Particle& p, const std::vector<Plane>& bodies) {
  for (const Plane& b : bodies) p.v = collide(p.x, p.v, b);
}
void position_update(Particle& p, double dt) { p.x = p.x + dt * p.v; }

// ---------------------------------------------------------- implicit update
// The semi-implicit grid velocity update of Stomakhin et al., "A material
// point method for snow simulation", SIGGRAPH 2013, Section 4 (eq. 9) and its
// technical report's differentials.  The reference declares the functions
// (include/snow/grid.hpp:76,80,88-92: constitutive_differential, index_nodes,
// deformation_differential, force_differential, apply_A, Conjugate_residual)
// and defines none; these follow the paper:
//   (I + beta dt^2 M^-1 H) v = v*   on the nodes with mass, v* the explicit
// update after collisions, H u = -delta f(u) with
//   delta F_p = dt (sum_i u_i grad w_ip^T) F_Ep,
//   delta f_i = -sum_p V_p0 A_p(delta F_p) F_Ep^T grad w_ip,
// A_p the differential of the fixed-corotated P at F_Ep (F_P and so the
// hardening held fixed).  The operator is self-adjoint in the mass-weighted
// inner product <a, b>_M = sum_i m_i a_i . b_i, in which the conjugate
// residual method is run (it also handles the indefinite case).

inline Mat3 cofactor(const Mat3& F) {  // J F^-T
  Mat3 C;
  for (int r = 0; r < 3; ++r)
    for (int c = 0; c < 3; ++c) {
      const int r1 = (r + 1) % 3, r2 = (r + 2) % 3, c1 = (c + 1) % 3, c2 = (c + 2) % 3;
      C(r, c) = F(r1, c1) * F(r2, c2) - F(r1, c2) * F(r2, c1);
    }
  return C;
}
inline Mat3 cofactor_differential(const Mat3& F, const Mat3& dF) {
  Mat3 C;
  for (int r = 0; r < 3; ++r)
    for (int c = 0; c < 3; ++c) {
      const int r1 = (r + 1) % 3, r2 = (r + 2) % 3, c1 = (c + 1) % 3, c2 = (c + 2) % 3;
      C(r, c) = dF(r1, c1) * F(r2, c2) + F(r1, c1) * dF(r2, c2) - dF(r1, c2) * F(r2, c1) - F(r1, c2) * dF(r2, c1);
    }
  return C;
}

// constitutive_differential (declared at grid.hpp:76): dP for P = 2 mu (F - R)
// + lambda (J - 1) J F^-T at F = F_E:
//   dP = 2 mu (dF - dR) + lambda (J F^-T : dF) J F^-T + lambda (J - 1) d(J F^-T).
// dR from F = R S: W = R^T dR is skew and W S + S W = R^T dF - dF^T R, i.e.
// (tr(S) I - S) w = m for the axial vectors w of W and m of the right side.
Mat3 constitutive_differential(const Particle& p, const Mat3& dF, double mu0, double lambda0, double xi) {
  const double h = std::exp(xi * (1.0 - det(p.FP)));
  const double mu = mu0 * h, lambda = lambda0 * h;
  Mat3 U, V;
  Vec3 sv;
  svd3(p.FE, U, sv, V);
  const Mat3 R = U * transpose(V);
  const Mat3 S = V * diag(sv) * transpose(V);
  const Mat3 M = transpose(R) * dF - transpose(dF) * R;
  const Vec3 m{M(2, 1), M(0, 2), M(1, 0)};
  const double tr = S(0, 0) + S(1, 1) + S(2, 2);
  const Mat3 A = tr * Mat3::identity() - S;
  const Vec3 w = inverse(A) * m;
  Mat3 W;
  W(0, 1) = -w[2];
  W(0, 2) = w[1];
  W(1, 0) = w[2];
  W(1, 2) = -w[0];
  W(2, 0) = -w[1];
  W(2, 1) = w[0];
  const Mat3 dR = R * W;
  const Mat3 C = cofactor(p.FE);
  const double J = det(p.FE);
  double dJ = 0.0;
  for (int e = 0; e < 9; ++e) dJ += C.a[e] * dF.a[e];
  return (2 * mu) * (dF - dR) + (lambda * dJ) * C + (lambda * (J - 1)) * cofactor_differential(p.FE, dF);
}

// index_nodes (declared at grid.hpp:80): the nodes with mass, the unknowns.
std::vector<Node*> index_nodes(Grid& grid) {
  std::vector<Node*> out;
  for (auto& [idx, node] : grid)
    if (node.mass > 0) out.push_back(&node);
  return out;
}

// Stencil gradient of node idx at gp = x / dx (the same product as
// stress_update's basis_gradient, grid.cpp:262-270).
inline Vec3 basis_gradient(const NodeIdx& idx, const Vec3& gp, double dx) {
  const double Nx = N(idx.i, gp[0]), Ny = N(idx.j, gp[1]), Nz = N(idx.k, gp[2]);
  const double dNx = N_dash(idx.i, gp[0]), dNy = N_dash(idx.j, gp[1]), dNz = N_dash(idx.k, gp[2]);
  return Vec3{dNx * Ny * Nz * (1 / dx), Nx * dNy * Nz * (1 / dx), Nx * Ny * dNz * (1 / dx)};
}

// deformation_differential (declared at grid.hpp:88): dt (sum_i dv_i grad w_ip^T) F_Ep.
Mat3 deformation_differential(const Grid& grid, const Particle& p, double dx, double dt) {
  const Vec3 gp = p.x / dx;
  int base[3];
  base_of(gp, base);
  Mat3 g;
  for (int i = 0; i < 4; ++i)
    for (int j = 0; j < 4; ++j)
      for (int k = 0; k < 4; ++k) {
        const NodeIdx idx{i + base[0], j + base[1], k + base[2]};
        auto it = grid.find(idx);
        if (it == grid.end()) continue;
        g = g + outer(it->second.delta_v, basis_gradient(idx, gp, dx));
      }
  return dt * (g * p.FE);
}

// force_differential (declared at grid.hpp:89): node delta_force += -V_p0 dP F_E^T grad w.
void force_differential(Grid& grid, const Particle& p, double dx, double dt, double mu0, double lambda0,
                        double xi) {
  const Mat3 dP = constitutive_differential(p, deformation_differential(grid, p, dx, dt), mu0, lambda0, xi);
  const Mat3 G = (-p.V0) * (dP * transpose(p.FE));
  const Vec3 gp = p.x / dx;
  int base[3];
  base_of(gp, base);
  for (int i = 0; i < 4; ++i)
    for (int j = 0; j < 4; ++j)
      for (int k = 0; k < 4; ++k) {
        const NodeIdx idx{i + base[0], j + base[1], k + base[2]};
        auto it = grid.find(idx);
        if (it == grid.end()) continue;
        it->second.delta_force += G * basis_gradient(idx, gp, dx);
      }
}

// apply_A (declared at grid.hpp:90): (A q)_i = q_i - beta dt delta f_i(q) / m_i
// over the Krylov nodes.
std::vector<Vec3> apply_A(Grid& grid, const std::vector<Particle>& snow, const std::vector<Node*>& nodes,
                          const std::vector<Vec3>& q, double dx, double dt, double mu0, double lambda0, double xi,
                          double beta) {
  for (auto& [idx, node] : grid) node.delta_v = node.delta_force = Vec3{};
  for (std::size_t i = 0; i < nodes.size(); ++i) nodes[i]->delta_v = q[i];
  for (const Particle& p : snow) force_differential(grid, p, dx, dt, mu0, lambda0, xi);
  std::vector<Vec3> out(nodes.size());
  for (std::size_t i = 0; i < nodes.size(); ++i)
    out[i] = q[i] - (beta * dt / nodes[i]->mass) * nodes[i]->delta_force;
  return out;
}

inline double mdot(const std::vector<Node*>& nodes, const std::vector<Vec3>& a, const std::vector<Vec3>& b) {
  double s = 0.0;
  for (std::size_t i = 0; i < nodes.size(); ++i) s += nodes[i]->mass * dot(a[i], b[i]);
  return s;
}

// Conjugate_residual (declared at grid.hpp:91): solves A v = v* from v = v*
// until <r, r>_M <= squared_tolerance <v*, v*>_M or maximum_iterations;
// writes the node velocities.  Returns the iterations taken.
int Conjugate_residual(Grid& grid, const std::vector<Particle>& snow, const std::vector<Node*>& nodes, double dx,
                       double dt, double mu0, double lambda0, double xi, double beta, double squared_tolerance,
                       int maximum_iterations, double* residual = nullptr) {
  const std::size_t n = nodes.size();
  std::vector<Vec3> b(n), x(n), r(n), p(n), Ar, Ap;
  for (std::size_t i = 0; i < n; ++i) b[i] = x[i] = nodes[i]->velocity;
  const double bb = mdot(nodes, b, b);
  const std::vector<Vec3> Ax = apply_A(grid, snow, nodes, x, dx, dt, mu0, lambda0, xi, beta);
  for (std::size_t i = 0; i < n; ++i) p[i] = r[i] = b[i] - Ax[i];
  Ar = apply_A(grid, snow, nodes, r, dx, dt, mu0, lambda0, xi, beta);
  Ap = Ar;
  double gamma = mdot(nodes, r, Ar);
  double rr = mdot(nodes, r, r);
  int it = 0;
  while (it < maximum_iterations && rr > squared_tolerance * bb) {
    const double alpha = gamma / mdot(nodes, Ap, Ap);
    for (std::size_t i = 0; i < n; ++i) {
      x[i] += alpha * p[i];
      r[i] = r[i] - alpha * Ap[i];
    }
    ++it;
    rr = mdot(nodes, r, r);
    if (rr <= squared_tolerance * bb) break;
    Ar = apply_A(grid, snow, nodes, r, dx, dt, mu0, lambda0, xi, beta);
    const double gamma_next = mdot(nodes, r, Ar);
    const double beta_k = gamma_next / gamma;
    gamma = gamma_next;
    for (std::size_t i = 0; i < n; ++i) {
      p[i] = r[i] + beta_k * p[i];
      Ap[i] = Ar[i] + beta_k * Ap[i];
    }
  }
  for (std::size_t i = 0; i < n; ++i) nodes[i]->velocity = x[i];
  if (residual) *residual = bb > 0 ? std::sqrt(rr / bb) : 0.0;
  return it;
}

// setup (grid.cpp:340-357).
void setup(std::vector<Particle>& snow, double dx) {
  Grid grid;
  std::vector<Stencil> st(snow.size());
  for (std::size_t i = 0; i < snow.size(); ++i) st[i] = build_stencil(snow[i], dx);
  for (std::size_t j = 0; j < snow.size(); ++j) p2g(grid, snow[j], st[j]);
  for (Particle& p : snow) calculate_volume(grid, p, dx);
}

struct StepParams {
  double gravity[3];
  double dt, dx, mu0, lambda0, xi, theta_c, theta_s, alpha;
};

// step (grid.cpp:359-450): same stage order and OpenMP placement.  `ms` gets
// the ten stage times in StepTimings order (include/snow/debug.hpp:3-15).
// Optional semi-implicit update (beta = 0: the reference's explicit step).
struct ImplicitParams {
  double beta = 0.0, squared_tolerance = 1e-12;
  int max_iterations = 50;
  int iterations = 0;     // out: Conjugate_residual iterations of the last step
  double residual = 0.0;  // out: its relative residual
};

void step(std::vector<Particle>& snow, const std::vector<Plane>& bodies,
          std::vector<Stencil>& stencils, const StepParams& prm, double ms[10],
          ImplicitParams* imp = nullptr) {
  using clk = std::chrono::steady_clock;
  auto since = [](clk::time_point t0) {
    return std::chrono::duration<double, std::milli>(clk::now() - t0).count();
  };
  Grid grid;
  const std::size_t n = snow.size();
  auto t0 = clk::now();
#pragma omp parallel for schedule(static)
  for (std::size_t i = 0; i < n; ++i) stencils[i] = build_stencil(snow[i], prm.dx);
  ms[0] += since(t0);
  t0 = clk::now();
  for (std::size_t i = 0; i < n; ++i) p2g(grid, snow[i], stencils[i]);
  ms[1] += since(t0);
  std::vector<Mat3> stress(n);
  t0 = clk::now();
  for (std::size_t i = 0; i < n; ++i) stress[i] = force_constitutive(snow[i], prm.mu0, prm.lambda0, prm.xi);
  ms[2] += since(t0);
  t0 = clk::now();
  for (std::size_t i = 0; i < n; ++i) force_grid_accumulation(stress[i], snow[i], stencils[i]);
  ms[3] += since(t0);
  t0 = clk::now();
  grid_velocity(grid, Vec3{prm.gravity[0], prm.gravity[1], prm.gravity[2]}, prm.dt);
  ms[4] += since(t0);
  t0 = clk::now();
  grid_collisions(grid, bodies, prm.dx);
  if (imp && imp->beta > 0) {
    const std::vector<Node*> nodes = index_nodes(grid);
    imp->iterations = Conjugate_residual(grid, snow, nodes, prm.dx, prm.dt, prm.mu0, prm.lambda0, prm.xi, imp->beta,
                                         imp->squared_tolerance, imp->max_iterations, &imp->residual);
  }
  ms[5] += since(t0);
  t0 = clk::now();
#pragma omp parallel for
  for (std::size_t i = 0; i < n; ++i)
    stress_update(grid, snow[i], prm.dx, prm.dt, prm.theta_c, prm.theta_s);
  ms[6] += since(t0);
  t0 = clk::now();
#pragma omp parallel for
  for (std::size_t i = 0; i < n; ++i) g2p(grid, snow[i], prm.dx, prm.alpha);
  ms[7] += since(t0);
  t0 = clk::now();
  for (Particle& p : snow) particle_collisions(p, bodies);
  ms[8] += since(t0);
  t0 = clk::now();
  for (Particle& p : snow) position_update(p, prm.dt);
  ms[9] += since(t0);
}

}  // namespace oracle

// ------------------------------------------------------------------ C API
// Flat C entry points for the Python tests (ctypes).  Particles are arrays of
// 26-double records (oracle::Particle); grids travel as node lists: int32
// ijk[n][3] and double fields[n][10] = mass, momentum[3], velocity[3], force[3].
using namespace oracle;

namespace {
std::vector<Particle> to_vec(const double* rec, int64_t n) {
  std::vector<Particle> v((std::size_t)n);
  if (n) std::memcpy(static_cast<void*>(v.data()), rec, (std::size_t)n * sizeof(Particle));
  return v;
}
void from_vec(const std::vector<Particle>& v, double* rec) {
  if (!v.empty()) std::memcpy(rec, static_cast<const void*>(v.data()), v.size() * sizeof(Particle));
}
std::vector<Plane> to_planes(const double* planes, int n) {
  // planes: n x 7 doubles = point[3], normal[3] (not necessarily unit), friction
  std::vector<Plane> b;
  for (int i = 0; i < n; ++i) {
    const double* q = planes + 7 * i;
    b.push_back(make_plane(Vec3{q[0], q[1], q[2]}, Vec3{q[3], q[4], q[5]}, q[6]));
  }
  return b;
}
// bodies: n x 18 doubles = kind, point[3], normal[3], velocity[3], friction,
// radius, axis[3], half extents[3]
std::vector<Plane> to_bodies(const double* rows, int n) {
  std::vector<Plane> b;
  for (int i = 0; i < n; ++i) {
    const double* q = rows + 18 * i;
    Plane c = make_plane(Vec3{q[1], q[2], q[3]}, Vec3{q[4], q[5], q[6]}, q[10]);
    c.kind = (int)q[0];
    c.velocity = Vec3{q[7], q[8], q[9]};
    c.radius = q[11];
    c.axis = Vec3{q[12], q[13], q[14]};
    c.half = Vec3{q[15], q[16], q[17]};
    b.push_back(c);
  }
  return b;
}
struct GridBox {
  Grid g;
};
}  // namespace

extern "C" {

int oracle_record_bytes(void) { return (int)sizeof(Particle); }

void oracle_setup(double* rec, int64_t n, double dx) {
  auto v = to_vec(rec, n);
  setup(v, dx);
  from_vec(v, rec);
}

// params: gravity[3], dt, dx, mu0, lambda0, xi, theta_c, theta_s, alpha (11 doubles)
static void run_steps(double* rec, int64_t n, const double* params, const std::vector<Plane>& b, int steps,
                      double* stage_ms) {
  auto v = to_vec(rec, n);
  StepParams p;
  std::memcpy(&p, params, sizeof(StepParams));
  std::vector<Stencil> st(v.size());
  double ms[10] = {0};
  const auto t0 = std::chrono::steady_clock::now();
  for (int s = 0; s < steps; ++s) step(v, b, st, p, ms);
  const double wall = std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
  if (stage_ms) {  // ten stage times, then the wall time of the step loop
    for (int i = 0; i < 10; ++i) stage_ms[i] = ms[i];
    stage_ms[10] = wall;
  }
  from_vec(v, rec);
}

void oracle_step(double* rec, int64_t n, const double* params, const double* planes, int n_planes,
                 int steps, double* stage_ms) {
  run_steps(rec, n, params, to_planes(planes, n_planes), steps, stage_ms);
}
// The same with general bodies (rows as in to_bodies).
void oracle_step_bodies(double* rec, int64_t n, const double* params, const double* bodies, int n_bodies,
                        int steps, double* stage_ms) {
  run_steps(rec, n, params, to_bodies(bodies, n_bodies), steps, stage_ms);
}

// Steps with the semi-implicit update (beta > 0); iterations[k] and
// residual[k] report step k's solve.
void oracle_step_implicit(double* rec, int64_t n, const double* params, const double* planes, int n_planes,
                          int steps, double beta, double squared_tolerance, int max_iterations, int* iterations,
                          double* residual) {
  auto v = to_vec(rec, n);
  StepParams p;
  std::memcpy(&p, params, sizeof(StepParams));
  const auto bodies = to_planes(planes, n_planes);
  std::vector<Stencil> st(v.size());
  double ms[10] = {0};
  for (int k = 0; k < steps; ++k) {
    ImplicitParams imp;
    imp.beta = beta;
    imp.squared_tolerance = squared_tolerance;
    imp.max_iterations = max_iterations;
    step(v, bodies, st, p, ms, &imp);
    if (iterations) iterations[k] = imp.iterations;
    if (residual) residual[k] = imp.residual;
  }
  from_vec(v, rec);
}

// constitutive_differential of one particle record; dF and dP column-major.
void oracle_constitutive_differential(const double* rec, const double* dF, double mu0, double lambda0, double xi,
                                      double* dP) {
  const Particle p = to_vec(rec, 1)[0];
  Mat3 d;
  std::memcpy(d.a, dF, sizeof d.a);
  const Mat3 out = constitutive_differential(p, d, mu0, lambda0, xi);
  std::memcpy(dP, out.a, sizeof out.a);
}
void oracle_force_constitutive(const double* rec, double mu0, double lambda0, double xi, double* P) {
  const Particle p = to_vec(rec, 1)[0];
  const Mat3 out = force_constitutive(p, mu0, lambda0, xi);
  std::memcpy(P, out.a, sizeof out.a);
}

// The grid that P2G + forces + grid_velocity + collisions of one step build
// from the records (the state the implicit solve starts from), over its
// nodes with mass in index_nodes' order: ijk[m][3] and fields[m][10] (mass,
// momentum, velocity, force) when given; with q (m x 3): out = A q; without q
// (out given): out = the Conjugate_residual solution.  Returns m (the node
// count; nothing is written when out is NULL or m > cap).
int64_t oracle_implicit_grid(const double* rec, int64_t n, const double* params, const double* planes,
                             int n_planes, double beta, double squared_tolerance, int max_iterations,
                             const double* q, double* out, int32_t* ijk, double* fields, int64_t cap,
                             int* iterations) {
  auto snow = to_vec(rec, n);
  StepParams prm;
  std::memcpy(&prm, params, sizeof(StepParams));
  const auto bodies = to_planes(planes, n_planes);
  Grid grid;
  std::vector<Stencil> st(snow.size());
  for (std::size_t i = 0; i < snow.size(); ++i) st[i] = build_stencil(snow[i], prm.dx);
  for (std::size_t i = 0; i < snow.size(); ++i) p2g(grid, snow[i], st[i]);
  for (std::size_t i = 0; i < snow.size(); ++i)
    force_grid_accumulation(force_constitutive(snow[i], prm.mu0, prm.lambda0, prm.xi), snow[i], st[i]);
  grid_velocity(grid, Vec3{prm.gravity[0], prm.gravity[1], prm.gravity[2]}, prm.dt);
  grid_collisions(grid, bodies, prm.dx);
  std::vector<Node*> nodes;
  std::vector<NodeIdx> idx;
  for (auto& [k, node] : grid)
    if (node.mass > 0) {
      nodes.push_back(&node);
      idx.push_back(k);
    }
  const int64_t m = (int64_t)nodes.size();
  if (!out || m > cap) return m;
  for (int64_t i = 0; i < m; ++i) {
    if (ijk) {
      ijk[3 * i] = idx[i].i;
      ijk[3 * i + 1] = idx[i].j;
      ijk[3 * i + 2] = idx[i].k;
    }
    if (fields) {
      double* f = fields + 10 * i;
      f[0] = nodes[i]->mass;
      for (int c = 0; c < 3; ++c) {
        f[1 + c] = nodes[i]->momentum[c];
        f[4 + c] = nodes[i]->velocity[c];
        f[7 + c] = nodes[i]->force[c];
      }
    }
  }
  if (q) {
    std::vector<Vec3> qq(m);
    for (int64_t i = 0; i < m; ++i) qq[i] = Vec3{q[3 * i], q[3 * i + 1], q[3 * i + 2]};
    const auto a = apply_A(grid, snow, nodes, qq, prm.dx, prm.dt, prm.mu0, prm.lambda0, prm.xi, beta);
    for (int64_t i = 0; i < m; ++i)
      for (int c = 0; c < 3; ++c) out[3 * i + c] = a[i][c];
    return m;
  }
  const int it = Conjugate_residual(grid, snow, nodes, prm.dx, prm.dt, prm.mu0, prm.lambda0, prm.xi, beta,
                                    squared_tolerance, max_iterations);
  if (iterations) *iterations = it;
  for (int64_t i = 0; i < m; ++i)
    for (int c = 0; c < 3; ++c) out[3 * i + c] = nodes[i]->velocity[c];
  return m;
}

double oracle_N(double a, double b) { return N(a, b); }
double oracle_N_dash(double a, double b) { return N_dash(a, b); }

void oracle_svd3(const double* F, double* U, double* s, double* V) {
  Mat3 f, u, vv;
  Vec3 sv;
  std::memcpy(f.a, F, sizeof f.a);
  svd3(f, u, sv, vv);
  std::memcpy(U, u.a, sizeof u.a);
  std::memcpy(V, vv.a, sizeof vv.a);
  for (int i = 0; i < 3; ++i) s[i] = sv[i];
}

void* oracle_grid_new(void) { return new GridBox; }
void oracle_grid_free(void* g) { delete static_cast<GridBox*>(g); }
int64_t oracle_grid_size(void* g) { return (int64_t) static_cast<GridBox*>(g)->g.size(); }
void oracle_grid_export(void* g, int32_t* ijk, double* fields) {
  int64_t r = 0;
  for (const auto& [idx, node] : static_cast<GridBox*>(g)->g) {
    ijk[3 * r] = idx.i;
    ijk[3 * r + 1] = idx.j;
    ijk[3 * r + 2] = idx.k;
    double* f = fields + 10 * r;
    f[0] = node.mass;
    for (int a = 0; a < 3; ++a) {
      f[1 + a] = node.momentum[a];
      f[4 + a] = node.velocity[a];
      f[7 + a] = node.force[a];
    }
    ++r;
  }
}
void oracle_grid_set(void* g, const int32_t* ijk, const double* fields, int64_t n) {
  auto& grid = static_cast<GridBox*>(g)->g;
  for (int64_t r = 0; r < n; ++r) {
    Node& node = grid[NodeIdx{ijk[3 * r], ijk[3 * r + 1], ijk[3 * r + 2]}];
    const double* f = fields + 10 * r;
    node.mass = f[0];
    for (int a = 0; a < 3; ++a) {
      node.momentum[a] = f[1 + a];
      node.velocity[a] = f[4 + a];
      node.force[a] = f[7 + a];
    }
  }
}
void oracle_p2g(void* g, const double* rec, int64_t n, double dx) {
  auto v = to_vec(rec, n);
  for (auto& p : v) p2g(static_cast<GridBox*>(g)->g, p, dx);
}
void oracle_calculate_volume(void* g, double* rec, int64_t n, double dx) {
  auto v = to_vec(rec, n);
  for (auto& p : v) calculate_volume(static_cast<GridBox*>(g)->g, p, dx);
  from_vec(v, rec);
}
void oracle_force_calculation(void* g, const double* rec, int64_t n, double dx, double mu0,
                              double lambda0, double xi) {
  auto v = to_vec(rec, n);
  for (auto& p : v) force_calculation(static_cast<GridBox*>(g)->g, p, dx, mu0, lambda0, xi);
}
void oracle_grid_velocity(void* g, const double* gravity, double dt) {
  grid_velocity(static_cast<GridBox*>(g)->g, Vec3{gravity[0], gravity[1], gravity[2]}, dt);
}
void oracle_grid_collisions(void* g, const double* planes, int n_planes, double dx) {
  grid_collisions(static_cast<GridBox*>(g)->g, to_planes(planes, n_planes), dx);
}
void oracle_stress_update(void* g, double* rec, int64_t n, double dx, double dt, double theta_c,
                          double theta_s) {
  auto v = to_vec(rec, n);
  for (auto& p : v) stress_update(static_cast<GridBox*>(g)->g, p, dx, dt, theta_c, theta_s);
  from_vec(v, rec);
}
void oracle_g2p(void* g, double* rec, int64_t n, double dx, double alpha) {
  auto v = to_vec(rec, n);
  for (auto& p : v) g2p(static_cast<GridBox*>(g)->g, p, dx, alpha);
  from_vec(v, rec);
}
void oracle_particle_collisions(double* rec, int64_t n, const double* planes, int n_planes) {
  auto v = to_vec(rec, n);
  auto b = to_planes(planes, n_planes);
  for (auto& p : v) particle_collisions(p, b);
  from_vec(v, rec);
}
void oracle_position_update(double* rec, int64_t n, double dt) {
  auto v = to_vec(rec, n);
  for (auto& p : v) position_update(p, dt);
  from_vec(v, rec);
}

}  // extern "C"
