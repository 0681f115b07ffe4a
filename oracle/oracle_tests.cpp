// ORACLE self-test -- test infrastructure only.
// Pins the CPU restatement (snow_oracle.cpp) against the known answers of the
// reference's unit tests, tests/snow_tests.cpp:30-407 (24 cases, tolerance 1e-10
// absolute and exact zero where the reference asks for it).  Each case below
// names the reference test it restates.  Exit status 0 = all pass.
#include <cstdio>
#include <functional>
#include <string>

#include "snow_oracle.cpp"

using namespace oracle;

namespace {
int failures = 0;
void check(bool ok, const char* what) {
  if (!ok) {
    std::printf("FAIL: %s\n", what);
    ++failures;
  }
}
bool near(double a, double b, double tol = 1e-10) { return std::abs(a - b) < tol; }
double dist(const Vec3& a, const Vec3& b) { return norm(a - b); }
Particle particle(Vec3 x, Vec3 v, double m, double V0) {
  Particle p;
  p.x = x;
  p.v = v;
  p.m = m;
  p.V0 = V0;
  p.FP = Mat3::identity();
  p.FE = Mat3::identity();
  return p;
}
// Nodes (0..3)^3 with a given velocity field, as in tests/snow_tests.cpp:228-240.
Grid lattice_grid(const std::function<Vec3(int, int, int)>& vel) {
  Grid g;
  for (int i = 0; i < 4; ++i)
    for (int j = 0; j < 4; ++j)
      for (int k = 0; k < 4; ++k) g[NodeIdx{i, j, k}].velocity = vel(i, j, k);
  return g;
}
std::vector<Plane> ground(double mu) { return {make_plane({0, 0, 0}, {0, 1, 0}, mu)}; }
Mat3 diag3(double a, double b, double c) { return diag(Vec3{a, b, c}); }

struct Case {
  const char* name;
  std::function<void()> body;
};
}  // namespace

int main() {
  const Case cases[] = {
      {"spline (snow_tests.cpp:30)",
       [] {
         check(near(N(1, 1), 2.0 / 3.0), "N(1,1)=2/3");
         check(near(N(1, 2), 1.0 / 6.0), "N(1,2)=1/6");
         check(N(1, 3) == 0, "N(1,3)==0");
         check(N(1, 10) == 0, "N(1,10)==0");
         check(near(N(1.5, 0.75), N(0.75, 1.5)), "N symmetric");
       }},
      {"N_dash (snow_tests.cpp:46)",
       [] {
         check(near(N_dash(4, 4.3), -N_dash(4.3, 4)), "N' antisymmetric");
         check(near(N_dash(1, 1), 0), "N'(1,1)=0");
         check(near(N_dash(0, 1), -0.5), "N'(0,1)=-0.5");
         check(near(N_dash(0, 2), 0), "N'(0,2)=0");
         check(near(N_dash(0, 0.5), -0.625), "N'(0,0.5)=-0.625");
       }},
      {"P2G conservation (snow_tests.cpp:62)",
       [] {
         Grid g;
         p2g(g, particle({2.1, 3.5, 4.7}, {3, -2, 0.5}, 2, 1), 0.5);
         double m = 0;
         Vec3 p;
         for (auto& [i, n] : g) m += n.mass, p += n.momentum;
         check(near(m, 2), "mass 2");
         check(dist(p, {6, -4, 1}) < 1e-10, "momentum (6,-4,1)");
       }},
      {"P2G overlap (snow_tests.cpp:79)",
       [] {
         Grid g;
         p2g(g, particle({2.1, 3.5, 4.7}, {3, -2, 0.5}, 2, 1), 0.5);
         p2g(g, particle({2.3, 3.7, 4.4}, {-1, 4, 2}, 1.5, 1), 0.5);
         double m = 0;
         Vec3 p;
         for (auto& [i, n] : g) m += n.mass, p += n.momentum;
         check(near(m, 3.5), "mass 3.5");
         check(dist(p, {4.5, 2, 4}) < 1e-10, "momentum (4.5,2,4)");
       }},
      {"P2G translation (snow_tests.cpp:98)",
       [] {
         Grid a, b;
         p2g(a, particle({2.15, 3.35, 4.65}, {1, 2, 3}, 1, 1), 0.5);
         p2g(b, particle({2.65, 3.35, 4.65}, {1, 2, 3}, 1, 1), 0.5);
         check(a.size() == b.size(), "same node count");
         for (auto& [i, n] : a) {
           auto it = b.find(NodeIdx{i.i + 1, i.j, i.k});
           check(it != b.end(), "translated node exists");
           if (it == b.end()) continue;
           check(near(n.mass, it->second.mass), "translated mass");
           check(dist(n.momentum, it->second.momentum) < 1e-10, "translated momentum");
         }
       }},
      {"volume (snow_tests.cpp:124)",
       [] {
         Grid g;
         Particle p = particle({1, 2, 3}, {1, 2, 3}, 1, 7);
         p2g(g, p, 0.5);
         calculate_volume(g, p, 0.5);
         check(near(p.V0, 1), "V_p0 = 1");
       }},
      {"zero force (snow_tests.cpp:133)",
       [] {
         Grid g;
         Particle p = particle({1, 2, 3}, {1, 2, 3}, 1, 7);
         p2g(g, p, 0.5);
         calculate_volume(g, p, 0.5);
         force_calculation(g, p, 0.5, 1, 1, 0);
         for (auto& [i, n] : g) check(norm(n.force) < 1e-10, "force zero at F_E = I");
       }},
      {"non-zero force (snow_tests.cpp:146)",
       [] {
         Grid g;
         Particle p = particle({0.5, 0.5, 0.5}, {0, 0, 0}, 1, 1);
         p.FE(0, 0) = 0.8;
         p.FE(1, 0) = 0;
         p.FE(2, 0) = 0;
         p2g(g, p, 1);
         force_calculation(g, p, 1, 1, 1, 0);
         const Vec3 f = g.find(NodeIdx{0, 0, 0})->second.force;
         check(near(f[0], -0.06888020833), "f_x at node 0");
         check(near(f[1], -0.02296006944), "f_y at node 0");
         check(near(f[2], -0.02296006944), "f_z at node 0");
         Vec3 tot;
         for (auto& [i, n] : g) tot += n.force;
         check(near(norm(tot), 0), "net force zero");
       }},
      {"grid velocity (snow_tests.cpp:164)",
       [] {
         Grid g;
         g[NodeIdx{0, 0, 0}].mass = 2;
         g[NodeIdx{0, 0, 0}].momentum = {6, 4, 0};
         g[NodeIdx{0, 0, 0}].force = {2, -4, 1};
         g[NodeIdx{0, 0, 1}].mass = 0;
         g[NodeIdx{0, 0, 1}].force = {2, -4, 1};
         grid_velocity(g, {0, -9.81, 0}, 0.01);
         const Vec3 v0 = g[NodeIdx{0, 0, 0}].velocity, v1 = g[NodeIdx{0, 0, 1}].velocity;
         check(near(v0[0], 3.01) && near(v0[1], 1.8819) && near(v0[2], 0.005), "v = p/m + dt(f/m+g)");
         check(near(v1[0], 0) && near(v1[1], 0) && near(v1[2], 0), "massless node untouched");
       }},
      {"grid collision outside (snow_tests.cpp:182)",
       [] {
         Grid g;
         g[NodeIdx{0, 1, 0}].velocity = {2, -3, 0};
         grid_collisions(g, ground(1), 0.1);
         check(dist(g[NodeIdx{0, 1, 0}].velocity, {2, -3, 0}) < 1e-10, "phi > 0 untouched");
       }},
      {"grid collision escaping (snow_tests.cpp:193)",
       [] {
         Grid g;
         g[NodeIdx{0, -1, 0}].velocity = {2, 3, 0};
         grid_collisions(g, ground(1), 1);
         check(dist(g[NodeIdx{0, -1, 0}].velocity, {2, 3, 0}) < 1e-10, "v_n >= 0 untouched");
       }},
      {"grid collision sticking (snow_tests.cpp:204)",
       [] {
         Grid g;
         g[NodeIdx{0, -1, 0}].velocity = {0.2, -3, 0};
         grid_collisions(g, ground(0.6), 0.1);
         check(dist(g[NodeIdx{0, -1, 0}].velocity, {0, 0, 0}) < 1e-10, "stick");
       }},
      {"grid collision sliding (snow_tests.cpp:215)",
       [] {
         Grid g;
         g[NodeIdx{0, -1, 0}].velocity = {2, -3, 0};
         grid_collisions(g, ground(0.2), 0.1);
         check(dist(g[NodeIdx{0, -1, 0}].velocity, {1.4, 0, 0}) < 1e-10, "slide");
       }},
      {"rigid translation (snow_tests.cpp:226)",
       [] {
         Grid g = lattice_grid([](int, int, int) { return Vec3{3, -2, 1}; });
         Particle p = particle({0.15, 0.15, 0.15}, {0, 0, 0}, 0, 0);
         stress_update(g, p, 0.1, 0.1, 0.1, 0.1);
         check(frob(p.FE - Mat3::identity()) < 1e-10, "F_E = I");
         check(frob(p.FP - Mat3::identity()) < 1e-10, "F_P = I");
       }},
      {"elastic (snow_tests.cpp:248)",
       [] {
         Grid g = lattice_grid([](int, int, int) { return Vec3{3, -2, 1}; });
         Particle p = particle({0.15, 0.15, 0.15}, {0, 0, 0}, 0, 0);
         p.FE = diag3(0.99, 1, 1);
         stress_update(g, p, 0.1, 0.1, 0.025, 0.1);
         check(frob(p.FE - diag3(0.99, 1, 1)) < 1e-10, "F_E unchanged");
         check(frob(p.FP - Mat3::identity()) < 1e-10, "F_P = I");
       }},
      {"plastic (snow_tests.cpp:274)",
       [] {
         Grid g = lattice_grid([](int, int, int) { return Vec3{3, -2, 1}; });
         Particle p = particle({0.15, 0.15, 0.15}, {0, 0, 0}, 0, 0);
         p.FE = diag3(0.95, 1, 1);
         stress_update(g, p, 0.1, 0.1, 0.025, 0.1);
         check(frob(p.FE - diag3(0.975, 1, 1)) < 1e-10, "F_E clamped");
         check(frob(p.FP - diag3(0.95 / 0.975, 1, 1)) < 1e-10, "F_P takes the rest");
         check(frob(p.FE * p.FP - diag3(0.95, 1, 1)) < 1e-10, "F_E F_P = trial F");
       }},
      {"linear velocity field (snow_tests.cpp:303)",
       [] {
         Grid g = lattice_grid([](int i, int, int) { return Vec3{-0.1 * (0.1 * i), 0, 0}; });
         Particle p = particle({0.15, 0.15, 0.15}, {0, 0, 0}, 0, 0);
         stress_update(g, p, 0.1, 0.1, 0.025, 0.1);
         check(frob(p.FE - diag3(0.99, 1, 1)) < 1e-10, "F_E = diag(.99,1,1)");
         check(frob(p.FP - Mat3::identity()) < 1e-10, "F_P = I");
       }},
      {"G2P (snow_tests.cpp:329)",
       [] {
         Grid g;
         Particle p = particle({0.15, 0.15, 0.15}, {2, 3, 4}, 0, 0);
         p2g(g, p, 0.1);
         for (auto& [i, n] : g) n.mass = 1, n.momentum = {2, 3, 4}, n.velocity = {2, 2, 4};
         g2p(g, p, 0.1, 0.95);
         check(dist(p.v, {2, 2, 4}) < 1e-10, "v = (2,2,4)");
       }},
      {"FLIP/PIC blend (snow_tests.cpp:345)",
       [] {
         Grid g;
         Particle p = particle({0.15, 0.15, 0.15}, {10, 0, 0}, 0, 0);
         p2g(g, p, 0.1);
         for (auto& [i, n] : g) n.mass = 1, n.momentum = {1, 0, 0}, n.velocity = {3, 0, 0};
         g2p(g, p, 0.1, 0.95);
         check(dist(p.v, {11.55, 0, 0}) < 1e-10, "v_x = 11.55");
       }},
      {"particle collision outside (snow_tests.cpp:361)",
       [] {
         Particle p = particle({0, 1, 0}, {2, -3, 0}, 1, 1);
         particle_collisions(p, ground(1));
         check(dist(p.v, {2, -3, 0}) < 1e-10, "phi > 0 untouched");
       }},
      {"particle collision escaping (snow_tests.cpp:371)",
       [] {
         Particle p = particle({0, -1, 0}, {2, 3, 0}, 1, 1);
         particle_collisions(p, ground(1));
         check(dist(p.v, {2, 3, 0}) < 1e-10, "v_n >= 0 untouched");
       }},
      {"particle collision sticking (snow_tests.cpp:381)",
       [] {
         Particle p = particle({0, -1, 0}, {0.2, -3, 0}, 1, 1);
         particle_collisions(p, ground(0.6));
         check(dist(p.v, {0, 0, 0}) < 1e-10, "stick");
       }},
      {"particle collision sliding (snow_tests.cpp:391)",
       [] {
         Particle p = particle({0, -1, 0}, {2, -3, 0}, 1, 1);
         particle_collisions(p, ground(0.2));
         check(dist(p.v, {1.4, 0, 0}) < 1e-10, "slide");
       }},
      {"position update (snow_tests.cpp:401)",
       [] {
         Particle p = particle({1, 2, 3}, {2, -1, 0.5}, 1, 1);
         position_update(p, 0.1);
         check(dist(p.x, {1.2, 1.9, 3.05}) < 1e-10, "x + dt v");
       }},
  };
  int n = 0;
  for (const Case& c : cases) {
    const int before = failures;
    c.body();
    std::printf("%-48s %s\n", c.name, failures == before ? "ok" : "FAILED");
    ++n;
  }
  // SVD sanity beyond the reference's cases: reconstruction, orthogonality and
  // non-negative sorted singular values on a few awkward matrices.
  const double mats[][9] = {
      {1, 0, 0, 0, 1, 0, 0, 0, 1},
      {0.8, 0, 0, 0, 1, 0, 0, 0, 1},
      {-1, 0, 0, 0, 1, 0, 0, 0, 1},
      {1, 2, 3, 4, 5, 6, 7, 8, 10},
      {1, 1e-9, 0, 0, 1, 1e-9, 0, 0, 1},
      {0, 0, 0, 0, 0, 0, 0, 0, 0},
      {1, 2, 3, 2, 4, 6, 3, 6, 9},
      {0.99, 0.01, -0.02, 0.005, 1.01, 0.003, 0.0, -0.01, 0.97},
  };
  for (const auto& m : mats) {
    Mat3 F, U, V;
    Vec3 s;
    std::memcpy(F.a, m, sizeof F.a);
    svd3(F, U, s, V);
    const Mat3 R = U * diag(s) * transpose(V);
    check(frob(R - F) <= 1e-13 * std::max(1.0, frob(F)), "svd reconstructs");
    check(frob(transpose(U) * U - Mat3::identity()) < 1e-13, "U orthogonal");
    check(frob(transpose(V) * V - Mat3::identity()) < 1e-13, "V orthogonal");
    check(s[0] >= s[1] && s[1] >= s[2] && s[2] >= 0, "sigma sorted, >= 0");
  }
  std::printf("%d reference cases + svd checks: %s\n", n, failures ? "FAILED" : "all passed");
  return failures ? 1 : 0;
}
