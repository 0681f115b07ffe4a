// The reference's unit tests (tests/snow_tests.cpp:30-407 of the reference
// tree), restated against the GPU-backed drop-in API (libsnow.so): every stage
// call below runs on the device.  Plus API behaviour the reference relies on:
// setup()+step() conservation, residency, CSV import errors and frame export.
// Exit status 0 = all pass.
#include <algorithm>
#include <cmath>
#include <cstdio>
#include <filesystem>
#include <fstream>
#include <functional>
#include <sstream>
#include <stdexcept>
#include <string>
#include <vector>

#include "snow/collision.hpp"
#include "snow/export.hpp"
#include "snow/grid.hpp"
#include "snow/import.hpp"
#include "snow/particle.hpp"

namespace
{
int failures = 0;
void expect(bool ok, const std::string& what)
{
    if (!ok)
    {
        std::printf("FAIL: %s\n", what.c_str());
        ++failures;
    }
}
bool close(double a, double b, double tol = 1e-10) { return std::abs(a - b) < tol; }
double dist(const Eigen::Vector3d& a, const Eigen::Vector3d& b) { return (a - b).norm(); }

Grid lattice(const std::function<Eigen::Vector3d(int, int, int)>& v)
{
    Grid g;
    for (int i = 0; i < 4; ++i)
        for (int j = 0; j < 4; ++j)
            for (int k = 0; k < 4; ++k) g[GridIndex{i, j, k}].velocity = v(i, j, k);
    return g;
}
std::vector<CollisionBody> ground(double mu) { return {make_plane({0, 0, 0}, {0, 1, 0}, mu)}; }
Eigen::Matrix3d diag(double a, double b, double c) { return Eigen::Vector3d{a, b, c}.asDiagonal(); }

struct Case
{
    const char* name;
    std::function<void()> body;
};
}  // namespace

int main()
{
    const Case cases[] = {
        {"spline values", [] {
             expect(close(N(1, 1), 2.0 / 3.0) && close(N(1, 2), 1.0 / 6.0), "N at 0 and 1");
             expect(N(1, 3) == 0 && N(1, 10) == 0, "N outside support");
             expect(close(N(1.5, 0.75), N(0.75, 1.5)), "N symmetric");
         }},
        {"spline slopes", [] {
             expect(close(N_dash(4, 4.3), -N_dash(4.3, 4)), "N' antisymmetric");
             expect(close(N_dash(1, 1), 0) && close(N_dash(0, 1), -0.5), "N' at 0 and 1");
             expect(close(N_dash(0, 2), 0) && close(N_dash(0, 0.5), -0.625), "N' at 2 and 0.5");
         }},
        {"P2G conserves one particle", [] {
             Grid g;
             P2G(g, Particle({2.1, 3.5, 4.7}, {3, -2, 0.5}, 2, 1), 0.5);
             double m = 0;
             Eigen::Vector3d p = Eigen::Vector3d::Zero();
             for (auto& [i, n] : g) m += n.mass, p += n.momentum;
             expect(close(m, 2) && dist(p, {6, -4, 1}) < 1e-10, "mass 2, momentum (6,-4,1)");
             expect(g.size() == 64, "64 nodes inserted");
         }},
        {"P2G sums two particles", [] {
             Grid g;
             P2G(g, Particle({2.1, 3.5, 4.7}, {3, -2, 0.5}, 2, 1), 0.5);
             P2G(g, Particle({2.3, 3.7, 4.4}, {-1, 4, 2}, 1.5, 1), 0.5);
             double m = 0;
             Eigen::Vector3d p = Eigen::Vector3d::Zero();
             for (auto& [i, n] : g) m += n.mass, p += n.momentum;
             expect(close(m, 3.5) && dist(p, {4.5, 2, 4}) < 1e-10, "mass 3.5, momentum (4.5,2,4)");
         }},
        {"P2G is translation invariant", [] {
             Grid a, b;
             P2G(a, Particle({2.15, 3.35, 4.65}, {1, 2, 3}, 1, 1), 0.5);
             P2G(b, Particle({2.65, 3.35, 4.65}, {1, 2, 3}, 1, 1), 0.5);
             expect(a.size() == b.size(), "same node count");
             for (auto& [i, n] : a)
             {
                 auto it = b.find(GridIndex{i.i + 1, i.j, i.k});
                 expect(it != b.end(), "shifted node present");
                 if (it == b.end()) continue;
                 expect(close(n.mass, it->second.mass) && dist(n.momentum, it->second.momentum) < 1e-10,
                        "shifted node values");
             }
         }},
        {"P2G with a stencil caches node pointers", [] {
             Grid g;
             Particle p({2.1, 3.5, 4.7}, {3, -2, 0.5}, 2, 1);
             ParticleStencil st = build_stencil(p, 0.5);
             P2G(g, p, st);
             double m = 0;
             for (auto& e : st) m += e.node ? e.node->mass : -1e9;
             expect(close(m, 2), "stencil nodes hold the mass");
         }},
        {"rest volume", [] {
             Grid g;
             Particle p({1, 2, 3}, {1, 2, 3}, 1, 7);
             P2G(g, p, 0.5);
             calculate_volume(g, p, 0.5);
             expect(close(p.V_p0, 1), "V_p0 = 1");
         }},
        {"no force at rest", [] {
             Grid g;
             Particle p({1, 2, 3}, {1, 2, 3}, 1, 7);
             P2G(g, p, 0.5);
             calculate_volume(g, p, 0.5);
             force_calculation(g, p, 0.5, 1, 1, 0);
             for (auto& [i, n] : g) expect(n.force.norm() < 1e-10, "force zero at F_E = I");
         }},
        {"force of a compressed particle", [] {
             Grid g;
             Particle p({0.5, 0.5, 0.5}, {0, 0, 0}, 1, 1);
             p.F_E.col(0) << 0.8, 0, 0;
             P2G(g, p, 1);
             force_calculation(g, p, 1, 1, 1, 0);
             const Eigen::Vector3d f = g.find({0, 0, 0})->second.force;
             expect(close(f[0], -0.06888020833) && close(f[1], -0.02296006944) && close(f[2], -0.02296006944),
                    "node (0,0,0) force");
             Eigen::Vector3d tot = Eigen::Vector3d::Zero();
             for (auto& [i, n] : g) tot += n.force;
             expect(tot.norm() < 1e-10, "net force zero");
         }},
        {"constitutive + accumulation = force_calculation", [] {
             Particle p({0.5, 0.5, 0.5}, {0, 0, 0}, 1, 1);
             p.F_E.col(0) << 0.8, 0, 0;
             Grid a, b;
             ParticleStencil st = build_stencil(p, 1);
             P2G(a, p, st);
             force_grid_accumulation(force_constitutive(p, 1, 1, 0), p, st);
             P2G(b, p, 1);
             force_calculation(b, p, 1, 1, 1, 0);
             for (auto& [i, n] : a) expect(dist(n.force, b[i].force) < 1e-12, "same nodal force");
         }},
        {"grid velocity", [] {
             Grid g;
             g[{0, 0, 0}].mass = 2;
             g[{0, 0, 0}].momentum = {6, 4, 0};
             g[{0, 0, 0}].force = {2, -4, 1};
             g[{0, 0, 1}].mass = 0;
             g[{0, 0, 1}].force = {2, -4, 1};
             grid_velocity(g, {0, -9.81, 0}, 0.01);
             expect(dist(g[{0, 0, 0}].velocity, {3.01, 1.8819, 0.005}) < 1e-10, "p/m + dt(f/m + g)");
             expect(g[{0, 0, 1}].velocity.norm() == 0, "massless node untouched");
         }},
        {"grid collisions", [] {
             Grid g;
             g[{0, 1, 0}].velocity = {2, -3, 0};
             grid_collisions(g, ground(1), 0.1);
             expect(dist(g[{0, 1, 0}].velocity, {2, -3, 0}) < 1e-10, "outside");
             Grid h;
             h[{0, -1, 0}].velocity = {2, 3, 0};
             grid_collisions(h, ground(1), 1);
             expect(dist(h[{0, -1, 0}].velocity, {2, 3, 0}) < 1e-10, "escaping");
             Grid s;
             s[{0, -1, 0}].velocity = {0.2, -3, 0};
             grid_collisions(s, ground(0.6), 0.1);
             expect(s[{0, -1, 0}].velocity.norm() < 1e-10, "sticking");
             Grid l;
             l[{0, -1, 0}].velocity = {2, -3, 0};
             grid_collisions(l, ground(0.2), 0.1);
             expect(dist(l[{0, -1, 0}].velocity, {1.4, 0, 0}) < 1e-10, "sliding");
         }},
        {"stress update: rigid, elastic, plastic, linear field", [] {
             const auto uniform = [](int, int, int) { return Eigen::Vector3d{3, -2, 1}; };
             Particle r({0.15, 0.15, 0.15}, {0, 0, 0}, 0, 0);
             stress_update(lattice(uniform), r, 0.1, 0.1, 0.1, 0.1);
             expect((r.F_E - Eigen::Matrix3d::Identity()).norm() < 1e-10 &&
                        (r.F_P - Eigen::Matrix3d::Identity()).norm() < 1e-10,
                    "rigid translation");
             Particle e({0.15, 0.15, 0.15}, {0, 0, 0}, 0, 0);
             e.F_E = diag(0.99, 1, 1);
             stress_update(lattice(uniform), e, 0.1, 0.1, 0.025, 0.1);
             expect((e.F_E - diag(0.99, 1, 1)).norm() < 1e-10 && (e.F_P - Eigen::Matrix3d::Identity()).norm() < 1e-10,
                    "elastic");
             Particle p({0.15, 0.15, 0.15}, {0, 0, 0}, 0, 0);
             p.F_E = diag(0.95, 1, 1);
             stress_update(lattice(uniform), p, 0.1, 0.1, 0.025, 0.1);
             expect((p.F_E - diag(0.975, 1, 1)).norm() < 1e-10, "plastic F_E");
             expect((p.F_P - diag(0.95 / 0.975, 1, 1)).norm() < 1e-10, "plastic F_P");
             expect((p.F_E * p.F_P - diag(0.95, 1, 1)).norm() < 1e-10, "F_E F_P = trial");
             Particle l({0.15, 0.15, 0.15}, {0, 0, 0}, 0, 0);
             stress_update(lattice([](int i, int, int) { return Eigen::Vector3d{-0.1 * (0.1 * i), 0, 0}; }), l, 0.1,
                           0.1, 0.025, 0.1);
             expect((l.F_E - diag(0.99, 1, 1)).norm() < 1e-10 && (l.F_P - Eigen::Matrix3d::Identity()).norm() < 1e-10,
                    "linear velocity field");
         }},
        {"G2P and the PIC/FLIP blend", [] {
             Grid g;
             Particle p({0.15, 0.15, 0.15}, {2, 3, 4}, 0, 0);
             P2G(g, p, 0.1);
             for (auto& [i, n] : g) n.mass = 1, n.momentum = {2, 3, 4}, n.velocity = {2, 2, 4};
             G2P(g, p, 0.1, 0.95);
             expect(dist(p.v_p, {2, 2, 4}) < 1e-10, "uniform grid velocity");
             Grid f;
             Particle q({0.15, 0.15, 0.15}, {10, 0, 0}, 0, 0);
             P2G(f, q, 0.1);
             for (auto& [i, n] : f) n.mass = 1, n.momentum = {1, 0, 0}, n.velocity = {3, 0, 0};
             G2P(f, q, 0.1, 0.95);
             expect(dist(q.v_p, {11.55, 0, 0}) < 1e-10, "11.55");
         }},
        {"particle collisions", [] {
             Particle a({0, 1, 0}, {2, -3, 0}, 1, 1), b({0, -1, 0}, {2, 3, 0}, 1, 1);
             Particle c({0, -1, 0}, {0.2, -3, 0}, 1, 1), d({0, -1, 0}, {2, -3, 0}, 1, 1);
             particle_collisions(a, ground(1));
             particle_collisions(b, ground(1));
             particle_collisions(c, ground(0.6));
             particle_collisions(d, ground(0.2));
             expect(dist(a.v_p, {2, -3, 0}) < 1e-10 && dist(b.v_p, {2, 3, 0}) < 1e-10, "outside / escaping");
             expect(c.v_p.norm() < 1e-10 && dist(d.v_p, {1.4, 0, 0}) < 1e-10, "sticking / sliding");
         }},
        {"position update", [] {
             Particle p({1, 2, 3}, {2, -1, 0.5}, 1, 1);
             position_update(p, 0.1);
             expect(dist(p.x_p, {1.2, 1.9, 3.05}) < 1e-10, "x + dt v");
         }},
        {"setup + step conserve mass; resident equals literal", [] {
             std::vector<Particle> a;
             for (int i = 0; i < 10; ++i)
                 for (int j = 0; j < 10; ++j)
                     for (int k = 0; k < 10; ++k)
                         a.emplace_back(Eigen::Vector3d{0.3 + 0.011 * i, 0.3 + 0.011 * j, 0.3 + 0.011 * k},
                                        Eigen::Vector3d{0.1, -1.0, 0.2}, 0.0005, 0.0);
             setup(a, 0.02);
             expect(a[0].V_p0 > 0, "setup sets V_p0");
             std::vector<Particle> b = a;
             std::vector<ParticleStencil> st(a.size());
             StepTimings t;
             const auto cols = ground(0.2);
             for (int s = 0; s < 5; ++s)
                 step(a, cols, st, {0, -9.81, 0}, 1e-4, 0.02, 58333.3, 38888.9, 10, 0.025, 0.0075, 0.95, t);
             expect(t.p2g > 0 && t.stress_update > 0, "timings accumulate");
             snow::gpu::set_resident(true);
             for (int s = 0; s < 5; ++s)
                 step(b, cols, st, {0, -9.81, 0}, 1e-4, 0.02, 58333.3, 38888.9, 10, 0.025, 0.0075, 0.95, t);
             snow::gpu::sync_to_host(b);
             snow::gpu::set_resident(false);
             double worst = 0;
             for (std::size_t i = 0; i < a.size(); ++i)
                 worst = std::max(worst, (a[i].x_p - b[i].x_p).norm() + (a[i].F_E - b[i].F_E).norm());
             expect(worst < 1e-12, "resident and literal steps agree");
         }},
        {"foreign colliders are rejected", [] {
             std::vector<Particle> a{Particle({0.5, 0.5, 0.5}, {0, 0, 0}, 1, 1)};
             std::vector<ParticleStencil> st(1);
             StepTimings t;
             std::vector<CollisionBody> bad{
                 CollisionBody{[](const Eigen::Vector3d& x) { return x[1]; },
                               [](const Eigen::Vector3d&) { return Eigen::Vector3d{0, 1, 0}; },
                               [](const Eigen::Vector3d&) { return Eigen::Vector3d::Zero(); }, 0.2}};
             bool threw = false;
             try
             {
                 step(a, bad, st, {0, -9.81, 0}, 1e-4, 0.02, 1, 1, 1, 0.02, 0.01, 0.95, t);
             }
             catch (const std::invalid_argument&)
             {
                 threw = true;
             }
             expect(threw, "std::invalid_argument for a std::function collider");
         }},
        {"sphere and moving-plane bodies run on the device", [] {
             // a particle falling onto a resting sphere stops moving into it; one
             // under a rising plane is carried up with the plane's velocity
             std::vector<Particle> a{Particle({0.5, 0.5801, 0.5}, {0, -1, 0}, 1, 1e-6),
                                     Particle({0.2, 0.0995, 0.2}, {0, 0, 0}, 1, 1e-6)};
             std::vector<ParticleStencil> st(2);
             StepTimings t;
             std::vector<CollisionBody> bodies{snow::make_sphere({0.5, 0.5, 0.5}, 0.08, 0.0),
                                               snow::make_moving_plane({0, 0.1, 0}, {0, 3, 0}, {0, 0.5, 0}, 1.0)};
             step(a, bodies, st, {0, 0, 0}, 1e-4, 0.02, 1, 1, 1, 0.02, 0.01, 0.95, t);
             expect(a[0].v_p[1] > -1.0 + 1e-6, "sphere pushes back the falling particle");
             expect(a[1].v_p[1] > 0.0, "the rising plane lifts the particle");
         }},
        {"oriented box bodies run on the device and match their phi", [] {
             // a particle falling onto the tilted top face of a resting box is turned
             // back along the face normal; make_box's phi is the exact signed
             // distance (negative inside, the face distance at the centre)
             const Eigen::Vector3d u{1, 0.2, 0}, w{-0.2, 1, 0};
             CollisionBody box = snow::make_box({0.5, 0.4, 0.5}, {0.1, 0.05, 0.1}, u, w, 0.0);
             expect(std::abs(box.phi({0.5, 0.4, 0.5}) + 0.05) < 1e-12, "phi at the centre is -h_min");
             expect(std::abs(box.phi({0.5, 0.4, 0.8}) - 0.2) < 1e-12, "phi beyond a face");
             const Eigen::Vector3d top = box.normal({0.5, 0.44, 0.5});
             expect(std::abs(top.dot(w.normalized()) - 1.0) < 1e-12, "inside normal of the nearest face");
             std::vector<Particle> a{Particle({0.5, 0.449, 0.5}, {0, -1, 0}, 1, 1e-6)};
             std::vector<ParticleStencil> st(1);
             StepTimings t;
             std::vector<CollisionBody> bodies{box};
             step(a, bodies, st, {0, 0, 0}, 1e-4, 0.02, 1, 1, 1, 0.02, 0.01, 0.95, t);
             expect(a[0].v_p.dot(w.normalized()) > -1e-9, "the box stops motion into its face");
             bool threw = false;
             try
             {
                 snow::make_box({0, 0, 0}, {1, 1, 1}, {1, 0, 0}, {2, 0, 0}, 0.1);
             }
             catch (const std::invalid_argument&)
             {
                 threw = true;
             }
             expect(threw, "parallel box axes are rejected");
         }},
        {"CSV import, its errors, and frame export", [] {
             namespace fs = std::filesystem;
             const fs::path dir = fs::temp_directory_path() / "snow_gpu_io_test";
             fs::create_directories(dir / "output");
             auto write = [&](const char* name, const char* text) {
                 std::ofstream(dir / name) << text;
                 return (dir / name).string();
             };
             const auto g = write("g.csv", "group_id,vx,vy,vz,mass\n0,0.0,-2.0,-0.0,0.05\n\n3,1,2,3,0.5\r\n");
             const auto p = write("p.csv", "group_id,x,y,z\n0,-0.1,1.0,0.05\n3,0.2,0.3,0.4\n");
             const auto parts = import_particles(g, p);
             expect(parts.size() == 2 && parts[1].m_p == 0.5 && parts[0].v_p[1] == -2.0 && parts[0].V_p0 == 0,
                    "records assembled");
             auto fails_with = [&](const std::string& gfile, const std::string& pfile, const std::string& msg) {
                 try
                 {
                     import_particles(gfile, pfile);
                 }
                 catch (const std::runtime_error& e)
                 {
                     return std::string(e.what()).find(msg) != std::string::npos;
                 }
                 return false;
             };
             expect(fails_with((dir / "none.csv").string(), p, "File not open"), "missing file");
             expect(fails_with(write("e.csv", ""), p, "Group data file is empty"), "empty file");
             expect(fails_with(write("d.csv", "h\n1,0,0,0,1\n1,0,0,0,1\n"), p, "Duplicate group id: 1"), "duplicate");
             expect(fails_with(g, write("u.csv", "h\n7,0,0,0\n"), "undefined group id: 7"), "undefined group");
             expect(fails_with(g, write("m.csv", "h\n0,1,2\n"), "Missing CSV field: z"), "missing field");
             expect(fails_with(g, write("f.csv", "h\n0,,2,3\n"), "Empty CSV field: x"), "empty field");
             const fs::path cwd = fs::current_path();
             fs::current_path(dir);
             export_particles(parts, 7);
             std::vector<Particle> copy = parts;
             snow::gpu::export_particles_async(copy, 8);
             copy[0].x_p[0] = 99.0;  // the asynchronous export copied the state already
             snow::gpu::wait_exports();
             fs::current_path(cwd);
             auto slurp = [&](const char* f) {
                 std::ifstream in(dir / "output" / f);
                 std::stringstream ss;
                 ss << in.rdbuf();
                 return ss.str();
             };
             expect(slurp("frame_000007.csv") == "x,y,z\n-0.1,-0.05,1\n0.2,-0.4,0.3\n", "export axes and format");
             expect(slurp("frame_000008.csv") == slurp("frame_000007.csv"), "asynchronous export writes the same file");
         }},
        {"implicit update: Conjugate_residual solves what apply_A applies", [] {
             const double dx = 0.1, dt = 1e-3, mu = 1e4, lambda = 1.5e4, xi = 10;
             std::vector<Particle> snow;
             for (int i = 0; i < 4; ++i)
             {
                 Particle p({1.0 + 0.031 * i, 1.2 - 0.017 * i, 0.9 + 0.023 * i}, {0.3 * i, -0.2, 0.1}, 1.0, 1e-3);
                 p.F_E = diag(1.02, 0.97, 1.01);
                 p.F_E(0, 1) = 0.01 * i;
                 p.F_P = diag(1.0, 1.0, 0.999);
                 snow.push_back(p);
             }
             Grid g;
             for (const Particle& p : snow) P2G(g, p, dx);
             for (auto& [i, n] : g) n.velocity = n.momentum / n.mass;
             const std::vector<GridNode*> nodes = index_nodes(g);
             expect(nodes.size() == g.size(), "every node of a particle stencil has mass");
             KrylovVector want(nodes.size());
             for (std::size_t k = 0; k < nodes.size(); ++k) want[k] = nodes[k]->velocity;
             Conjugate_residual(g, snow, nodes, dx, dt, mu, lambda, xi, 1.0, 1e-28, 400);
             KrylovVector v(nodes.size());
             double moved = 0;
             for (std::size_t k = 0; k < nodes.size(); ++k)
                 v[k] = nodes[k]->velocity, moved = std::max(moved, dist(v[k], want[k]));
             expect(moved > 1e-9, "the implicit term changes the velocities");
             const KrylovVector av = apply_A(g, snow, nodes, v, dx, dt, mu, lambda, xi, 1.0);
             double err = 0;
             for (std::size_t k = 0; k < nodes.size(); ++k) err = std::max(err, dist(av[k], want[k]));
             expect(err < 1e-10, "A v = v* (" + std::to_string(err) + ")");
             for (std::size_t k = 0; k < nodes.size(); ++k) nodes[k]->velocity = want[k];
             Conjugate_residual(g, snow, nodes, dx, dt, mu, lambda, xi, 0.0, 1e-28, 400);
             double still = 0;
             for (std::size_t k = 0; k < nodes.size(); ++k) still = std::max(still, dist(nodes[k]->velocity, want[k]));
             expect(still == 0, "beta 0 keeps v*");
             const Eigen::Matrix3d dP = constitutive_differential(snow[1], Eigen::Matrix3d::Zero(), mu, lambda, xi);
             expect(dP.norm() == 0, "zero dF gives zero dP");
         }},
    };
    int n = 0;
    for (const Case& c : cases)
    {
        const int before = failures;
        try
        {
            c.body();
        }
        catch (const std::exception& e)
        {
            std::printf("EXCEPTION in %s: %s\n", c.name, e.what());
            ++failures;
        }
        std::printf("%-56s %s\n", c.name, failures == before ? "ok" : "FAILED");
        ++n;
    }
    std::printf("%d cases: %s\n", n, failures ? "FAILED" : "all passed");
    return failures ? 1 : 0;
}
