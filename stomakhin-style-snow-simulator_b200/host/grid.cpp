// The reference solver's C++ API (include/snow/grid.hpp) over the GPU C ABI.
//
// step()/setup() call the fused kernels on the whole particle vector; the
// stage functions move the reference's host Grid (an unordered_map) to node
// lists, run one stage of the same device code, and merge the result back.
#include "snow/grid.hpp"

#include <cmath>
#include <cstdint>
#include <cstring>
#include <stdexcept>
#include <string>
#include <type_traits>
#include <vector>

#include "snow_bspline.h"
#include "snow_gpu.h"
#include "snow_host_detail.hpp"

static_assert(sizeof(Particle) == SNOW_RECORD_DOUBLES * sizeof(double),
              "Particle must be 26 packed doubles to cross the C ABI");
static_assert(std::is_standard_layout_v<Eigen::Vector3d>, "Eigen types must be plain storage");

namespace snow::host
{
namespace
{
const double* record(const Particle& p) { return reinterpret_cast<const double*>(&p); }
double* record(Particle& p) { return reinterpret_cast<double*>(&p); }

constexpr int kFields = 10;  // mass, momentum[3], velocity[3], force[3]

struct NodeList
{
    std::vector<int32_t> ijk;
    std::vector<double> f;
    int64_t size() const { return static_cast<int64_t>(ijk.size() / 3); }
};

NodeList to_nodes(const Grid& grid)
{
    NodeList out;
    out.ijk.reserve(grid.size() * 3);
    out.f.reserve(grid.size() * kFields);
    for (const auto& [index, node] : grid)
    {
        out.ijk.insert(out.ijk.end(), {index.i, index.j, index.k});
        out.f.push_back(node.mass);
        for (int a = 0; a < 3; ++a) out.f.push_back(node.momentum[a]);
        for (int a = 0; a < 3; ++a) out.f.push_back(node.velocity[a]);
        for (int a = 0; a < 3; ++a) out.f.push_back(node.force[a]);
    }
    return out;
}

// The 64 stencil nodes of a particle, in the reference's i-major order.
std::array<GridIndex, 64> stencil_nodes(const Particle& p, double dx)
{
    std::array<GridIndex, 64> out{};
    int base[3];
    for (int a = 0; a < 3; ++a) base[a] = static_cast<int>(std::floor(p.x_p[a] / dx)) - 1;
    int n = 0;
    for (int i = 0; i < 4; ++i)
        for (int j = 0; j < 4; ++j)
            for (int k = 0; k < 4; ++k) out[n++] = GridIndex{base[0] + i, base[1] + j, base[2] + k};
    return out;
}

// Contributions of one particle on an empty grid (every node of the blocks its
// stencil touches), as a map from node index to fields.
std::unordered_map<GridIndex, std::array<double, kFields>, GridIndexHash> contributions(
    const NodeList& nodes)
{
    std::unordered_map<GridIndex, std::array<double, kFields>, GridIndexHash> out;
    out.reserve(static_cast<std::size_t>(nodes.size()));
    for (int64_t r = 0; r < nodes.size(); ++r)
    {
        std::array<double, kFields> f{};
        std::memcpy(f.data(), &nodes.f[kFields * r], sizeof f);
        out.emplace(GridIndex{nodes.ijk[3 * r], nodes.ijk[3 * r + 1], nodes.ijk[3 * r + 2]}, f);
    }
    return out;
}

NodeList run_p2g(const Particle& p, double dx, bool force, double mu0 = 0, double lambda0 = 0,
                 double xi = 0)
{
    NodeList out;
    const int64_t cap = 8 * 64;
    out.ijk.resize(cap * 3);
    out.f.resize(cap * kFields);
    int64_t n = 0;
    if (force)
        check(snow_gpu_stage_force(record(p), 1, dx, mu0, lambda0, xi, out.ijk.data(), out.f.data(), cap, &n));
    else
        check(snow_gpu_stage_p2g(record(p), 1, dx, out.ijk.data(), out.f.data(), cap, &n));
    out.ijk.resize(n * 3);
    out.f.resize(n * kFields);
    return out;
}

void merge_mass_momentum(Grid& grid, const Particle& p, double dx)
{
    const auto c = contributions(run_p2g(p, dx, false));
    const auto idx = stencil_nodes(p, dx);
    for (int e = 0; e < 64; ++e)
    {
        GridNode& node = grid[idx[e]];
        const auto it = c.find(idx[e]);
        if (it == c.end()) continue;
        node.mass += it->second[0];
        for (int a = 0; a < 3; ++a) node.momentum[a] += it->second[1 + a];
    }
}

std::vector<snow_collider> to_colliders(const std::vector<CollisionBody>& bodies);
}  // namespace
}  // namespace snow::host

using namespace snow::host;

double N(const double& a, const double& b) { return snow::bspline(a, b); }
double N_dash(const double& grid_node, const double& particle_coordinate)
{
    return snow::bspline_slope(grid_node, particle_coordinate);
}

ParticleStencil build_stencil(const Particle& particle, double grid_spacing)
{
    ParticleStencil stencil;
    const auto idx = stencil_nodes(particle, grid_spacing);
    double w[3][4], d[3][4];
    for (int a = 0; a < 3; ++a)
    {
        const double gp = particle.x_p[a] / grid_spacing;
        const int base = static_cast<int>(std::floor(gp)) - 1;
        for (int i = 0; i < 4; ++i)
        {
            w[a][i] = N(base + i, gp);
            d[a][i] = N_dash(base + i, gp) / grid_spacing;
        }
    }
    int n = 0;
    for (int i = 0; i < 4; ++i)
        for (int j = 0; j < 4; ++j)
            for (int k = 0; k < 4; ++k, ++n)
            {
                StencilEntry& e = stencil[n];
                e.index = idx[n];
                e.weight = w[0][i] * w[1][j] * w[2][k];
                e.gradient = Eigen::Vector3d{d[0][i] * w[1][j] * w[2][k], w[0][i] * d[1][j] * w[2][k],
                                             w[0][i] * w[1][j] * d[2][k]};
                e.node = nullptr;
            }
    return stencil;
}

void P2G(Grid& grid, const Particle& particle, ParticleStencil& stencil)
{
    // The caller's stencil carries the weights (grid.cpp:119-129): the device
    // forms m w and m v w; the nodes are inserted and their pointers cached.
    double w[64], c[64 * 4];
    for (int e = 0; e < 64; ++e) w[e] = stencil[e].weight;
    check(snow_gpu_stage_p2g_stencil(record(particle), 1, w, c));
    for (int e = 0; e < 64; ++e)
    {
        GridNode& node = grid[stencil[e].index];
        stencil[e].node = &node;
        node.mass += c[4 * e];
        for (int a = 0; a < 3; ++a) node.momentum[a] += c[4 * e + 1 + a];
    }
}

void P2G(Grid& grid, const Particle& particle, double grid_spacing)
{
    merge_mass_momentum(grid, particle, grid_spacing);
}

void calculate_volume(Grid& grid, Particle& particle, double grid_spacing)
{
    for (const GridIndex& i : stencil_nodes(particle, grid_spacing)) grid[i];  // inserts, as the reference does
    const NodeList nodes = to_nodes(grid);
    check(snow_gpu_stage_volume(nodes.ijk.data(), nodes.f.data(), nodes.size(), record(particle), 1, grid_spacing));
}

Eigen::Matrix3d force_constitutive(const Particle& particle, double mu_0, double lambda_0,
                                   double hardening_coefficient)
{
    Eigen::Matrix3d P;
    check(snow_gpu_stage_stress(record(particle), 1, mu_0, lambda_0, hardening_coefficient, P.data()));
    return P;
}

void force_grid_accumulation(const Eigen::Matrix3d& dphidF_E, const Particle& particle,
                             const ParticleStencil& stencil)
{
    double grad[64 * 3], force[64 * 3];
    for (int e = 0; e < 64; ++e)
        for (int a = 0; a < 3; ++a) grad[3 * e + a] = stencil[e].gradient[a];
    check(snow_gpu_stage_force_scatter(record(particle), 1, dphidF_E.data(), grad, force));
    for (int e = 0; e < 64; ++e)
    {
        if (!stencil[e].node) throw std::invalid_argument("force_grid_accumulation: stencil has no node pointers (run P2G first)");
        for (int a = 0; a < 3; ++a) stencil[e].node->force[a] += force[3 * e + a];
    }
}

void force_calculation(Grid& grid, const Particle& particle, double grid_spacing, double mu_0, double lambda_0,
                       double hardening_coefficient)
{
    const auto c = contributions(run_p2g(particle, grid_spacing, true, mu_0, lambda_0, hardening_coefficient));
    for (const GridIndex& i : stencil_nodes(particle, grid_spacing))
    {
        GridNode& node = grid[i];
        const auto it = c.find(i);
        if (it == c.end()) continue;
        for (int a = 0; a < 3; ++a) node.force[a] += it->second[7 + a];
    }
}

void grid_velocity(Grid& grid, const Eigen::Vector3d gravity, const double time_step)
{
    NodeList nodes = to_nodes(grid);
    check(snow_gpu_stage_grid_velocity(nodes.f.data(), nodes.size(), gravity.data(), time_step));
    int64_t r = 0;
    for (auto& [index, node] : grid)
    {
        for (int a = 0; a < 3; ++a) node.velocity[a] = nodes.f[kFields * r + 4 + a];
        ++r;
    }
}

void grid_collisions(Grid& grid, const std::vector<CollisionBody>& collisions, double grid_spacing)
{
    const auto cols = to_colliders(collisions);
    NodeList nodes = to_nodes(grid);
    check(snow_gpu_stage_grid_collisions(nodes.ijk.data(), nodes.f.data(), nodes.size(), cols.data(),
                                         static_cast<int>(cols.size()), grid_spacing));
    int64_t r = 0;
    for (auto& [index, node] : grid)
    {
        for (int a = 0; a < 3; ++a) node.velocity[a] = nodes.f[kFields * r + 4 + a];
        ++r;
    }
}

void stress_update(const Grid& grid, Particle& particle, double grid_spacing, double time_step,
                   double max_compression, double max_stretch)
{
    const NodeList nodes = to_nodes(grid);
    check(snow_gpu_stage_stress_update(nodes.ijk.data(), nodes.f.data(), nodes.size(), record(particle), 1,
                                       grid_spacing, time_step, max_compression, max_stretch));
}

void G2P(const Grid& grid, Particle& particle, double grid_spacing, double alpha)
{
    const NodeList nodes = to_nodes(grid);
    check(snow_gpu_stage_g2p(nodes.ijk.data(), nodes.f.data(), nodes.size(), record(particle), 1, grid_spacing,
                             alpha));
}

// ---------------------------------------------------------- implicit update
// The functions the reference declares for Stomakhin et al.'s semi-implicit
// update (include/snow/grid.hpp:76,80,88-92) and defines nowhere: the
// per-particle work runs in the GPU stage entry points, the bookkeeping of the
// host Grid here.

Eigen::Matrix3d constitutive_differential(const Particle& particle, const Eigen::Matrix3d& delta_f, double mu_0,
                                          double lambda_0, double hardening_coefficient)
{
    Eigen::Matrix3d dP;
    check(snow_gpu_stage_constitutive_differential(record(particle), 1, delta_f.data(), mu_0, lambda_0,
                                                   hardening_coefficient, dP.data()));
    return dP;
}

// The nodes with mass: the unknowns of the implicit solve.
std::vector<GridNode*> index_nodes(Grid& grid)
{
    std::vector<GridNode*> out;
    for (auto& [index, node] : grid)
        if (node.mass > 0) out.push_back(&node);
    return out;
}

// dt (sum_i delta_v_i grad w_i^T) F_E over the particle's stencil.
Eigen::Matrix3d deformation_differential(const Grid& grid, const Particle& particle, double grid_spacing,
                                         double time_step)
{
    const ParticleStencil st = build_stencil(particle, grid_spacing);
    double grad[64 * 3], dv[64 * 3];
    for (int e = 0; e < 64; ++e)
    {
        const auto it = grid.find(st[e].index);
        for (int a = 0; a < 3; ++a)
        {
            grad[3 * e + a] = st[e].gradient[a];
            dv[3 * e + a] = it == grid.end() ? 0.0 : it->second.delta_v[a];
        }
    }
    Eigen::Matrix3d dF;
    check(snow_gpu_stage_deformation_differential(record(particle), 1, time_step, grad, dv, dF.data()));
    return dF;
}

// delta_force += -V_p0 dP F_E^T grad w at the particle's stencil nodes, dP the
// constitutive differential of the deformation differential.
void force_differential(Grid& grid, const Particle& particle, double grid_spacing, double time_step, double mu_0,
                        double lambda_0, double hardening_coefficient)
{
    const Eigen::Matrix3d dP = constitutive_differential(
        particle, deformation_differential(grid, particle, grid_spacing, time_step), mu_0, lambda_0,
        hardening_coefficient);
    const ParticleStencil st = build_stencil(particle, grid_spacing);
    double grad[64 * 3], force[64 * 3];
    for (int e = 0; e < 64; ++e)
        for (int a = 0; a < 3; ++a) grad[3 * e + a] = st[e].gradient[a];
    check(snow_gpu_stage_force_scatter(record(particle), 1, dP.data(), grad, force));
    for (int e = 0; e < 64; ++e)
    {
        GridNode& node = grid[st[e].index];
        for (int a = 0; a < 3; ++a) node.delta_force[a] += force[3 * e + a];
    }
}

namespace
{
// The grid as a node list with each node's position in `krylov` (or -1).
NodeList krylov_list(const Grid& grid, const std::vector<GridNode*>& krylov, std::vector<int64_t>& slot)
{
    std::unordered_map<const GridNode*, int64_t> pos;
    for (std::size_t i = 0; i < krylov.size(); ++i) pos[krylov[i]] = static_cast<int64_t>(i);
    NodeList nodes = to_nodes(grid);
    slot.clear();
    for (const auto& [index, node] : grid)
    {
        const auto it = pos.find(&node);
        slot.push_back(it == pos.end() ? -1 : it->second);
    }
    return nodes;
}

std::vector<double> particle_records(const std::vector<Particle>& snow)
{
    std::vector<double> rec(snow.size() * SNOW_RECORD_DOUBLES);
    if (!snow.empty()) std::memcpy(rec.data(), snow.data(), rec.size() * sizeof(double));
    return rec;
}
}  // namespace

// (A q)_i = q_i - beta dt delta f_i(q) / m_i over the Krylov nodes (the grid's
// nodes with mass, as index_nodes gives them; other nodes take q = 0).
KrylovVector apply_A(Grid& grid, const std::vector<Particle>& snow, const std::vector<GridNode*>& krylov_nodes,
                     const KrylovVector& q, double grid_spacing, double time_step, double mu_0, double lambda_0,
                     double hardening_coefficent, double beta)
{
    if (q.size() != krylov_nodes.size()) throw std::invalid_argument("apply_A: q and krylov_nodes differ in size");
    std::vector<int64_t> slot;
    const NodeList nodes = krylov_list(grid, krylov_nodes, slot);
    std::vector<double> qq(static_cast<std::size_t>(nodes.size()) * 3, 0.0), out(qq.size());
    for (int64_t r = 0; r < nodes.size(); ++r)
        if (slot[r] >= 0)
            for (int a = 0; a < 3; ++a) qq[3 * r + a] = q[slot[r]][a];
    const std::vector<double> rec = particle_records(snow);
    check(snow_gpu_stage_implicit(nodes.ijk.data(), nodes.f.data(), nodes.size(), rec.data(),
                                  static_cast<int64_t>(snow.size()), grid_spacing, time_step, mu_0, lambda_0,
                                  hardening_coefficent, beta, 1e-24, 1, qq.data(), out.data(), nullptr));
    KrylovVector aq(krylov_nodes.size(), Eigen::Vector3d::Zero());
    for (int64_t r = 0; r < nodes.size(); ++r)
        if (slot[r] >= 0) aq[slot[r]] = Eigen::Vector3d(out[3 * r], out[3 * r + 1], out[3 * r + 2]);
    return aq;
}

// Solves A v = velocity over the Krylov nodes, from v = velocity, until
// <r, r>_M <= squared_tolerance <velocity, velocity>_M (mass-weighted) or
// maximum_iterations, and writes the velocities back.
void Conjugate_residual(Grid& grid, const std::vector<Particle>& snow, const std::vector<GridNode*>& krylov_nodes,
                        double grid_spacing, double time_step, double mu_0, double lambda_0,
                        double hardening_coefficent, double beta, double squared_tolerance, int maximum_iterations)
{
    std::vector<int64_t> slot;
    const NodeList nodes = krylov_list(grid, krylov_nodes, slot);
    std::vector<double> out(static_cast<std::size_t>(nodes.size()) * 3);
    const std::vector<double> rec = particle_records(snow);
    int iterations = 0;
    check(snow_gpu_stage_implicit(nodes.ijk.data(), nodes.f.data(), nodes.size(), rec.data(),
                                  static_cast<int64_t>(snow.size()), grid_spacing, time_step, mu_0, lambda_0,
                                  hardening_coefficent, beta, squared_tolerance, maximum_iterations, nullptr,
                                  out.data(), &iterations));
    for (int64_t r = 0; r < nodes.size(); ++r)
        if (slot[r] >= 0)
            for (int a = 0; a < 3; ++a) krylov_nodes[slot[r]]->velocity[a] = out[3 * r + a];
}

void particle_collisions(Particle& particle, const std::vector<CollisionBody>& colliders)
{
    const auto cols = to_colliders(colliders);
    check(snow_gpu_stage_particle_collisions(record(particle), 1, cols.data(), static_cast<int>(cols.size())));
}

void position_update(Particle& particle, double time_step)
{
    check(snow_gpu_stage_position_update(record(particle), 1, time_step));
}

void setup(std::vector<Particle>& snow, double grid_spacing)
{
    snow_host_invalidate_resident();
    check(snow_gpu_setup(reinterpret_cast<double*>(snow.data()), static_cast<int64_t>(snow.size()), grid_spacing));
}

void step(std::vector<Particle>& snow, const std::vector<CollisionBody>& colliders,
          std::vector<ParticleStencil>& stencils, Eigen::Vector3d gravity, double time_step, double grid_spacing,
          double mu_0, double lambda_0, double hardening_coefficient, double max_compression, double max_stretch,
          double alpha, StepTimings& timings)
{
    (void)stencils;  // never materialised on the GPU; see include/snow/grid.hpp
    snow_step_params p{};
    for (int a = 0; a < 3; ++a) p.gravity[a] = gravity[a];
    p.time_step = time_step;
    p.grid_spacing = grid_spacing;
    p.mu_0 = mu_0;
    p.lambda_0 = lambda_0;
    p.hardening_coefficient = hardening_coefficient;
    p.max_compression = max_compression;
    p.max_stretch = max_stretch;
    p.alpha = alpha;
    const auto cols = to_colliders(colliders);
    snow_step_timings t{};
    if (snow::gpu::resident())
        snow_host_resident_step(snow, p, cols, t);
    else
        check(snow_gpu_step(reinterpret_cast<double*>(snow.data()), static_cast<int64_t>(snow.size()), &p,
                            cols.data(), static_cast<int>(cols.size()), 1, &t));
    timings.stencil += t.stencil;
    timings.p2g += t.p2g;
    timings.forces_constitutive += t.forces_constitutive;
    timings.forces_accumulative += t.forces_accumulative;
    timings.grid_velocity += t.grid_velocity;
    timings.grid_collisions += t.grid_collisions;
    timings.stress_update += t.stress_update;
    timings.g2p += t.g2p;
    timings.particle_collisions += t.particle_collisions;
    timings.position_update += t.position_update;
}

namespace snow::host
{
namespace
{
std::vector<snow_collider> to_colliders(const std::vector<CollisionBody>& bodies)
{
    std::vector<snow_collider> out;
    for (const CollisionBody& b : bodies)
    {
        const auto* vel = b.velocity.target<snow::ConstantVelocity>();
        const auto* d = b.phi.target<snow::PlaneDistance>();
        const auto* nrm = b.normal.target<snow::PlaneNormal>();
        const auto* sd = b.phi.target<snow::SphereDistance>();
        const auto* sn = b.normal.target<snow::SphereNormal>();
        const auto* bd = b.phi.target<snow::BoxDistance>();
        const auto* bn = b.normal.target<snow::BoxNormal>();
        snow_collider c{};
        if (vel && d && nrm && d->unit_normal == nrm->unit_normal)
        {
            c.kind = SNOW_COLLIDER_PLANE;
            for (int a = 0; a < 3; ++a)
            {
                c.point[a] = d->point[a];
                c.normal[a] = d->unit_normal[a];
            }
        }
        else if (vel && sd && sn && sd->center == sn->center && sd->radius > 0.0)
        {
            c.kind = SNOW_COLLIDER_SPHERE;
            for (int a = 0; a < 3; ++a) c.point[a] = sd->center[a];
            c.param[0] = sd->radius;
        }
        else if (vel && bd && bn && bd->center == bn->center && bd->u == bn->u && bd->w == bn->w &&
                 bd->half == bn->half)
        {
            c.kind = SNOW_COLLIDER_BOX;
            for (int a = 0; a < 3; ++a)
            {
                c.point[a] = bd->center[a];
                c.normal[a] = bd->u[a];
                c.axis[a] = bd->w[a];
                c.extent[a] = bd->half[a];
            }
        }
        else
        {
            throw std::invalid_argument(
                "collider is not a make_plane, snow::make_moving_plane, snow::make_sphere or snow::make_box "
                "body (a std::function cannot execute on the device)");
        }
        for (int a = 0; a < 3; ++a) c.velocity[a] = vel->value[a];
        c.friction = b.friction;
        out.push_back(c);
    }
    return out;
}
}  // namespace
}  // namespace snow::host
