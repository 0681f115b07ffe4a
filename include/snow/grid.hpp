// The explicit MPM step and its stages (reference include/snow/grid.hpp), run on
// the GPU.  Signatures and types are the reference's, so callers of the
// reference solver compile and link unchanged against libsnow.so.
//
//  * setup() and step() run the fused CUDA kernels over the whole particle set
//    (C ABI snow_gpu_setup / snow_gpu_step).  By default every step() call
//    uploads the particles, steps and downloads them, so the caller's vector is
//    always current -- the reference's semantics.  snow::gpu::set_resident(true)
//    keeps the state on the GPU between calls instead (see below).
//  * The stage functions (P2G, calculate_volume, force_calculation, ...) take
//    the reference's host Grid (an unordered_map of nodes); they upload the
//    nodes and particles they need, run the same device code as step(), and
//    merge the results back into the map.
//  * The `stencils` argument of step() is accepted and left untouched: its node
//    pointers would dangle once step() returns (the grid is local to a step),
//    and the GPU never materialises 64-entry stencils.
//  * N, N_dash and build_stencil are evaluated on the host from the same
//    B-spline code the kernels use; they return host data.
//  * constitutive_differential, index_nodes, deformation_differential,
//    force_differential, apply_A and Conjugate_residual, which the reference
//    declares and never defines, implement Stomakhin et al.'s semi-implicit
//    velocity update: the particle work on the GPU (snow_gpu_stage_*), the
//    Krylov vectors over the nodes with mass.  Conjugate_residual solves
//    (I + beta dt^2 M^-1 H) v = v* from the nodes' velocities, until
//    <r, r>_M <= squared_tolerance <v*, v*>_M (mass-weighted) or
//    maximum_iterations, and writes the velocities back.
#pragma once

#include <array>
#include <cstddef>
#include <unordered_map>
#include <vector>

#include <Eigen/Dense>

#include "snow/collision.hpp"
#include "snow/debug.hpp"
#include "snow/particle.hpp"

struct GridNode
{
    double mass = 0.0;
    double density = 0.0;
    Eigen::Vector3d momentum = Eigen::Vector3d::Zero();
    Eigen::Vector3d velocity = Eigen::Vector3d::Zero();
    Eigen::Vector3d force = Eigen::Vector3d::Zero();
    Eigen::Vector3d delta_v = Eigen::Vector3d::Zero();
    Eigen::Vector3d delta_force = Eigen::Vector3d::Zero();
    bool colision_constrained = false;
};

struct GridIndex
{
    int i;
    int j;
    int k;

    auto operator<=>(const GridIndex&) const = default;
};

struct GridIndexHash
{
    std::size_t operator()(const GridIndex& index) const noexcept
    {
        unsigned long long h = static_cast<unsigned int>(index.i) * 0xD6E8FEB86659FD93ull;
        h = (h ^ (h >> 29)) + static_cast<unsigned int>(index.j) * 0x9E3779B97F4A7C15ull;
        h = (h ^ (h >> 31)) + static_cast<unsigned int>(index.k) * 0xC2B2AE3D27D4EB4Full;
        return static_cast<std::size_t>(h ^ (h >> 33));
    }
};

struct StencilEntry
{
    GridIndex index;
    double weight{0.0};
    Eigen::Vector3d gradient{Eigen::Vector3d::Zero()};
    GridNode* node{nullptr};
};

using ParticleStencil = std::array<StencilEntry, 64>;
using Grid = std::unordered_map<GridIndex, GridNode, GridIndexHash>;
using KrylovVector = std::vector<Eigen::Vector3d>;

double N(const double& a, const double& b);
double N_dash(const double& grid_node, const double& particle_coordinate);
Eigen::Matrix3d constitutive_differential(const Particle& particle, const Eigen::Matrix3d& delta_f, double mu_0,
                                          double lambda_0, double hardening_coefficient);
ParticleStencil build_stencil(const Particle& particle, double grid_spacing);
void P2G(Grid& grid, const Particle& particle, ParticleStencil& stencil);
void P2G(Grid& grid, const Particle& particle, double grid_spacing);
std::vector<GridNode*> index_nodes(Grid& grid);
void calculate_volume(Grid& grid, Particle& particle, double grid_spacing);
Eigen::Matrix3d force_constitutive(const Particle& particle, double mu_0, double lambda_0,
                                   double hardening_coefficient);
void force_grid_accumulation(const Eigen::Matrix3d& dphidF_E, const Particle& particle,
                             const ParticleStencil& stencil);
void force_calculation(Grid& grid, const Particle& particle, double grid_spacing, double mu_0, double lambda_0,
                       double hardening_coefficient);
void grid_velocity(Grid& grid, const Eigen::Vector3d gravity, const double time_step);
void grid_collisions(Grid& grid, const std::vector<CollisionBody>& collisions, double grid_spacing);
void stress_update(const Grid& grid, Particle& particle, double grid_spacing, double time_step,
                   double max_compression, double max_stretch);
Eigen::Matrix3d deformation_differential(const Grid& grid, const Particle& particle, double grid_spacing,
                                         double time_step);
void force_differential(Grid& grid, const Particle& particle, double grid_spacing, double time_step, double mu_0,
                        double lambda_0, double hardening_coefficient);
KrylovVector apply_A(Grid& grid, const std::vector<Particle>& snow, const std::vector<GridNode*>& krylov_nodes,
                     const KrylovVector& q, double grid_spacing, double time_step, double mu_0, double lambda_0,
                     double hardening_coefficent, double beta);
void Conjugate_residual(Grid& grid, const std::vector<Particle>& snow, const std::vector<GridNode*>& krylov_nodes,
                        double grid_spacing, double time_step, double mu_0, double lambda_0,
                        double hardening_coefficent, double beta, double squared_tolerance, int maximum_iterations);
void G2P(const Grid& grid, Particle& particle, double grid_spacing, double alpha);
void particle_collisions(Particle& particle, const std::vector<CollisionBody>& colliders);
void position_update(Particle& particle, double time_step);
void setup(std::vector<Particle>& snow, double grid_spacing);
void step(std::vector<Particle>& snow, const std::vector<CollisionBody>& colliders,
          std::vector<ParticleStencil>& stencils, Eigen::Vector3d gravity, double time_step, double grid_spacing,
          double mu_0, double lambda_0, double hardening_coefficient, double max_compression, double max_stretch,
          double alpha, StepTimings& timings);

// GPU residency (no reference counterpart).
namespace snow::gpu
{
// With residency on, step() keeps the particle state of the vector it was last
// given on the GPU (keyed by its data pointer and size) and does not copy it
// back; sync_to_host() (and export_particles) copy it into the vector.  The
// vector must not be modified between steps unless invalidate() is called.
void set_resident(bool on);
bool resident();
void sync_to_host(std::vector<Particle>& snow);
void invalidate();
// Resident steps fill StepTimings per stage by default, which times each
// stage between events and waits for the step.  With stage timings off a
// resident step() launches the captured step graph and returns at once,
// leaving StepTimings untouched; the GPU runs ahead of the host until the next
// read-back (sync_to_host, export_particles, a non-resident call).
void set_stage_timings(bool on);
}  // namespace snow::gpu
