// Particle import (reference include/snow/import.hpp): groups.csv
// (group_id,vx,vy,vz,mass) and particles.csv (group_id,x,y,z), header lines
// skipped, blank lines ignored; std::runtime_error on a missing file, an empty
// file, a missing or empty field, a duplicate group id or an undefined group.
#pragma once

#include <map>
#include <string>
#include <vector>

#include <Eigen/Dense>

#include "snow/particle.hpp"

struct ParticleGroup
{
    Eigen::Vector3d velocity;
    double mass;
};

struct ParticleSeed
{
    int group_id;
    Eigen::Vector3d position;
};

std::map<int, ParticleGroup> import_groups(const std::string& filename);
std::vector<ParticleSeed> import_particle_seeds(const std::string& filename);
std::vector<Particle> assemble_particles(const std::vector<ParticleSeed>& seed,
                                         const std::map<int, ParticleGroup>& groups);
std::vector<Particle> import_particles(const std::string& filename_group,
                                       const std::string& filename_particle_seed);
