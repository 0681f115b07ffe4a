// Internals shared by the C++ API's translation units.
#pragma once

#include <vector>

#include "snow/grid.hpp"
#include "snow_gpu.h"

namespace snow::host
{
// Throws std::runtime_error with the C ABI's last error text on failure.
void check(int rc);
}  // namespace snow::host

// Resident mode (snow::gpu::set_resident): one step of the vector's GPU copy.
void snow_host_resident_step(std::vector<Particle>& snow, const snow_step_params& p,
                             const std::vector<snow_collider>& colliders, snow_step_timings& t);
// Forgets the resident copy (its host vector changed or was replaced).
void snow_host_invalidate_resident();
// If `snow` is the resident vector, copies the GPU state into `out` (n records)
// and returns true.
bool snow_host_resident_copy(const std::vector<Particle>& snow, double* out);
// The positions only (x y z per particle) of a vector kept on the GPU; false
// when `snow` is not the resident vector or the host copy is current.
bool snow_host_resident_positions(const std::vector<Particle>& snow, double* xyz);
