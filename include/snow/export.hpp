// Frame export (reference include/snow/export.hpp): writes
// output/frame_<6-digit frame>.csv with header "x,y,z" and one row per particle
// (x, -z, y) -- solver axes to Blender axes -- at the default stream precision.
#pragma once

#include <vector>

#include "snow/particle.hpp"

void export_particles(const std::vector<Particle>& particles, int frame_no);

namespace snow::gpu
{
// Not in the reference: the same file written on a background thread.  The
// particle state is copied (read back from the GPU for a resident vector)
// before the call returns, so the caller may step on; wait_exports() returns
// once every file is written.
void export_particles_async(const std::vector<Particle>& particles, int frame_no);
void wait_exports();
}  // namespace snow::gpu
