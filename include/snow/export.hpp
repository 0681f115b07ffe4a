// Frame export (reference include/snow/export.hpp): writes
// output/frame_<6-digit frame>.csv with header "x,y,z" and one row per particle
// (x, -z, y) -- solver axes to Blender axes -- at the default stream precision.
#pragma once

#include <vector>

#include "snow/particle.hpp"

void export_particles(const std::vector<Particle>& particles, int frame_no);
