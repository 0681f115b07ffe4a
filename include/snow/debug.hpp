// Per-stage step timings (reference include/snow/debug.hpp).  The GPU step
// accumulates device time from CUDA events; its fused kernels report under
// the first stage each contains: stencil (keys, sort, block build), p2g
// (P2G with the constitutive force and its scatter), grid_velocity (grid
// update with collisions), stress_update (elastoplastic update, G2P,
// particle collisions, advection).
#pragma once

struct StepTimings
{
    double stencil{0.0};
    double p2g{0.0};
    double forces_constitutive{0.0};
    double forces_accumulative{0.0};
    double grid_velocity{0.0};
    double grid_collisions{0.0};
    double stress_update{0.0};
    double g2p{0.0};
    double particle_collisions{0.0};
    double position_update{0.0};
};

// Prints each stage's milliseconds and share; returns their sum.
double print_timings(StepTimings timings);
