// print_timings (reference src/debug.cpp:5-30): each stage's milliseconds and share.
#include <iostream>

#include "snow/debug.hpp"

double print_timings(StepTimings t)
{
    const double total = t.stencil + t.p2g + t.forces_constitutive + t.forces_accumulative + t.grid_velocity +
                         t.grid_collisions + t.stress_update + t.g2p + t.particle_collisions + t.position_update;
    const struct
    {
        const char* name;
        double ms;
    } rows[] = {{"Stencil", t.stencil},
                {"P2G", t.p2g},
                {"Forces constitutive", t.forces_constitutive},
                {"Forces accumulative", t.forces_accumulative},
                {"Grid velocity", t.grid_velocity},
                {"Grid collisions", t.grid_collisions},
                {"Stress update", t.stress_update},
                {"G2P", t.g2p},
                {"Particle collisions", t.particle_collisions},
                {"Position update", t.position_update}};
    for (const auto& r : rows) std::cout << r.name << ": " << r.ms << "ms  " << 100.0 * r.ms / total << "% \n";
    return total;
}
