// snow_frames: the reference's demo frame loop (src/main.cpp:33-60) on the
// drop-in API -- import groups.csv/particles.csv, setup(), then frames of
// substeps, each frame written to output/frame_<n>.csv -- with the state kept on
// the GPU between steps (snow::gpu::set_resident) and the frames written by
// a background thread while the next frame steps (export_particles_async).
//
//   snow_frames GROUPS PARTICLES [--frames F] [--substeps S] [--dx DX] [--dt DT]
//               [--E E] [--nu NU] [--xi XI] [--theta-c TC] [--theta-s TS]
//               [--alpha A] [--gravity GY] [--plane-y Y] [--friction MU]
//               [--export none|sync|async] [--literal] [--stage-timings]
//
// Defaults are the reference main's constants (dx 0.05, dt 5e-4, 80 substeps,
// 50 frames, E 2.5e5, nu 0.2, xi 10, theta_c 0.015, theta_s 0.0075, alpha 0.95,
// gravity -10, ground plane y = 0 with friction 1).  --literal steps the
// reference way (upload, step, download every call); --stage-timings keeps the
// per-stage StepTimings of every resident step (each step then waits for the
// GPU).  Prints one JSON line: particle count, import / setup / loop / export
// milliseconds, per-frame milliseconds and particle-steps per second.
#include <chrono>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <filesystem>
#include <string>
#include <vector>

#include "snow/collision.hpp"
#include "snow/debug.hpp"
#include "snow/export.hpp"
#include "snow/grid.hpp"
#include "snow/import.hpp"

namespace
{
using clock_type = std::chrono::steady_clock;
double ms_since(clock_type::time_point t0)
{
    return std::chrono::duration<double, std::milli>(clock_type::now() - t0).count();
}

[[noreturn]] void usage(const char* msg)
{
    std::fprintf(stderr, "snow_frames: %s\n", msg);
    std::exit(2);
}
}  // namespace

int main(int argc, char** argv)
{
    if (argc < 3) usage("usage: snow_frames GROUPS PARTICLES [options]");
    const std::string groups = argv[1], seeds = argv[2];
    int frames = 50, substeps = 80;
    double dx = 0.05, dt = 0.0005, E = 2.5e5, nu = 0.2, xi = 10.0, theta_c = 0.015, theta_s = 0.0075;
    double alpha = 0.95, gy = -10.0, plane_y = 0.0, friction = 1.0;
    std::string export_mode = "async";
    bool literal = false, stage_timings = false;
    for (int i = 3; i < argc; ++i)
    {
        const std::string a = argv[i];
        auto next = [&]() -> const char* {
            if (i + 1 >= argc) usage(("missing value after " + a).c_str());
            return argv[++i];
        };
        if (a == "--frames") frames = std::atoi(next());
        else if (a == "--substeps") substeps = std::atoi(next());
        else if (a == "--dx") dx = std::atof(next());
        else if (a == "--dt") dt = std::atof(next());
        else if (a == "--E") E = std::atof(next());
        else if (a == "--nu") nu = std::atof(next());
        else if (a == "--xi") xi = std::atof(next());
        else if (a == "--theta-c") theta_c = std::atof(next());
        else if (a == "--theta-s") theta_s = std::atof(next());
        else if (a == "--alpha") alpha = std::atof(next());
        else if (a == "--gravity") gy = std::atof(next());
        else if (a == "--plane-y") plane_y = std::atof(next());
        else if (a == "--friction") friction = std::atof(next());
        else if (a == "--export") export_mode = next();
        else if (a == "--literal") literal = true;
        else if (a == "--stage-timings") stage_timings = true;
        else usage(("unknown option " + a).c_str());
    }
    if (export_mode != "none" && export_mode != "sync" && export_mode != "async") usage("--export none|sync|async");
    if (frames < 0 || substeps < 1) usage("bad frame or substep count");
    const double mu_0 = E / (2 * (1 + nu));
    const double lambda_0 = E * nu / ((1 + nu) * (1 - 2 * nu));

    auto t0 = clock_type::now();
    std::vector<Particle> particles{import_particles(groups, seeds)};
    const double import_ms = ms_since(t0);
    std::vector<CollisionBody> colliders{make_plane({0, plane_y, 0}, {0, 1, 0}, friction)};
    const Eigen::Vector3d gravity{0, gy, 0};
    std::vector<ParticleStencil> stencils(particles.size());
    if (export_mode != "none") std::filesystem::create_directories("output");

    snow::gpu::set_resident(!literal);
    snow::gpu::set_stage_timings(stage_timings);
    t0 = clock_type::now();
    setup(particles, dx);
    const double setup_ms = ms_since(t0);
    if (export_mode != "none") export_particles(particles, 0);

    std::vector<double> frame_ms;
    StepTimings timings;
    const auto loop0 = clock_type::now();
    for (int frame = 1; frame <= frames; ++frame)
    {
        const auto f0 = clock_type::now();
        for (int s = 0; s < substeps; ++s)
            step(particles, colliders, stencils, gravity, dt, dx, mu_0, lambda_0, xi, theta_c, theta_s, alpha,
                 timings);
        if (export_mode == "sync")
            export_particles(particles, frame);
        else if (export_mode == "async")
            snow::gpu::export_particles_async(particles, frame);
        frame_ms.push_back(ms_since(f0));
    }
    snow::gpu::sync_to_host(particles);  // the last frame's steps are done
    const double steps_ms = ms_since(loop0);
    const auto w0 = clock_type::now();
    snow::gpu::wait_exports();
    const double wait_ms = ms_since(w0);
    const double loop_ms = ms_since(loop0);

    std::printf("{\"particles\": %zu, \"frames\": %d, \"substeps\": %d, \"export\": \"%s\", \"resident\": %s, "
                "\"import_ms\": %.3f, \"setup_ms\": %.3f, \"loop_ms\": %.3f, \"steps_done_ms\": %.3f, "
                "\"export_wait_ms\": %.3f, \"particle_steps_per_s\": %.6e, \"frame_ms\": [",
                particles.size(), frames, substeps, export_mode.c_str(), literal ? "false" : "true", import_ms,
                setup_ms, loop_ms, steps_ms, wait_ms,
                loop_ms > 0 ? (double)particles.size() * frames * substeps / (loop_ms * 1e-3) : 0.0);
    for (std::size_t i = 0; i < frame_ms.size(); ++i) std::printf("%s%.3f", i ? ", " : "", frame_ms[i]);
    std::printf("]}\n");
    return 0;
}
