// GPU residency for the drop-in step(): one batch holding the particle vector
// last stepped, keyed by its data pointer and size.
#include <cstring>
#include <mutex>
#include <stdexcept>
#include <string>

#include "snow_host_detail.hpp"

namespace snow::host
{
void check(int rc)
{
    if (rc != SNOW_OK) throw std::runtime_error(std::string("snow GPU: ") + snow_gpu_last_error());
}

namespace
{
struct Resident
{
    std::mutex mu;
    bool on = false;
    snow_gpu_batch* batch = nullptr;
    int32_t scene = -1;
    const Particle* data = nullptr;
    std::size_t size = 0;
    bool host_stale = false;  // the vector lags the GPU copy
    bool stage_timings = true;
    // the parameters and colliders the batch holds (set_params only when they
    // change: it makes the next step recompute every particle's force matrix)
    snow_step_params params{};
    std::vector<snow_collider> colliders;

    void drop()
    {
        if (batch) snow_gpu_batch_destroy(batch);
        batch = nullptr;
        scene = -1;
        data = nullptr;
        size = 0;
        host_stale = false;
    }
    ~Resident() { drop(); }
};
Resident& state()
{
    static Resident r;
    return r;
}
}  // namespace
}  // namespace snow::host

using snow::host::check;
using snow::host::state;

namespace snow::gpu
{
void set_resident(bool on)
{
    auto& r = state();
    std::lock_guard<std::mutex> lk(r.mu);
    r.on = on;
    if (!on) r.drop();
}
void set_stage_timings(bool on)
{
    auto& r = state();
    std::lock_guard<std::mutex> lk(r.mu);
    r.stage_timings = on;
}
bool resident()
{
    auto& r = state();
    std::lock_guard<std::mutex> lk(r.mu);
    return r.on;
}
void invalidate()
{
    auto& r = state();
    std::lock_guard<std::mutex> lk(r.mu);
    r.drop();
}
void sync_to_host(std::vector<Particle>& snow)
{
    auto& r = state();
    std::lock_guard<std::mutex> lk(r.mu);
    if (!r.batch || r.data != snow.data() || r.size != snow.size()) return;
    check(snow_gpu_batch_download(r.batch, r.scene, reinterpret_cast<double*>(snow.data()),
                                  static_cast<int64_t>(snow.size()), nullptr));
    r.host_stale = false;
}
}  // namespace snow::gpu

void snow_host_invalidate_resident() { snow::gpu::invalidate(); }

void snow_host_resident_step(std::vector<Particle>& snow, const snow_step_params& p,
                             const std::vector<snow_collider>& colliders, snow_step_timings& t)
{
    auto& r = state();
    std::lock_guard<std::mutex> lk(r.mu);
    const int64_t n = static_cast<int64_t>(snow.size());
    const bool same_params =
        std::memcmp(&r.params, &p, sizeof p) == 0 && r.colliders.size() == colliders.size() &&
        (colliders.empty() ||
         std::memcmp(r.colliders.data(), colliders.data(), colliders.size() * sizeof(snow_collider)) == 0);
    if (!r.batch || r.data != snow.data() || r.size != snow.size())
    {
        r.drop();
        check(snow_gpu_batch_create(&r.batch, SNOW_FP64));
        check(snow_gpu_batch_add_scene(r.batch, reinterpret_cast<const double*>(snow.data()), n, &p,
                                       colliders.data(), static_cast<int>(colliders.size()), &r.scene, nullptr));
        r.data = snow.data();
        r.size = snow.size();
    }
    else if (!same_params)
    {
        check(snow_gpu_batch_set_params(r.batch, r.scene, &p, colliders.data(),
                                        static_cast<int>(colliders.size())));
    }
    r.params = p;
    r.colliders = colliders;
    // With stage timings the step is launched kernel by kernel between events
    // and waited for; without, it is the batch's captured step graph, left
    // running on the GPU (the next read-back waits for it).
    check(snow_gpu_batch_step(r.batch, 1, r.stage_timings ? &t : nullptr, nullptr));
    r.host_stale = true;
}

bool snow_host_resident_positions(const std::vector<Particle>& snow, double* xyz)
{
    auto& r = state();
    std::lock_guard<std::mutex> lk(r.mu);
    if (!r.batch || r.data != snow.data() || r.size != snow.size() || !r.host_stale) return false;
    check(snow_gpu_batch_download_positions(r.batch, r.scene, xyz, static_cast<int64_t>(snow.size()), nullptr));
    return true;
}

bool snow_host_resident_copy(const std::vector<Particle>& snow, double* out)
{
    auto& r = state();
    std::lock_guard<std::mutex> lk(r.mu);
    if (!r.batch || r.data != snow.data() || r.size != snow.size() || !r.host_stale) return false;
    check(snow_gpu_batch_download(r.batch, r.scene, out, static_cast<int64_t>(snow.size()), nullptr));
    return true;
}
