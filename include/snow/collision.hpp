// Colliders (reference include/snow/collision.hpp).  CollisionBody keeps the
// reference's std::function members so that existing code compiles; bodies
// made by make_plane (and snow::make_moving_plane, snow::make_sphere) hold the
// named functors below, from which the GPU step recovers the body (any other
// callable is rejected with std::invalid_argument: a std::function cannot run
// on the device).
#pragma once

#include <functional>

#include <Eigen/Dense>

struct CollisionBody
{
    std::function<double(const Eigen::Vector3d&)> phi;
    std::function<Eigen::Vector3d(const Eigen::Vector3d&)> normal;
    std::function<Eigen::Vector3d(const Eigen::Vector3d&)> velocity;
    double friction;
};

namespace snow
{
// phi(x) = n . (x - p) of a plane through `point` with unit normal `unit_normal`.
struct PlaneDistance
{
    Eigen::Vector3d point;
    Eigen::Vector3d unit_normal;
    double operator()(const Eigen::Vector3d& x) const { return unit_normal.dot(x - point); }
};
struct PlaneNormal
{
    Eigen::Vector3d unit_normal;
    Eigen::Vector3d operator()(const Eigen::Vector3d&) const { return unit_normal; }
};
struct ConstantVelocity
{
    Eigen::Vector3d value;
    Eigen::Vector3d operator()(const Eigen::Vector3d&) const { return value; }
};
// phi(x) = |x - center| - radius of a solid sphere, and its outward normal.
struct SphereDistance
{
    Eigen::Vector3d center;
    double radius;
    double operator()(const Eigen::Vector3d& x) const { return (x - center).norm() - radius; }
};
struct SphereNormal
{
    Eigen::Vector3d center;
    Eigen::Vector3d operator()(const Eigen::Vector3d& x) const { return (x - center).normalized(); }
};

// Solid oriented box centred at `center` with orthonormal axes u, w, u x w and
// half extents h along them.  phi is the exact signed distance
// |max(q, 0)| + min(max_k q_k, 0) with q_k = |l_k| - h_k, l the point in the
// box's axes.  The normal inside the box (where collisions act) is the outward
// normal of the face with the largest q_k (the first on a tie, +1 side at
// l_k = 0); outside it is the gradient of phi.
struct BoxDistance
{
    Eigen::Vector3d center, u, w, half;
    double operator()(const Eigen::Vector3d& x) const;
};
struct BoxNormal
{
    Eigen::Vector3d center, u, w, half;
    Eigen::Vector3d operator()(const Eigen::Vector3d& x) const;
};

// Not in the reference (which takes any CollisionBody): bodies the GPU step
// can run besides make_plane -- a plane moving with a constant velocity, a
// solid sphere and a solid oriented box, resting or moving.
CollisionBody make_moving_plane(const Eigen::Vector3d& point, const Eigen::Vector3d& normal,
                                const Eigen::Vector3d& velocity, double friction);
CollisionBody make_sphere(const Eigen::Vector3d& center, double radius, double friction,
                          const Eigen::Vector3d& velocity = Eigen::Vector3d::Zero());
// `axis_u` and `axis_w` are normalised and w is made orthogonal to u
// (Gram-Schmidt); they must not be parallel.
CollisionBody make_box(const Eigen::Vector3d& center, const Eigen::Vector3d& half_extents,
                       const Eigen::Vector3d& axis_u, const Eigen::Vector3d& axis_w, double friction,
                       const Eigen::Vector3d& velocity = Eigen::Vector3d::Zero());
}  // namespace snow

CollisionBody make_plane(const Eigen::Vector3d& point, const Eigen::Vector3d& normal, double friction);
