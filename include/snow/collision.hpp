// Colliders (reference include/snow/collision.hpp).  CollisionBody keeps the
// reference's std::function members so that existing code compiles; bodies
// made by make_plane hold the named functors below, from which the GPU step
// recovers the plane (any other callable is rejected with
// std::invalid_argument: a std::function cannot run on the device).
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
}  // namespace snow

CollisionBody make_plane(const Eigen::Vector3d& point, const Eigen::Vector3d& normal, double friction);
