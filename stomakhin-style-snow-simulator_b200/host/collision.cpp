// make_plane (reference src/collision.cpp:5-27) with named functors, so that
// the GPU step can read the plane back out of the CollisionBody.
#include "snow/collision.hpp"

CollisionBody make_plane(const Eigen::Vector3d& point, const Eigen::Vector3d& normal, double friction)
{
    const Eigen::Vector3d unit_normal = normal.normalized();
    return CollisionBody{snow::PlaneDistance{point, unit_normal}, snow::PlaneNormal{unit_normal},
                         snow::ConstantVelocity{Eigen::Vector3d::Zero()}, friction};
}

namespace snow
{
CollisionBody make_moving_plane(const Eigen::Vector3d& point, const Eigen::Vector3d& normal,
                                const Eigen::Vector3d& velocity, double friction)
{
    const Eigen::Vector3d unit_normal = normal.normalized();
    return CollisionBody{PlaneDistance{point, unit_normal}, PlaneNormal{unit_normal}, ConstantVelocity{velocity},
                         friction};
}

CollisionBody make_sphere(const Eigen::Vector3d& center, double radius, double friction,
                          const Eigen::Vector3d& velocity)
{
    return CollisionBody{SphereDistance{center, radius}, SphereNormal{center}, ConstantVelocity{velocity}, friction};
}
}  // namespace snow
