// make_plane (reference src/collision.cpp:5-27) with named functors, so that
// the GPU step can read the plane back out of the CollisionBody.
#include "snow/collision.hpp"

#include <cmath>
#include <stdexcept>

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

namespace
{
// The point in the box's axes and the third axis u x w.
Eigen::Vector3d box_local(const Eigen::Vector3d& center, const Eigen::Vector3d& u, const Eigen::Vector3d& w,
                          const Eigen::Vector3d& x, Eigen::Vector3d& t)
{
    t = Eigen::Vector3d(u[1] * w[2] - u[2] * w[1], u[2] * w[0] - u[0] * w[2], u[0] * w[1] - u[1] * w[0]);
    const Eigen::Vector3d d = x - center;
    return Eigen::Vector3d(u.dot(d), w.dot(d), t.dot(d));
}
}  // namespace

double BoxDistance::operator()(const Eigen::Vector3d& x) const
{
    Eigen::Vector3d t;
    const Eigen::Vector3d l = box_local(center, u, w, x, t);
    double out2 = 0.0, qmax = -INFINITY;
    for (int k = 0; k < 3; ++k)
    {
        const double q = std::abs(l[k]) - half[k];
        qmax = std::max(qmax, q);
        if (q > 0.0) out2 += q * q;
    }
    return std::sqrt(out2) + std::min(qmax, 0.0);
}

Eigen::Vector3d BoxNormal::operator()(const Eigen::Vector3d& x) const
{
    Eigen::Vector3d t;
    const Eigen::Vector3d l = box_local(center, u, w, x, t);
    const Eigen::Vector3d axes[3] = {u, w, t};
    int k = 0;
    double qmax = std::abs(l[0]) - half[0];
    for (int a = 1; a < 3; ++a)
    {
        const double q = std::abs(l[a]) - half[a];
        if (q > qmax)
        {
            qmax = q;
            k = a;
        }
    }
    if (qmax <= 0.0) return (l[k] < 0.0 ? -1.0 : 1.0) * axes[k];
    Eigen::Vector3d g = Eigen::Vector3d::Zero();
    for (int a = 0; a < 3; ++a)
    {
        const double q = std::abs(l[a]) - half[a];
        if (q > 0.0) g = g + ((l[a] < 0.0 ? -q : q) * axes[a]);
    }
    return g.normalized();
}

CollisionBody make_box(const Eigen::Vector3d& center, const Eigen::Vector3d& half_extents,
                       const Eigen::Vector3d& axis_u, const Eigen::Vector3d& axis_w, double friction,
                       const Eigen::Vector3d& velocity)
{
    const Eigen::Vector3d u = axis_u.normalized();
    const Eigen::Vector3d w0 = axis_w - u.dot(axis_w) * u;
    if (!(w0.norm() > 1e-12 * axis_w.norm())) throw std::invalid_argument("make_box: the two axes are parallel");
    const Eigen::Vector3d w = w0.normalized();
    return CollisionBody{BoxDistance{center, u, w, half_extents}, BoxNormal{center, u, w, half_extents},
                         ConstantVelocity{velocity}, friction};
}
}  // namespace snow
