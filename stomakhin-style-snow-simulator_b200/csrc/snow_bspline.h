// Cubic B-spline of the reference solver (src/grid.cpp:15-58), shared by the
// CUDA kernels and the host side of the C++ API (build_stencil, N, N_dash).
#pragma once

#include <cmath>

#ifdef __CUDACC__
#define SNOW_HD __host__ __device__ __forceinline__
#else
#define SNOW_HD inline
#endif

namespace snow {

template <typename T>
SNOW_HD T sgn(T x) {  // signum (grid.cpp:15-20)
  return x > T(0) ? T(1) : (x < T(0) ? T(-1) : T(0));
}

// N(a, b): cubic B-spline of |a - b| (grid.cpp:24-40).
template <typename T>
SNOW_HD T bspline(T a, T b) {
  using std::fabs;
  const T d = fabs(a - b);
  if (d >= T(0) && d < T(1)) return T(0.5) * d * d * d - d * d + T(2.0 / 3.0);
  if (d >= T(1) && d < T(2)) return T(-1.0 / 6.0) * d * d * d + d * d - T(2) * d + T(4.0 / 3.0);
  return T(0);
}

// N_dash(node, x) = dN/dx (grid.cpp:42-58).
template <typename T>
SNOW_HD T bspline_slope(T node, T x) {
  using std::fabs;
  const T d = fabs(node - x);
  if (d >= T(0) && d < T(1)) return (T(1.5) * d * d - T(2) * d) * sgn(x - node);
  if (d >= T(1) && d < T(2)) return (T(-1.0 / 2.0) * d * d + T(2) * d - T(2)) * sgn(x - node);
  return T(0);
}

// Lower stencil corner base = floor(x / dx) - 1 (grid.cpp:64-67).
template <typename T>
SNOW_HD int stencil_base(T gp) {
  using std::floor;
  return static_cast<int>(floor(gp)) - 1;
}

}  // namespace snow
