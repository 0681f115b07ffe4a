// Per-particle and per-node arithmetic of the explicit MPM snow step, shared by
// the fused kernels and the single-stage entry points (host + device).
//
// Formulas follow the reference solver src/grid.cpp line by line; where the GPU
// form differs algebraically (never numerically beyond round-off) the comment
// says how and why.
#pragma once

#include <cstdint>
#include <cmath>

#include "snow_bspline.h"

namespace snow {

// Weights and weight slopes of the 4 stencil nodes along one axis.
// slope[i] = N_dash / dx, as build_stencil stores it (grid.cpp:80).
template <typename T>
struct AxisWeights {
  T w[4];
  T dw[4];
  int base;
};
// The grid position x / dx is a true division, as in the reference, so the
// stencil base is the reference's exactly; the slopes are scaled by 1 / dx
// (one rounding away from the reference's N_dash / dx).
//
// With f = gp - floor(gp) the four nodes sit at distances 1 + f, f, 1 - f and
// 2 - f from gp, each inside one fixed piece of N and N_dash (grid.cpp:24-58),
// so the weights and slopes are those pieces written as polynomials in f and
// g = 1 - f, without the per-node branches:
//   w  = (g^3/6,  f^3/2 - f^2 + 2/3,  g^3/2 - g^2 + 2/3,  f^3/6)
//   dw = (-g^2/2, 3f^2/2 - 2f,       -(3g^2/2 - 2g),      f^2/2)
// (equal to bspline / bspline_slope up to rounding).
template <typename T>
SNOW_HD AxisWeights<T> axis_weights(T x, T dx) {
  using std::floor;
  AxisWeights<T> a;
  const T gp = x / dx;
  const T inv_dx = T(1) / dx;
  const T fl = floor(gp);
  a.base = static_cast<int>(fl) - 1;  // stencil_base(gp)
  const T f = gp - fl, g = T(1) - f;
  const T f2 = f * f, g2 = g * g;
  a.w[0] = g2 * g * T(1.0 / 6.0);
  a.w[1] = (T(0.5) * f - T(1)) * f2 + T(2.0 / 3.0);
  a.w[2] = (T(0.5) * g - T(1)) * g2 + T(2.0 / 3.0);
  a.w[3] = f2 * f * T(1.0 / 6.0);
  a.dw[0] = -T(0.5) * g2 * inv_dx;
  a.dw[1] = (T(1.5) * f - T(2)) * f * inv_dx;
  a.dw[2] = -(T(1.5) * g - T(2)) * g * inv_dx;
  a.dw[3] = T(0.5) * f2 * inv_dx;
  return a;
}

// ----------------------------------------------------------------- 3x3 algebra
// Matrices are column-major, m[c * 3 + r], like the reference's Eigen::Matrix3d.
template <typename T>
struct M3 {
  T a[9];
  SNOW_HD T& operator()(int r, int c) { return a[c * 3 + r]; }
  SNOW_HD T operator()(int r, int c) const { return a[c * 3 + r]; }
};

template <typename T>
SNOW_HD M3<T> mat_mul(const M3<T>& x, const M3<T>& y) {
  M3<T> m;
#pragma unroll
  for (int c = 0; c < 3; ++c)
#pragma unroll
    for (int r = 0; r < 3; ++r) m(r, c) = x(r, 0) * y(0, c) + x(r, 1) * y(1, c) + x(r, 2) * y(2, c);
  return m;
}

// Cofactor expansion along the first row.
template <typename T>
SNOW_HD T det3(const M3<T>& m) {
  return m(0, 0) * (m(1, 1) * m(2, 2) - m(1, 2) * m(2, 1)) -
         m(0, 1) * (m(1, 0) * m(2, 2) - m(1, 2) * m(2, 0)) +
         m(0, 2) * (m(1, 0) * m(2, 1) - m(1, 1) * m(2, 0));
}

// Symmetric 3x3 as six scalars.
template <typename T>
struct Sym3 {
  T xx, yy, zz, xy, xz, yz;
};

// F <- D F for a symmetric D, column by column in place (the same sums as
// mat_mul with D written out, with a third of the live registers).
template <typename T>
SNOW_HD void sym_mul_inplace(const Sym3<T>& D, M3<double>& F) {
  const double xx = D.xx, yy = D.yy, zz = D.zz, xy = D.xy, xz = D.xz, yz = D.yz;
#pragma unroll
  for (int c = 0; c < 3; ++c) {
    const double a = F(0, c), b = F(1, c), d = F(2, c);
    F(0, c) = xx * a + xy * b + xz * d;
    F(1, c) = xy * a + yy * b + yz * d;
    F(2, c) = xz * a + yz * b + zz * d;
  }
}

// Eigen-decomposition S = Q diag(lam) Q^T of a symmetric 3x3 by cyclic Jacobi
// rotations (Golub & Van Loan, Matrix Computations, 4th ed., Alg. 8.5.2 with
// the stable rotation of Alg. 8.5.1).  Converges quadratically; the sweep loop
// stops when the off-diagonal mass falls below tol^2 of the diagonal mass.
// The rotation's tangent t = sgn(theta) / (|theta| + sqrt(theta^2 + 1)) with
// theta = (a_qq - a_pp) / (2 a_pq) is evaluated as
// t = sgn(a) b / (|a| + sqrt(a^2 + b^2)), a = a_qq - a_pp, b = 2 a_pq
// (numerator and denominator multiplied by |b|): one division, one square
// root, and cos = rsqrt(1 + t^2).
//
// 1 / sqrt(x) for x in [1, 2] (the rotation's 1 + t^2, |t| <= 1): in double on
// the device, a float seed refined by two Newton-Raphson steps for the
// reciprocal square root, y <- y (3 - x y^2) / 2, each of which squares the
// relative error (seed 2^-22 -> 2^-44 -> below the double rounding).
template <typename T>
SNOW_HD T rsqrt_unit(T x) {
#ifdef __CUDA_ARCH__
  if constexpr (sizeof(T) == 8) {
    T y = (T)rsqrtf((float)x);
    y = y * (T(1.5) - T(0.5) * x * y * y);
    y = y * (T(1.5) - T(0.5) * x * y * y);
    return y;
  } else {
    return rsqrt(x);
  }
#else
  return T(1) / std::sqrt(x);
#endif
}

template <typename T>
SNOW_HD void rotate_pq(T& app, T& aqq, T& apq, T& arp, T& arq, T q[9], int p, int qq) {
  if (apq == T(0)) return;
  const T a = aqq - app, b = T(2) * apq;
  const T t = (a >= T(0) ? b : -b) / (fabs(a) + sqrt(a * a + b * b));
  const T c = rsqrt_unit(t * t + T(1));
  const T s = t * c;
  app -= t * apq;
  aqq += t * apq;
  apq = T(0);
  const T rp = arp, rq = arq;
  arp = c * rp - s * rq;
  arq = s * rp + c * rq;
#pragma unroll
  for (int k = 0; k < 3; ++k) {
    const T vp = q[p * 3 + k], vq = q[qq * 3 + k];
    q[p * 3 + k] = c * vp - s * vq;
    q[qq * 3 + k] = s * vp + c * vq;
  }
}

template <typename T>
SNOW_HD void sym_eig3(Sym3<T> s, T lam[3], T q[9], T tol, int max_sweeps) {
#pragma unroll
  for (int i = 0; i < 9; ++i) q[i] = T(i % 4 == 0 ? 1 : 0);
  for (int sweep = 0; sweep < max_sweeps; ++sweep) {
    const T off = s.xy * s.xy + s.xz * s.xz + s.yz * s.yz;
    const T dia = s.xx * s.xx + s.yy * s.yy + s.zz * s.zz;
    if (!(off > tol * tol * dia)) break;
    rotate_pq(s.xx, s.yy, s.xy, s.xz, s.yz, q, 0, 1);  // (p,q)=(0,1), r=2
    rotate_pq(s.xx, s.zz, s.xz, s.xy, s.yz, q, 0, 2);  // (0,2), r=1
    rotate_pq(s.yy, s.zz, s.yz, s.xy, s.xz, q, 1, 2);  // (1,2), r=0
  }
  lam[0] = s.xx;
  lam[1] = s.yy;
  lam[2] = s.zz;
}

template <typename T>
struct EigTol;
template <>
struct EigTol<double> {
  static constexpr double tol = 1e-17;
  static constexpr int sweeps = 12;
};
template <>
struct EigTol<float> {
  static constexpr float tol = 1e-8f;
  static constexpr int sweeps = 8;
};

// Q diag(f) Q^T.
template <typename T>
SNOW_HD Sym3<T> spectral(const T q[9], const T f[3]) {
  Sym3<T> r;
  r.xx = q[0] * q[0] * f[0] + q[3] * q[3] * f[1] + q[6] * q[6] * f[2];
  r.yy = q[1] * q[1] * f[0] + q[4] * q[4] * f[1] + q[7] * q[7] * f[2];
  r.zz = q[2] * q[2] * f[0] + q[5] * q[5] * f[1] + q[8] * q[8] * f[2];
  r.xy = q[0] * q[1] * f[0] + q[3] * q[4] * f[1] + q[6] * q[7] * f[2];
  r.xz = q[0] * q[2] * f[0] + q[3] * q[5] * f[1] + q[6] * q[8] * f[2];
  r.yz = q[1] * q[2] * f[0] + q[4] * q[5] * f[1] + q[7] * q[8] * f[2];
  return r;
}

// --------------------------------------------------------- constitutive model
// F F^T and F^T F.
template <typename T>
SNOW_HD Sym3<T> gram_rows(const M3<T>& F) {
  Sym3<T> B;
  B.xx = F(0, 0) * F(0, 0) + F(0, 1) * F(0, 1) + F(0, 2) * F(0, 2);
  B.yy = F(1, 0) * F(1, 0) + F(1, 1) * F(1, 1) + F(1, 2) * F(1, 2);
  B.zz = F(2, 0) * F(2, 0) + F(2, 1) * F(2, 1) + F(2, 2) * F(2, 2);
  B.xy = F(0, 0) * F(1, 0) + F(0, 1) * F(1, 1) + F(0, 2) * F(1, 2);
  B.xz = F(0, 0) * F(2, 0) + F(0, 1) * F(2, 1) + F(0, 2) * F(2, 2);
  B.yz = F(1, 0) * F(2, 0) + F(1, 1) * F(2, 1) + F(1, 2) * F(2, 2);
  return B;
}
template <typename T>
SNOW_HD Sym3<T> gram_cols(const M3<T>& F) {
  Sym3<T> C;
  C.xx = F(0, 0) * F(0, 0) + F(1, 0) * F(1, 0) + F(2, 0) * F(2, 0);
  C.yy = F(0, 1) * F(0, 1) + F(1, 1) * F(1, 1) + F(2, 1) * F(2, 1);
  C.zz = F(0, 2) * F(0, 2) + F(1, 2) * F(1, 2) + F(2, 2) * F(2, 2);
  C.xy = F(0, 0) * F(0, 1) + F(1, 0) * F(1, 1) + F(2, 0) * F(2, 1);
  C.xz = F(0, 0) * F(0, 2) + F(1, 0) * F(1, 2) + F(2, 0) * F(2, 2);
  C.yz = F(0, 1) * F(0, 2) + F(1, 1) * F(1, 2) + F(2, 1) * F(2, 2);
  return C;
}
// G S G^T for symmetric S.
template <typename T>
SNOW_HD Sym3<T> sandwich(const M3<T>& G, const Sym3<T>& S) {
  T H[9];  // H = G S, column-major
#pragma unroll
  for (int r = 0; r < 3; ++r) {
    H[r] = G(r, 0) * S.xx + G(r, 1) * S.xy + G(r, 2) * S.xz;
    H[3 + r] = G(r, 0) * S.xy + G(r, 1) * S.yy + G(r, 2) * S.yz;
    H[6 + r] = G(r, 0) * S.xz + G(r, 1) * S.yz + G(r, 2) * S.zz;
  }
  Sym3<T> o;  // (H G^T)(r,c) = sum_k H(r,k) G(c,k)
  o.xx = H[0] * G(0, 0) + H[3] * G(0, 1) + H[6] * G(0, 2);
  o.yy = H[1] * G(1, 0) + H[4] * G(1, 1) + H[7] * G(1, 2);
  o.zz = H[2] * G(2, 0) + H[5] * G(2, 1) + H[8] * G(2, 2);
  o.xy = H[0] * G(1, 0) + H[3] * G(1, 1) + H[6] * G(1, 2);
  o.xz = H[0] * G(2, 0) + H[3] * G(2, 1) + H[6] * G(2, 2);
  o.yz = H[1] * G(2, 0) + H[4] * G(2, 1) + H[7] * G(2, 2);
  return o;
}

// Force matrix of one particle, M = -V_p0 * P(F_E) * F_E^T (grid.cpp:174-176)
// with the fixed-corotated stress P = 2 mu (F_E - R_E) + lambda (J-1) J F_E^-T
// and exponential hardening mu = mu0 h, lambda = lambda0 h, h = exp(xi (1 - det F_P))
// (grid.cpp:162-172).
//
// GPU form: P F^T = 2 mu (F F^T - R F^T) + lambda (J-1) J I, and R F^T = U S U^T
// = sqrt(F F^T) for every SVD F = U S V^T with S >= 0 (R = U V^T, the reference's
// polar factor from JacobiSVD).  So M needs B = F F^T, its symmetric square root
// and J; no inverse; M is symmetric.  `hardening` is exp(xi (1 - det F_P))
// evaluated by the caller in double.
template <typename T>
SNOW_HD Sym3<T> assemble_force(const Sym3<T>& B, const Sym3<T>& R, T J, T V0, T mu0, T lambda0,
                               T hardening) {
  const T mu = mu0 * hardening;
  const T lambda = lambda0 * hardening;
  const T two_mu = T(2) * mu;
  const T vol = lambda * (J - T(1)) * J;
  Sym3<T> M;
  M.xx = -V0 * (two_mu * (B.xx - R.xx) + vol);
  M.yy = -V0 * (two_mu * (B.yy - R.yy) + vol);
  M.zz = -V0 * (two_mu * (B.zz - R.zz) + vol);
  M.xy = -V0 * (two_mu * (B.xy - R.xy));
  M.xz = -V0 * (two_mu * (B.xz - R.xz));
  M.yz = -V0 * (two_mu * (B.yz - R.yz));
  return M;
}

// The same from F alone: sqrt(F F^T) by one symmetric Jacobi eigensolve.
template <typename T>
SNOW_HD Sym3<T> force_matrix(const M3<T>& F, T V0, T mu0, T lambda0, T hardening) {
  const Sym3<T> B = gram_rows(F);
  T lam[3], q[9];
  sym_eig3(B, lam, q, EigTol<T>::tol, EigTol<T>::sweeps);
  T sv[3];
#pragma unroll
  for (int i = 0; i < 3; ++i) sv[i] = sqrt(lam[i] > T(0) ? lam[i] : T(0));
  return assemble_force(B, spectral(q, sv), det3(F), V0, mu0, lambda0, hardening);
}

// Elastoplastic update (grid.cpp:277-285): trial F_E* = (I + dt grad v) F_E,
// SVD F_E* = U S V^T, S clamped to [1 - theta_c, 1 + theta_s],
// F_E <- U S_c V^T,  F_P <- F_E^-1 F_E* F_P.
//
// GPU form: with C = F_E*^T F_E* = V S^2 V^T (symmetric Jacobi eigensolve) and
// D = V diag(s_c / s) V^T,  U S_c V^T = F_E* D  and  F_E^-1 F_E* = V diag(s / s_c) V^T
// = D^-1, so F_E <- F_E* D and F_P <- D^-1 F_P: no U, no inverse.  Where no
// singular value is clamped D = I and F_E* passes through unchanged.
//
// The same eigenvectors give the square root the next step's force needs:
// sqrt(F_E F_E^T) = U S_c U^T = F_E* V diag(s_c / s^2) V^T F_E*^T (returned in
// `root`; `regular` is false when a singular value is too small for it).
template <typename T>
struct Plastic {
  Sym3<T> Dinv;
  Sym3<T> root;
  T sigma[3];  // singular values of the trial F_E
  bool clamped;
  bool regular;
};

template <typename T>
SNOW_HD Plastic<T> plastic_projection(M3<T>& FE, T lo, T hi) {
  Plastic<T> out;
  T lam[3], q[9];
  sym_eig3(gram_cols(FE), lam, q, EigTol<T>::tol, EigTol<T>::sweeps);
  T r[3], ri[3], e[3];
  out.clamped = false;
  out.regular = true;
#pragma unroll
  for (int i = 0; i < 3; ++i) {
    const T s = sqrt(lam[i] > T(0) ? lam[i] : T(0));
    out.sigma[i] = s;
    const T sc = s < lo ? lo : (s > hi ? hi : s);  // std::clamp (grid.cpp:281-283)
    if (sc != s) out.clamped = true;
    if (!(s > T(1e-6))) out.regular = false;
    // r = sc / s, ri = s / sc, e = sc / s^2 with one division where no clamp acts
    r[i] = ri[i] = T(1);
    e[i] = T(0);
    if (s > T(0)) {
      const T inv = T(1) / s;
      e[i] = inv;
      if (sc != s) {
        r[i] = sc * inv;
        ri[i] = s / sc;
        e[i] = r[i] * inv;
      }
    }
  }
  out.root = sandwich(FE, spectral(q, e));
  if (!out.clamped) {
    out.Dinv = Sym3<T>{T(1), T(1), T(1), T(0), T(0), T(0)};
    return out;
  }
  const Sym3<T> D = spectral(q, r);
  out.Dinv = spectral(q, ri);
  M3<T> o;
#pragma unroll
  for (int rr = 0; rr < 3; ++rr) {
    const T f0 = FE(rr, 0), f1 = FE(rr, 1), f2 = FE(rr, 2);
    o(rr, 0) = f0 * D.xx + f1 * D.xy + f2 * D.xz;
    o(rr, 1) = f0 * D.xy + f1 * D.yy + f2 * D.yz;
    o(rr, 2) = f0 * D.xz + f1 * D.yz + f2 * D.zz;
  }
  FE = o;
  return out;
}

// ------------------------------------------------------ elastic fast path
// Most particles are not clamped in a step; for them the projection is the
// identity and only sqrt(F F^T) is needed, which the polar factor gives
// without an eigensolve: F = R S (R orthogonal, S symmetric positive
// definite), sqrt(F F^T) = R S R^T = F R^T, and the singular values of F are
// the eigenvalues of S.
//
// polar_newton: Newton's iteration X <- (X + X^-T) / 2 from X = F (Higham,
// "Computing the polar decomposition -- with applications", SIAM J. Sci.
// Stat. Comput. 7 (1986) 1160-1174).  It keeps the singular vectors and maps
// each singular value s to (s + 1/s) / 2, so the error e = s - 1 becomes
// e^2 / (2 (1 + e)): from |e| <= 0.1, 4 iterations fall below double rounding
// (0.1 -> 4.5e-3 -> 1e-5 -> 5e-11 -> 1e-21) and 3 below float rounding.  The
// iteration is accepted when the last one moved X by at most last_step (so
// the error left is below last_step^2 / 2) and det X stayed positive; else the
// caller takes the general path.  X^-T = cof(X) / det X (cofactor matrix).
template <typename T>
struct PolarTol;
template <>
struct PolarTol<double> {
  static constexpr int iters = 4;
  static constexpr double last_step = 1e-8;
};
template <>
struct PolarTol<float> {
  static constexpr int iters = 3;
  static constexpr float last_step = 3e-4f;
};

template <typename T>
SNOW_HD bool polar_newton(const M3<T>& F, M3<T>& X) {
  X = F;
  T moved = T(0);
#pragma unroll
  for (int it = 0; it < PolarTol<T>::iters; ++it) {
    M3<T> C;  // cofactors: C(r, c) = (-1)^(r+c) minor(r, c)
    C(0, 0) = X(1, 1) * X(2, 2) - X(1, 2) * X(2, 1);
    C(0, 1) = X(1, 2) * X(2, 0) - X(1, 0) * X(2, 2);
    C(0, 2) = X(1, 0) * X(2, 1) - X(1, 1) * X(2, 0);
    C(1, 0) = X(0, 2) * X(2, 1) - X(0, 1) * X(2, 2);
    C(1, 1) = X(0, 0) * X(2, 2) - X(0, 2) * X(2, 0);
    C(1, 2) = X(0, 1) * X(2, 0) - X(0, 0) * X(2, 1);
    C(2, 0) = X(0, 1) * X(1, 2) - X(0, 2) * X(1, 1);
    C(2, 1) = X(0, 2) * X(1, 0) - X(0, 0) * X(1, 2);
    C(2, 2) = X(0, 0) * X(1, 1) - X(0, 1) * X(1, 0);
    const T det = X(0, 0) * C(0, 0) + X(0, 1) * C(0, 1) + X(0, 2) * C(0, 2);
    if (!(det > T(0))) return false;
    const T h = T(0.5) / det;
    moved = T(0);
#pragma unroll
    for (int e = 0; e < 9; ++e) {
      const T x = T(0.5) * X.a[e] + h * C.a[e];
      moved = fmax(moved, fabs(x - X.a[e]));
      X.a[e] = x;
    }
  }
  return moved <= PolarTol<T>::last_step;
}

// Positive definiteness of a symmetric 3x3 by its leading principal minors.
template <typename T>
SNOW_HD bool positive_definite(const Sym3<T>& A) {
  if (!(A.xx > T(0))) return false;
  if (!(A.xx * A.yy - A.xy * A.xy > T(0))) return false;
  const T det = A.xx * (A.yy * A.zz - A.yz * A.yz) - A.xy * (A.xy * A.zz - A.yz * A.xz) +
                A.xz * (A.xy * A.yz - A.yy * A.xz);
  return det > T(0);
}

// The projection of a particle whose singular values all lie in
// [lo + margin, hi - margin]: S - (lo + margin) I and (hi - margin) I - S are
// positive definite.  Then no clamp acts (F_E stays, D = I) and the root is
// F R^T; returns true with `out` filled in.  Returns false (out untouched)
// when the iteration did not settle or a singular value may lie outside, or
// within `margin` of a bound: the general path (plastic_projection) decides
// those, so every clamp decision near a bound is the eigensolve's, as before.
// margin: 1e-12 in double (rounding of S is ~1e-16), the mixed form's
// near-critical distance in float.
template <typename T>
SNOW_HD bool elastic_projection(const M3<T>& F, T lo, T hi, T margin, Plastic<T>& out) {
  M3<T> R;
  if (!polar_newton(F, R)) return false;
  Sym3<T> S;  // R^T F
  S.xx = R(0, 0) * F(0, 0) + R(1, 0) * F(1, 0) + R(2, 0) * F(2, 0);
  S.yy = R(0, 1) * F(0, 1) + R(1, 1) * F(1, 1) + R(2, 1) * F(2, 1);
  S.zz = R(0, 2) * F(0, 2) + R(1, 2) * F(1, 2) + R(2, 2) * F(2, 2);
  S.xy = R(0, 0) * F(0, 1) + R(1, 0) * F(1, 1) + R(2, 0) * F(2, 1);
  S.xz = R(0, 0) * F(0, 2) + R(1, 0) * F(1, 2) + R(2, 0) * F(2, 2);
  S.yz = R(0, 1) * F(0, 2) + R(1, 1) * F(1, 2) + R(2, 1) * F(2, 2);
  const T a = lo + margin, b = hi - margin;
  if (!positive_definite(Sym3<T>{S.xx - a, S.yy - a, S.zz - a, S.xy, S.xz, S.yz})) return false;
  if (!positive_definite(Sym3<T>{b - S.xx, b - S.yy, b - S.zz, -S.xy, -S.xz, -S.yz})) return false;
  out.root.xx = F(0, 0) * R(0, 0) + F(0, 1) * R(0, 1) + F(0, 2) * R(0, 2);  // (F R^T)(r, c) = sum_k F(r,k) R(c,k)
  out.root.yy = F(1, 0) * R(1, 0) + F(1, 1) * R(1, 1) + F(1, 2) * R(1, 2);
  out.root.zz = F(2, 0) * R(2, 0) + F(2, 1) * R(2, 1) + F(2, 2) * R(2, 2);
  out.root.xy = F(0, 0) * R(1, 0) + F(0, 1) * R(1, 1) + F(0, 2) * R(1, 2);
  out.root.xz = F(0, 0) * R(2, 0) + F(0, 1) * R(2, 1) + F(0, 2) * R(2, 2);
  out.root.yz = F(1, 0) * R(2, 0) + F(1, 1) * R(2, 1) + F(1, 2) * R(2, 2);
  out.Dinv = Sym3<T>{T(1), T(1), T(1), T(0), T(0), T(0)};
  out.sigma[0] = out.sigma[1] = out.sigma[2] = T(1);  // inside [lo, hi]; not used on this path
  out.clamped = false;
  out.regular = true;
  return true;
}

// ------------------------------------------------- implicit update algebra
// Differential of the fixed-corotated first Piola-Kirchhoff stress
// P = 2 mu (F - R) + lambda (J - 1) J F^-T at F (Stomakhin et al. 2013, the
// implicit update's A_p), given the polar factors F = R S:
//   dP = 2 mu (dF - dR) + lambda (C : dF) C + lambda (J - 1) dC,
// C = J F^-T = cof(F), dC its differential, and dR = R [w]_x with
// (tr(S) I - S) w = axial(R^T dF - dF^T R) (R^T dR is skew and
// R^T dR S + S R^T dR equals the skew right-hand side).
template <typename T>
SNOW_HD M3<T> cofactor3(const M3<T>& F) {
  M3<T> C;
#pragma unroll
  for (int r = 0; r < 3; ++r)
#pragma unroll
    for (int c = 0; c < 3; ++c) {
      const int r1 = (r + 1) % 3, r2 = (r + 2) % 3, c1 = (c + 1) % 3, c2 = (c + 2) % 3;
      C(r, c) = F(r1, c1) * F(r2, c2) - F(r1, c2) * F(r2, c1);
    }
  return C;
}

template <typename T>
SNOW_HD M3<T> corotated_differential(const M3<T>& F, const M3<T>& R, const Sym3<T>& S, T mu, T lambda,
                                     const M3<T>& dF) {
  // m = axial(R^T dF - dF^T R); K = R^T dF, so the skew part's axial vector is
  // (K(2,1) - K(1,2), K(0,2) - K(2,0), K(1,0) - K(0,1))
  T K[9];
#pragma unroll
  for (int c = 0; c < 3; ++c)
#pragma unroll
    for (int r = 0; r < 3; ++r) K[c * 3 + r] = R(0, r) * dF(0, c) + R(1, r) * dF(1, c) + R(2, r) * dF(2, c);
  const T m0 = K[1 * 3 + 2] - K[2 * 3 + 1], m1 = K[2 * 3 + 0] - K[0 * 3 + 2], m2 = K[0 * 3 + 1] - K[1 * 3 + 0];
  // A = tr(S) I - S (symmetric), w = A^-1 m by cofactors
  const T tr = S.xx + S.yy + S.zz;
  const T a = tr - S.xx, b = tr - S.yy, c = tr - S.zz, d = -S.xy, e = -S.xz, f = -S.yz;
  const T i00 = b * c - f * f, i01 = e * f - d * c, i02 = d * f - b * e;
  const T i11 = a * c - e * e, i12 = d * e - a * f, i22 = a * b - d * d;
  const T inv = T(1) / (a * i00 + d * i01 + e * i02);
  const T w0 = (i00 * m0 + i01 * m1 + i02 * m2) * inv;
  const T w1 = (i01 * m0 + i11 * m1 + i12 * m2) * inv;
  const T w2 = (i02 * m0 + i12 * m1 + i22 * m2) * inv;
  const M3<T> C = cofactor3(F);
  const T J = F(0, 0) * C(0, 0) + F(0, 1) * C(0, 1) + F(0, 2) * C(0, 2);
  T dJ = T(0);
#pragma unroll
  for (int k = 0; k < 9; ++k) dJ += C.a[k] * dF.a[k];
  M3<T> out;
#pragma unroll
  for (int r = 0; r < 3; ++r)
#pragma unroll
    for (int cc = 0; cc < 3; ++cc) {
      // dR(r, cc) = sum_k R(r, k) W(k, cc), W = [w]_x
      const T W0 = cc == 0 ? T(0) : (cc == 1 ? -w2 : w1);  // W(0, cc)
      const T W1 = cc == 0 ? w2 : (cc == 1 ? T(0) : -w0);  // W(1, cc)
      const T W2 = cc == 0 ? -w1 : (cc == 1 ? w0 : T(0));  // W(2, cc)
      const T dR = R(r, 0) * W0 + R(r, 1) * W1 + R(r, 2) * W2;
      const int r1 = (r + 1) % 3, r2 = (r + 2) % 3, c1 = (cc + 1) % 3, c2 = (cc + 2) % 3;
      const T dC = dF(r1, c1) * F(r2, c2) + F(r1, c1) * dF(r2, c2) - dF(r1, c2) * F(r2, c1) -
                   F(r1, c2) * dF(r2, c1);
      out(r, cc) = T(2) * mu * (dF(r, cc) - dR) + lambda * dJ * C(r, cc) + lambda * (J - T(1)) * dC;
    }
  return out;
}

// Polar factors F = R S of F (S symmetric positive definite): the Newton
// iteration when it settles, else the eigensolve of F^T F (S = V sqrt(L) V^T,
// R = F S^-1).  Returns false for a singular F.
template <typename T>
SNOW_HD bool polar_factors(const M3<T>& F, M3<T>& R, Sym3<T>& S) {
  if (!polar_newton(F, R)) {
    T lam[3], q[9];
    sym_eig3(gram_cols(F), lam, q, EigTol<T>::tol, EigTol<T>::sweeps);
    T inv[3];
#pragma unroll
    for (int i = 0; i < 3; ++i) {
      const T s = sqrt(lam[i] > T(0) ? lam[i] : T(0));
      if (!(s > T(0))) return false;
      inv[i] = T(1) / s;
    }
    const Sym3<T> Si = spectral(q, inv);
#pragma unroll
    for (int r = 0; r < 3; ++r) {
      const T f0 = F(r, 0), f1 = F(r, 1), f2 = F(r, 2);
      R(r, 0) = f0 * Si.xx + f1 * Si.xy + f2 * Si.xz;
      R(r, 1) = f0 * Si.xy + f1 * Si.yy + f2 * Si.yz;
      R(r, 2) = f0 * Si.xz + f1 * Si.yz + f2 * Si.zz;
    }
  }
  S.xx = R(0, 0) * F(0, 0) + R(1, 0) * F(1, 0) + R(2, 0) * F(2, 0);
  S.yy = R(0, 1) * F(0, 1) + R(1, 1) * F(1, 1) + R(2, 1) * F(2, 1);
  S.zz = R(0, 2) * F(0, 2) + R(1, 2) * F(1, 2) + R(2, 2) * F(2, 2);
  S.xy = R(0, 0) * F(0, 1) + R(1, 0) * F(1, 1) + R(2, 0) * F(2, 1);
  S.xz = R(0, 0) * F(0, 2) + R(1, 0) * F(1, 2) + R(2, 0) * F(2, 2);
  S.yz = R(0, 1) * F(0, 2) + R(1, 1) * F(1, 2) + R(2, 1) * F(2, 2);
  return true;
}

// Mixed-precision guard: true when a singular value of the trial F_E lies
// within `tau` of a clamp bound (the float eigensolve may decide the clamp
// wrongly), or when a clamp acts and two singular values lie within `tau` of
// each other (the float eigenvectors of the nearly repeated pair are then least
// reliable and the clamp acts along them) -- the cases in which the projection
// is redone in double.  Without a clamp the projection is the identity, and
// nearly repeated singular values (F_E close to a rotation, the common
// unstrained state) need no double.
template <typename T>
SNOW_HD bool near_critical(const T s[3], T lo, T hi, T tau, bool clamped) {
  bool crit = false;
#pragma unroll
  for (int i = 0; i < 3; ++i) {
    crit |= fabs(s[i] - lo) < tau || fabs(s[i] - hi) < tau;
    if (clamped) {
#pragma unroll
      for (int j = i + 1; j < 3; ++j) crit |= fabs(s[i] - s[j]) < tau;
    }
  }
  return crit;
}

// grid_velocity (grid.cpp:195-204): for a node with mass > 0,
// v = p / m + dt (f / m + g); p / m is returned in `pm` for the FLIP increment.
template <typename T>
SNOW_HD bool node_velocity(T m, const T p[3], const T f[3], const T g[3], T dt, T v[3], T pm[3]) {
  if (!(m > T(0))) return false;
#pragma unroll
  for (int a = 0; a < 3; ++a) {
    pm[a] = p[a] / m;
    v[a] = pm[a] + dt * ((f[a] / m) + g[a]);
  }
  return true;
}

// ------------------------------------------------------------------ colliders
// Collider record shared by host and device.  kind 0 = half-space bounded by a
// plane (make_plane, src/collision.cpp:5-27: phi = n.(x - p), normal n).
// `velocity` is the collider's rigid velocity (make_plane sets zero).
struct Collider {
  int32_t kind;
  int32_t pad;
  double point[3];
  double normal[3];
  double velocity[3];
  double friction;
  double param[2];   // sphere: param[0] = radius
  double axis[3];    // box: second axis w (unit, orthogonal to `normal`)
  double extent[3];  // box: half extents along u = normal, w, u x w
};
enum : int32_t { COLLIDER_PLANE = 0, COLLIDER_SPHERE = 1, COLLIDER_BOX = 2 };

// Solid oriented box: inside test and outward face normal.  l = the point in
// the box's axes (u, w, u x w), q_k = |l_k| - h_k; inside (phi = max_k q_k <= 0)
// the normal is sign(l_k) times the axis of the largest q_k (first k on a tie,
// sign +1 at l_k = 0).  Returns false outside, where phi > 0.
template <typename T>
SNOW_HD bool box_contact(const Collider& b, T x, T y, T z, T& nx, T& ny, T& nz) {
  const T dx = x - T(b.point[0]), dy = y - T(b.point[1]), dz = z - T(b.point[2]);
  const T u[3] = {T(b.normal[0]), T(b.normal[1]), T(b.normal[2])};
  const T w[3] = {T(b.axis[0]), T(b.axis[1]), T(b.axis[2])};
  const T t[3] = {u[1] * w[2] - u[2] * w[1], u[2] * w[0] - u[0] * w[2], u[0] * w[1] - u[1] * w[0]};
  const T l[3] = {u[0] * dx + u[1] * dy + u[2] * dz, w[0] * dx + w[1] * dy + w[2] * dz,
                  t[0] * dx + t[1] * dy + t[2] * dz};
  int k = 0;
  T qmax = fabs(l[0]) - T(b.extent[0]);
#pragma unroll
  for (int a = 1; a < 3; ++a) {
    const T q = fabs(l[a]) - T(b.extent[a]);
    if (q > qmax) {
      qmax = q;
      k = a;
    }
  }
  if (!(qmax <= T(0))) return false;
  const T s = l[k] < T(0) ? T(-1) : T(1);
  const T* e = k == 0 ? u : (k == 1 ? w : t);
  nx = s * e[0], ny = s * e[1], nz = s * e[2];
  return true;
}

// collision_helper (grid.cpp:206-231): Coulomb friction, stick when
// |v_t| <= -mu v_n, else slide.
// Bodies: a plane phi(x) = n . (x - p) with unit normal n (make_plane,
// src/collision.cpp:5-27), a solid sphere phi(x) = |x - c| - r with normal
// (x - c) / |x - c| (zero at the centre, as Eigen's normalized() leaves it), or
// a solid oriented box (box_contact); each moves with the constant velocity v_c.
template <typename T>
SNOW_HD void collide(const Collider& b, T x, T y, T z, T& vx, T& vy, T& vz) {
  T nx, ny, nz;
  if (b.kind == COLLIDER_BOX) {
    if (!box_contact(b, x, y, z, nx, ny, nz)) return;
  } else if (b.kind == COLLIDER_SPHERE) {
    const T ex = x - T(b.point[0]), ey = y - T(b.point[1]), ez = z - T(b.point[2]);
    const T len = sqrt(ex * ex + ey * ey + ez * ez);
    if (!(len - T(b.param[0]) <= T(0))) return;
    const T inv = len > T(0) ? T(1) / len : T(0);
    nx = ex * inv, ny = ey * inv, nz = ez * inv;
  } else {
    nx = T(b.normal[0]), ny = T(b.normal[1]), nz = T(b.normal[2]);
    const T phi = nx * (x - T(b.point[0])) + ny * (y - T(b.point[1])) + nz * (z - T(b.point[2]));
    if (!(phi <= T(0))) return;
  }
  const T cx = T(b.velocity[0]), cy = T(b.velocity[1]), cz = T(b.velocity[2]);
  const T rx = vx - cx, ry = vy - cy, rz = vz - cz;
  const T vn = rx * nx + ry * ny + rz * nz;
  if (!(vn < T(0))) return;
  const T tx = rx - vn * nx, ty = ry - vn * ny, tz = rz - vn * nz;
  const T tn = sqrt(tx * tx + ty * ty + tz * tz);
  const T mu = T(b.friction);
  T ox, oy, oz;
  if (tn <= T(-1) * mu * vn) {
    ox = oy = oz = T(0);
  } else {
    const T k = mu * vn;
    ox = tx + k * (tx / tn);
    oy = ty + k * (ty / tn);
    oz = tz + k * (tz / tn);
  }
  vx = ox + cx;
  vy = oy + cy;
  vz = oz + cz;
}

}  // namespace snow
