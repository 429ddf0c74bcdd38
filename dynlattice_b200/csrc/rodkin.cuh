// Rod kinematics of the two-node geometrically exact element, shared by the
// device kernels and the host set-up code (__host__ __device__).
//
// The reference formulates the element with 3x3 rotation matrices
// (Line3D.cpp:117-273, helpers.cpp:99-197): node frames
// Lambda_n = exp(theta_n) Lambda_N, reference rotation
// Lambda_r = Lambda_I exp(1/2 log(Lambda_I^T Lambda_J)), local rotation vectors
// psi_n = log(Lambda_r^T Lambda_n), Gauss-point frames
// Lambda(xi) = Lambda_r exp(sum N_n psi_n), curvature
// K = unskew(Lambda^T Lambda').  For two nodes psi_I = -phi/2, psi_J = +phi/2
// with phi = log(Lambda_I^T Lambda_J), so Lambda(xi) = Lambda_r exp(xi phi/2)
// and K = phi / L exactly (psi and psi' are parallel).  The engine evaluates
// these closed forms with unit quaternions: one log and one half-angle
// quaternion per element instead of three logs and three exps per call.
#pragma once

#ifndef __CUDACC_RTC__
#include <cmath>
#endif

#ifdef __CUDACC__
#define DL_HD __host__ __device__ __forceinline__
#else
#define DL_HD inline
#endif

namespace dl {

template <class T>
struct V3 {
  T x, y, z;
};
template <class T>
struct Q4 {  // w + (x, y, z)
  T w, x, y, z;
};

template <class T>
DL_HD V3<T> v3(T x, T y, T z) {
  return V3<T>{x, y, z};
}
template <class T>
DL_HD V3<T> operator+(V3<T> a, V3<T> b) {
  return V3<T>{a.x + b.x, a.y + b.y, a.z + b.z};
}
template <class T>
DL_HD V3<T> operator-(V3<T> a, V3<T> b) {
  return V3<T>{a.x - b.x, a.y - b.y, a.z - b.z};
}
template <class T>
DL_HD V3<T> operator*(T s, V3<T> a) {
  return V3<T>{s * a.x, s * a.y, s * a.z};
}
template <class T>
DL_HD T dot(V3<T> a, V3<T> b) {
  return a.x * b.x + a.y * b.y + a.z * b.z;
}
template <class T>
DL_HD V3<T> cross(V3<T> a, V3<T> b) {
  return V3<T>{a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x};
}
template <class T, class U>
DL_HD V3<T> cvt(V3<U> a) {
  return V3<T>{static_cast<T>(a.x), static_cast<T>(a.y), static_cast<T>(a.z)};
}
template <class T, class U>
DL_HD Q4<T> cvtq(Q4<U> a) {
  return Q4<T>{static_cast<T>(a.w), static_cast<T>(a.x), static_cast<T>(a.y), static_cast<T>(a.z)};
}

template <class T>
DL_HD Q4<T> qmul(Q4<T> a, Q4<T> b) {
  return Q4<T>{a.w * b.w - a.x * b.x - a.y * b.y - a.z * b.z,
               a.w * b.x + a.x * b.w + a.y * b.z - a.z * b.y,
               a.w * b.y - a.x * b.z + a.y * b.w + a.z * b.x,
               a.w * b.z + a.x * b.y - a.y * b.x + a.z * b.w};
}
template <class T>
DL_HD Q4<T> qconj(Q4<T> a) {
  return Q4<T>{a.w, -a.x, -a.y, -a.z};
}
// R(q) v - v = 2w (u x v) + 2 u x (u x v): the rotation's correction of v,
// computed without forming R(q) v (no cancellation for small rotations).
template <class T>
DL_HD V3<T> qrot_delta(Q4<T> q, V3<T> v) {
  V3<T> u{q.x, q.y, q.z};
  V3<T> t = cross(u, v);
  V3<T> tt = cross(u, t);
  return V3<T>{T(2) * (q.w * t.x + tt.x), T(2) * (q.w * t.y + tt.y), T(2) * (q.w * t.z + tt.z)};
}
template <class T>
DL_HD V3<T> qrot(Q4<T> q, V3<T> v) {
  return v + qrot_delta(q, v);
}

DL_HD float dl_sqrt(float x) { return sqrtf(x); }
DL_HD double dl_sqrt(double x) { return sqrt(x); }
DL_HD float dl_rsqrt(float x) {
#ifdef __CUDA_ARCH__
  return rsqrtf(x);
#else
  return 1.0f / std::sqrt(x);
#endif
}
DL_HD double dl_rsqrt(double x) {
#ifdef __CUDA_ARCH__
  return rsqrt(x);
#else
  return 1.0 / std::sqrt(x);
#endif
}
DL_HD float dl_atan2(float y, float x) { return atan2f(y, x); }
DL_HD double dl_atan2(double y, double x) { return atan2(y, x); }
DL_HD void dl_sincos(float x, float *s, float *c) {
#ifdef __CUDA_ARCH__
  sincosf(x, s, c);
#else
  *s = std::sin(x);
  *c = std::cos(x);
#endif
}
DL_HD void dl_sincos(double x, double *s, double *c) {
#ifdef __CUDA_ARCH__
  sincos(x, s, c);
#else
  *s = std::sin(x);
  *c = std::cos(x);
#endif
}
template <class T>
DL_HD T tiny_angle();
template <>
DL_HD float tiny_angle<float>() {
  return 1e-30f;
}
template <>
DL_HD double tiny_angle<double>() {
  return 1e-300;
}

// exp: rotation vector -> unit quaternion (helpers.cpp:139-157 as a quaternion)
template <class T>
DL_HD Q4<T> qexp(V3<T> phi) {
  T th = dl_sqrt(dot(phi, phi));
  if (th < tiny_angle<T>()) return Q4<T>{T(1), T(0.5) * phi.x, T(0.5) * phi.y, T(0.5) * phi.z};
  T s, c;
  dl_sincos(T(0.5) * th, &s, &c);
  T f = s / th;
  return Q4<T>{c, f * phi.x, f * phi.y, f * phi.z};
}
// exp for the per-step rotation increment dt*omega: for angles below 0.05 the
// Taylor series of cos(t/2) and sin(t/2)/t (through t^8) is exact to double
// rounding, which avoids the double-precision sincos in the node update.
template <class T>
DL_HD Q4<T> qexp_small(V3<T> phi) {
  const T t2 = dot(phi, phi);
  if (t2 > T(0.0025)) return qexp(phi);
  const T c = T(1) + t2 * (T(-1.0 / 8) + t2 * (T(1.0 / 384) + t2 * (T(-1.0 / 46080) + t2 * T(1.0 / 10321920))));
  const T f = T(0.5) + t2 * (T(-1.0 / 48) + t2 * (T(1.0 / 3840) + t2 * (T(-1.0 / 645120) + t2 * T(1.0 / 185794560))));
  return Q4<T>{c, f * phi.x, f * phi.y, f * phi.z};
}

// log: unit quaternion with w >= 0 -> rotation vector, angle in [0, pi]
// (helpers.cpp:99-111 as a quaternion)
template <class T>
DL_HD V3<T> qlog(Q4<T> q) {
  if (q.w < T(0)) q = Q4<T>{-q.w, -q.x, -q.y, -q.z};
  V3<T> u{q.x, q.y, q.z};
  T s = dl_sqrt(dot(u, u));
  T f = (s < tiny_angle<T>()) ? T(2) / q.w : T(2) * dl_atan2(s, q.w) / s;
  return f * u;
}
// square root of a unit quaternion with w >= 0: exp(log(q)/2)
template <class T>
DL_HD Q4<T> qhalf(Q4<T> q) {
  if (q.w < T(0)) q = Q4<T>{-q.w, -q.x, -q.y, -q.z};
  T c = T(1) + q.w;
  T inv = dl_rsqrt(T(2) * c);
  return Q4<T>{c * inv, q.x * inv, q.y * inv, q.z * inv};
}
template <class T>
DL_HD Q4<T> qnormalize(Q4<T> q) {
  T i = dl_rsqrt(q.w * q.w + q.x * q.x + q.y * q.y + q.z * q.z);
  return Q4<T>{q.w * i, q.x * i, q.y * i, q.z * i};
}

// Rotation matrix of a unit quaternion, row-major m[3][3].
template <class T>
DL_HD void qmat(Q4<T> q, T m[3][3]) {
  T ww = q.w * q.w, xx = q.x * q.x, yy = q.y * q.y, zz = q.z * q.z;
  T xy = q.x * q.y, xz = q.x * q.z, yz = q.y * q.z, wx = q.w * q.x, wy = q.w * q.y, wz = q.w * q.z;
  m[0][0] = ww + xx - yy - zz;
  m[0][1] = T(2) * (xy - wz);
  m[0][2] = T(2) * (xz + wy);
  m[1][0] = T(2) * (xy + wz);
  m[1][1] = ww - xx + yy - zz;
  m[1][2] = T(2) * (yz - wx);
  m[2][0] = T(2) * (xz - wy);
  m[2][1] = T(2) * (yz + wx);
  m[2][2] = ww - xx - yy + zz;
}

// Element kinematics common to the forward kernels and the host set-up.
// Inputs: node positions (FP64), node rotations R_I, R_J (FP64 state), the
// element-end frames Lambda_N (quaternions), 1/L0.  Outputs in the element's
// compute type T; the cancellation-prone parts (chord, relative rotation,
// Lambda_r^T phi' - e3) are formed in FP64.
template <class T>
struct ElemKin {
  V3<T> phi;      // log(Lambda_I^T Lambda_J)
  V3<T> d;        // Lambda_r^T phi'   (material-frame chord direction)
  V3<T> dme3;     // d - e3, formed in FP64
  V3<T> phiP;     // phi' = (x_J - x_I) / L0 (spatial)
  Q4<T> qr;       // Lambda_r
};

template <class T>
DL_HD ElemKin<T> elem_kin(V3<double> xi, V3<double> xj, Q4<double> Ri, Q4<double> Rj,
                          Q4<double> qNi, Q4<double> qNj, double invL0) {
  ElemKin<T> k;
  Q4<double> LI = qmul(Ri, qNi);
  Q4<double> LJ = qmul(Rj, qNj);
  Q4<double> qIJ = qmul(qconj(LI), LJ);
  if (qIJ.w < 0.0) qIJ = Q4<double>{-qIJ.w, -qIJ.x, -qIJ.y, -qIJ.z};
  k.phi = qlog(cvtq<T>(qIJ));
  Q4<double> qh = qhalf(qIJ);
  Q4<double> Lr = qmul(LI, qh);
  V3<double> pp = invL0 * (xj - xi);
  V3<double> dd = qrot(qconj(Lr), pp);
  k.d = cvt<T>(dd);
  k.dme3 = V3<T>{static_cast<T>(dd.x), static_cast<T>(dd.y), static_cast<T>(dd.z - 1.0)};
  k.phiP = cvt<T>(pp);
  k.qr = cvtq<T>(Lr);
  return k;
}

// Material strains at the Gauss point xi (SpecialCosseratRodModel.cpp:694-744):
//   Gamma = Lambda(xi)^T phi' - Gamma0, K = phi / L0 - K0,
// with Lambda(xi)^T phi' = exp(-xi phi/2) d = d + delta, and
// Gamma - Gamma0 = (d - e3) - (Gamma0 - e3) + delta.
// `e` = exp(-xi phi / 2) is supplied by the caller: for a symmetric Gauss rule
// the rotations of the points +xi and -xi are conjugate quaternions, so one
// exponential serves a pair of points.
template <class T>
DL_HD void gp_strain_e(const ElemKin<T> &k, Q4<T> e, T invL0, const T g0me3[3], const T k0[3],
                       T eps[6], Q4<T> *qgp) {
  V3<T> delta = qrot_delta(e, k.d);
  eps[0] = (k.dme3.x - g0me3[0]) + delta.x;
  eps[1] = (k.dme3.y - g0me3[1]) + delta.y;
  eps[2] = (k.dme3.z - g0me3[2]) + delta.z;
  eps[3] = k.phi.x * invL0 - k0[0];
  eps[4] = k.phi.y * invL0 - k0[1];
  eps[5] = k.phi.z * invL0 - k0[2];
  *qgp = qmul(k.qr, qconj(e));           // Lambda(xi) = Lambda_r exp(xi phi/2)
}

template <class T>
DL_HD void gp_strain(const ElemKin<T> &k, T xi, T invL0, const T g0me3[3], const T k0[3],
                     T eps[6], Q4<T> *qgp) {
  gp_strain_e(k, qexp((T(-0.5) * xi) * k.phi), invL0, g0me3, k0, eps, qgp);
}

// ---------------------------------------------------------------------------
// Elements of n = 3 or 4 nodes (FP64; Line3D.cpp:117-273 in the reference's
// matrix form).  Node frames Lambda_a = R_a Lambda_N,a; no closed form applies
// (the local rotation vectors are not parallel), so each Gauss point
// interpolates psi(xi) = sum N_a psi_a and forms exp(psi) and the curvature.
// ---------------------------------------------------------------------------
constexpr int kMaxElemNodes = 4;

// Reference rotation Lambda_r = Lambda_I exp(1/2 log(Lambda_I^T Lambda_J)),
// I = (n-1)/2, J = n/2 (Line3D::getRefRot_, Line3D.cpp:249-263), and the local
// rotation vectors psi_a = log(Lambda_r^T Lambda_a) (getNodeRotVecs_, :265-273).
DL_HD void line_ref(const Q4<double> *L, int n, Q4<double> &Lr, V3<double> *psi) {
  const int I = (n - 1) / 2, J = n / 2;
  Q4<double> qIJ = qmul(qconj(L[I]), L[J]);
  if (qIJ.w < 0.0) qIJ = Q4<double>{-qIJ.w, -qIJ.x, -qIJ.y, -qIJ.z};
  Lr = qmul(L[I], qhalf(qIJ));
  for (int a = 0; a < n; ++a) psi[a] = qlog(qmul(qconj(Lr), L[a]));
}

// J_r(psi) v with the right Jacobian of the exponential map,
//   J_r(psi) = I - (1 - cos t)/t^2 [psi]x + (t - sin t)/t^3 [psi]x^2,  t = |psi|:
// for Lambda(xi) = Lambda_r exp(psi(xi)) the material curvature
// unskew(Lambda^T Lambda') (getRotationGradients with expVecP, Line3D.cpp:216-244;
// getStrains_, SpecialCosseratRodModel.cpp:694-744) is J_r(psi) psi'.  Below
// t = 0.01 the coefficients come from their Taylor series (the closed forms
// cancel there).
DL_HD V3<double> exp_right_jacobian(V3<double> psi, V3<double> v) {
  const double t2 = dot(psi, psi);
  double c1, c2;
  if (t2 < 1e-4) {
    c1 = 0.5 - t2 * (1.0 / 24.0 - t2 / 720.0);
    c2 = 1.0 / 6.0 - t2 * (1.0 / 120.0 - t2 / 5040.0);
  } else {
    const double t = dl_sqrt(t2);
    c1 = (1.0 - cos(t)) / t2;
    c2 = (t - sin(t)) / (t2 * t);
  }
  const V3<double> pxv = cross(psi, v);
  return (v - c1 * pxv) + c2 * cross(psi, pxv);
}

// One Gauss point of an n-node element: the frame Lambda = Lambda_r exp(psi)
// (Line3D::getRotations, Line3D.cpp:117-139), phi' = sum x_a N_a', the
// material strains Lambda^T phi' - e3 and K (before the reference values are
// subtracted).  N, dN: the point's shape values and gradients per node.
struct GpKinN {
  Q4<double> L;
  V3<double> phiP;
  V3<double> gme3;
  V3<double> K;
};
DL_HD GpKinN gp_kin_n(const V3<double> *x, const Q4<double> &Lr, const V3<double> *psi, int n, const double *N,
                      const double *dN) {
  V3<double> ps{0.0, 0.0, 0.0}, pp{0.0, 0.0, 0.0}, phiP{0.0, 0.0, 0.0};
  for (int a = 0; a < n; ++a) {
    ps = ps + N[a] * psi[a];
    pp = pp + dN[a] * psi[a];
    phiP = phiP + dN[a] * x[a];
  }
  GpKinN k;
  k.L = qmul(Lr, qexp(ps));
  const V3<double> gam = qrot(qconj(k.L), phiP);
  k.gme3 = V3<double>{gam.x, gam.y, gam.z - 1.0};
  k.K = exp_right_jacobian(ps, pp);
  k.phiP = phiP;
  return k;
}

}  // namespace dl
