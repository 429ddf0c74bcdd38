// Reverse-mode (adjoint) building blocks of the explicit step, shared by the
// adjoint kernels (device) and the host check harness (__host__ __device__).
//
// The forward step is the one of step.cuh: element phase (rod kinematics with
// quaternions, strains, stress resultants with the cutting-plane return map
// and history commit, end forces) and node phase (lumped mass with the
// rotational block R S R^T, gyroscopic term, acceleration constraints,
// v += dt a, x += dt v, R <- exp(dt omega) R).  Here each of those functions
// has a pure form (explicit inputs and outputs, no memory side effects) and a
// hand-written vector-Jacobian product.
//
// Conventions.  Quaternion arguments are differentiated as plain 4-vectors of
// components (every quaternion formula is a smooth function of its
// components).  The adjoint of a node rotation is a 3-vector mu in the
// spatial tangent space: a perturbation R -> exp([dtheta]) R changes the
// objective by mu . dtheta.  Translational adjoints are plain 3-vectors.
#pragma once

#include "rodkin.cuh"

namespace dl {

// ---------------------------------------------------------------------------
// small helpers
// ---------------------------------------------------------------------------
template <class T>
DL_HD Q4<T> qadd(Q4<T> a, Q4<T> b) {
  return Q4<T>{a.w + b.w, a.x + b.x, a.y + b.y, a.z + b.z};
}
template <class T>
DL_HD Q4<T> qscale(T s, Q4<T> a) {
  return Q4<T>{s * a.w, s * a.x, s * a.y, s * a.z};
}
template <class T>
DL_HD Q4<T> qzero() {
  return Q4<T>{T(0), T(0), T(0), T(0)};
}
template <class T>
DL_HD V3<T> vzero() {
  return V3<T>{T(0), T(0), T(0)};
}
template <class T>
DL_HD V3<T> qvec(Q4<T> q) {
  return V3<T>{q.x, q.y, q.z};
}

// c = a b  ->  la += lc conj(b), lb += conj(a) lc   (L_a^T = L_conj(a), R_b^T = R_conj(b))
template <class T>
DL_HD void qmul_vjp(Q4<T> a, Q4<T> b, Q4<T> lc, Q4<T> &la, Q4<T> &lb) {
  la = qadd(la, qmul(lc, qconj(b)));
  lb = qadd(lb, qmul(qconj(a), lc));
}

// o = qrot_delta(q, v) = 2 w (u x v) + 2 u x (u x v)
template <class T>
DL_HD void qrot_delta_vjp(Q4<T> q, V3<T> v, V3<T> lo, Q4<T> &lq, V3<T> &lv) {
  const V3<T> u{q.x, q.y, q.z};
  const V3<T> t = cross(u, v);
  const V3<T> lxu = cross(lo, u);
  lv = lv + T(2) * (q.w * lxu + cross(lxu, u));
  lq.w += T(2) * dot(lo, t);
  const V3<T> lu = T(2) * (q.w * cross(v, lo) + cross(t, lo) + cross(v, lxu));
  lq.x += lu.x;
  lq.y += lu.y;
  lq.z += lu.z;
}
// o = qrot(q, v) = v + qrot_delta(q, v)
template <class T>
DL_HD void qrot_vjp(Q4<T> q, V3<T> v, V3<T> lo, Q4<T> &lq, V3<T> &lv) {
  lv = lv + lo;
  qrot_delta_vjp(q, v, lo, lq, lv);
}

// q = qexp(phi): (cos(t/2), f phi), f = sin(t/2)/t, t = |phi|
//   dq.w/dphi = -(f/2) phi,  d(f phi)/dphi = f I + g phi phi^T, g = f'(t)/t
template <class T>
DL_HD V3<T> qexp_vjp(V3<T> phi, Q4<T> lq) {
  const T t2 = dot(phi, phi);
  T f, g;
  if (t2 < T(1e-4)) {
    // f = 1/2 - t^2/48 + t^4/3840;  g = -1/24 + t^2/960 - t^4/64512
    f = T(0.5) + t2 * (T(-1.0 / 48) + t2 * T(1.0 / 3840));
    g = T(-1.0 / 24) + t2 * (T(1.0 / 960) + t2 * T(-1.0 / 64512));
  } else {
    const T t = dl_sqrt(t2);
    T s, c;
    dl_sincos(T(0.5) * t, &s, &c);
    f = s / t;
    g = (T(0.5) * c - f) / t2;
  }
  const V3<T> lu{lq.x, lq.y, lq.z};
  return (T(-0.5) * f * lq.w) * phi + f * lu + (g * dot(phi, lu)) * phi;
}

// phi = qlog(q) for w >= 0: phi = h(s, w) u, h = 2 atan2(s, w) / s, s = |u|
template <class T>
DL_HD Q4<T> qlog_vjp(Q4<T> q, V3<T> lphi) {
  const V3<T> u{q.x, q.y, q.z};
  const T s2 = dot(u, u);
  const T w = q.w;
  T h, hs_over_s;  // h and (dh/ds)/s
  const T r2 = s2 + w * w;
  if (s2 < T(1e-6) * w * w) {
    // atan(s/w)/s = (1/w)(1 - z/3 + z^2/5), z = s^2/w^2
    const T iw = T(1) / w, z = s2 * iw * iw;
    h = T(2) * iw * (T(1) + z * (T(-1.0 / 3) + z * T(1.0 / 5)));
    hs_over_s = iw * iw * iw * (T(-4.0 / 3) + z * T(8.0 / 5));
  } else {
    const T s = dl_sqrt(s2);
    const T at = dl_atan2(s, w);
    h = T(2) * at / s;
    hs_over_s = T(2) * (w / r2 - at / s) / s2;
  }
  const T hw = T(-2) / r2;  // dh/dw
  const T ul = dot(u, lphi);
  const V3<T> lu = h * lphi + (ul * hs_over_s) * u;
  return Q4<T>{ul * hw, lu.x, lu.y, lu.z};
}

// o = qhalf(q) for w >= 0: (sqrt((1+w)/2), u / sqrt(2 (1+w)))
template <class T>
DL_HD Q4<T> qhalf_vjp(Q4<T> q, Q4<T> lo) {
  const T c = T(1) + q.w;
  const T inv = dl_rsqrt(T(2) * c);
  const T ow = c * inv;
  const V3<T> u{q.x, q.y, q.z};
  const V3<T> lu{lo.x, lo.y, lo.z};
  const T lw = lo.w * T(0.25) / ow - dot(lu, u) * inv * inv * inv;
  return Q4<T>{lw, inv * lu.x, inv * lu.y, inv * lu.z};
}

// tangent adjoint of a unit quaternion R from its component adjoint lR:
// d(lR . R) under R -> (1, dtheta/2) R  gives mu = (-lw u + w lu + u x lu)/2
template <class T>
DL_HD V3<T> rot_tangent(Q4<T> R, Q4<T> lR) {
  const V3<T> u{R.x, R.y, R.z};
  const V3<T> lu{lR.x, lR.y, lR.z};
  return T(0.5) * ((-lR.w) * u + R.w * lu + cross(u, lu));
}

// 3x3 helpers (row-major)
template <class T>
DL_HD void m3_from_q(Q4<T> q, T m[3][3]) {
  qmat(q, m);
}
template <class T>
DL_HD V3<T> m3_mul(const T m[3][3], V3<T> v) {
  return V3<T>{m[0][0] * v.x + m[0][1] * v.y + m[0][2] * v.z, m[1][0] * v.x + m[1][1] * v.y + m[1][2] * v.z,
               m[2][0] * v.x + m[2][1] * v.y + m[2][2] * v.z};
}
template <class T>
DL_HD V3<T> m3_tmul(const T m[3][3], V3<T> v) {
  return V3<T>{m[0][0] * v.x + m[1][0] * v.y + m[2][0] * v.z, m[0][1] * v.x + m[1][1] * v.y + m[2][1] * v.z,
               m[0][2] * v.x + m[1][2] * v.y + m[2][2] * v.z};
}

// J_l(phi)^T lam for the left Jacobian of the SO(3) exponential:
// J_l = I + a [phi] + b [phi]^2, a = (1 - cos t)/t^2, b = (t - sin t)/t^3
template <class T>
DL_HD V3<T> jl_t(V3<T> phi, V3<T> lam) {
  const T t2 = dot(phi, phi);
  T a, b;
  if (t2 < T(1e-4)) {
    a = T(0.5) + t2 * (T(-1.0 / 24) + t2 * T(1.0 / 720));
    b = T(1.0 / 6) + t2 * (T(-1.0 / 120) + t2 * T(1.0 / 5040));
  } else {
    const T t = dl_sqrt(t2);
    T s, c;
    dl_sincos(t, &s, &c);
    a = (T(1) - c) / t2;
    b = (t - s) / (t2 * t);
  }
  // [phi]^T = -[phi]; ([phi]^2)^T = [phi]^2; [phi]^2 v = phi x (phi x v)
  return lam - a * cross(phi, lam) + b * cross(phi, cross(phi, lam));
}

// ---------------------------------------------------------------------------
// element: pure forward and its vector-Jacobian product
// ---------------------------------------------------------------------------
constexpr int kAdjMaxG = 3;
constexpr int kAdjMaxNh = 7;
constexpr int kAdjMaxIter = 32;

// Hardening-parameter count of a yield policy as array bound: the policy's
// compile-time count (at least 1), or kAdjMaxNh when it is known only at run
// time (kNh < 0).  With a compile-time count the loops over the hardening
// parameters unroll and their arrays stay in registers.
template <class Y>
struct AdjNhCap {
  static constexpr int value = Y::kNh > 0 ? Y::kNh : (Y::kNh == 0 ? 1 : kAdjMaxNh);
};

// Gauss points/weights of Gauss1..Gauss3 (same values as step.cuh)
DL_HD double adj_gxi(int G, int g) {
  const double t[3][3] = {{0.0, 0.0, 0.0},
                          {-0.57735026918962576451, 0.57735026918962576451, 0.0},
                          {-0.77459666924148337704, 0.0, 0.77459666924148337704}};
  return t[G - 1][g];
}
DL_HD double adj_gw(int G, int g) {
  const double t[3][3] = {{2.0, 0.0, 0.0}, {1.0, 1.0, 0.0},
                          {0.55555555555555555556, 0.88888888888888888889, 0.55555555555555555556}};
  return t[G - 1][g];
}

// constants and state of one element at the start of a step
template <class T>
struct ElemIn {
  V3<double> xi, xj;
  Q4<double> Ri, Rj, qNi, qNj;
  double invL0 = 0.0, L0 = 0.0;
  T C[6];
  T ec[2];                          // radius, area (yield-expression variables)
  T g0[kAdjMaxG][3], k0[kAdjMaxG][3];
  int G = 2, nh = 0, plastic = 0;
  // committed history (plastic only)
  T ep[kAdjMaxG][6], al[kAdjMaxG][kAdjMaxNh], epsc[kAdjMaxG][6];
};

// plasticity law constants (copied from DevModel)
template <class T>
struct PlastLaw {
  const T (*H)[7];
  int max_iter;
  T prec;
};

// history after the step and its adjoint
template <class T>
struct ElemHist {
  T ep[kAdjMaxG][6], al[kAdjMaxG][kAdjMaxNh], epsc[kAdjMaxG][6];
  double dediss[kAdjMaxG];  // dissipation added this step
};
struct ElemHistAdj {
  double ep[kAdjMaxG][6], al[kAdjMaxG][kAdjMaxNh], epsc[kAdjMaxG][6];
};

// Return map at one Gauss point (ElastoPlasticRodMaterial::getStress,
// ElastoPlasticRodMaterial.cpp:198-269, commit of applyDeform :271-307), pure
// form.  Y provides f(args), grad(args) and vjp(args, lf, lg, largs) for
// args = (sigma[6], q[nh] = -H alpha, radius, area).  When `iters` is given the
// iterates ep_i, alpha_i and the steps ddf_i are recorded (i < *n_it).
template <class T, class Y, class M>
DL_HD void rm_forward(const M &mdl, const PlastLaw<T> &law, int nh_in, const T ec[2], const T eps[6], const T C[6],
                      const T ep0[6], const T al0[], const T epsc_old[6], T sig[6], T ep[6], T al[],
                      double &dediss, bool &active, int &n_it, bool &overflow, T (*it_ep)[6] = nullptr,
                      T (*it_al)[AdjNhCap<Y>::value] = nullptr, T *it_ddf = nullptr) {
  constexpr int NHM = AdjNhCap<Y>::value;
  const int nh = Y::kNh >= 0 ? Y::kNh : nh_in;
  for (int k = 0; k < 6; ++k) ep[k] = ep0[k];
  for (int a = 0; a < nh; ++a) al[a] = al0[a];
  T args[6 + NHM + 2];
  args[6 + nh] = ec[0];
  args[7 + nh] = ec[1];
  T dflow = T(0);
  int it = 0;
  overflow = false;
  for (;;) {
    for (int k = 0; k < 6; ++k) sig[k] = C[k] * (eps[k] - ep[k]);
    for (int a = 0; a < nh; ++a) {
      T s = T(0);
      for (int b = 0; b < nh; ++b) s += law.H[a][b] * al[b];
      args[6 + a] = -s;
    }
    for (int k = 0; k < 6; ++k) args[k] = sig[k];
    const T fv = Y::f(mdl, args);
    if (!(it < law.max_iter) || it >= kAdjMaxIter) {
      overflow = true;
      break;
    }
    if (fv < law.prec) break;
    T gr[6 + NHM];
    Y::grad(mdl, args, gr);
    T den = T(0);
    for (int k = 0; k < 6; ++k) den += gr[k] * C[k] * gr[k];
    for (int a = 0; a < nh; ++a) {
      T s = T(0);
      for (int b = 0; b < nh; ++b) s += law.H[a][b] * gr[6 + b];
      den += gr[6 + a] * s;
    }
    const T ddf = fv / den;
    if (it_ep) {
      for (int k = 0; k < 6; ++k) it_ep[it][k] = ep[k];
      for (int a = 0; a < nh; ++a) it_al[it][a] = al[a];
      it_ddf[it] = ddf;
    }
    for (int k = 0; k < 6; ++k) ep[k] += ddf * gr[k];
    for (int a = 0; a < nh; ++a) al[a] += ddf * gr[6 + a];
    dflow += ddf;
    ++it;
  }
  n_it = it;
  dediss = 0.0;
  active = fabs(double(dflow)) > 2.220446049250313e-16;
  if (active) {
    for (int k = 0; k < 6; ++k) {
      const double so = double(C[k]) * double(epsc_old[k] - ep0[k]);
      dediss += (so + double(sig[k])) / 2.0 * double(ep[k] - ep0[k]);
    }
  }
}

// Reverse of rm_forward.  Inputs: the forward inputs, the recorded iterates,
// the adjoints of the outputs (lsig, lep_out, lal_out, ld = adjoint of the
// dissipation increment).  Accumulates into leps, lep0, lal0, lepsc_old, lC,
// lec.
template <class T, class Y, class M>
DL_HD void rm_reverse(const M &mdl, const PlastLaw<T> &law, int nh_in, const T ec[2], const T eps[6], const T C[6],
                      const T ep0[6], const T epsc_old[6], const T sig[6], const T ep[6], double dediss_active,
                      int n_it, const T (*it_ep)[6], const T (*it_al)[AdjNhCap<Y>::value], const T *it_ddf,
                      const double lsig_in[6], const double lep_out[6], const double lal_out[], double ld,
                      double leps[6], double lep0[6], double lal0[], double lepsc_old[6], double lC[6],
                      double lec[2]) {
  constexpr int NHM = AdjNhCap<Y>::value;
  const int nh = Y::kNh >= 0 ? Y::kNh : nh_in;
  double lsig[6], lep[6], lal[NHM];
  for (int k = 0; k < 6; ++k) {
    lsig[k] = lsig_in[k];
    lep[k] = lep_out[k];
  }
  for (int a = 0; a < nh; ++a) lal[a] = lal_out[a];
  // dissipation increment D = sum ((C (eold - ep0) + sig) / 2) (ep - ep0)
  if (dediss_active != 0.0 && ld != 0.0) {
    for (int k = 0; k < 6; ++k) {
      const double so = double(C[k]) * double(epsc_old[k] - ep0[k]);
      const double dep = double(ep[k] - ep0[k]);
      const double half = 0.5 * ld;
      lepsc_old[k] += half * double(C[k]) * dep;
      lep0[k] += -half * double(C[k]) * dep - half * (so + double(sig[k]));
      lsig[k] += half * dep;
      lep[k] += half * (so + double(sig[k]));
      lC[k] += half * double(epsc_old[k] - ep0[k]) * dep;
    }
  }
  // final stress sig = C (eps - ep_n)
  for (int k = 0; k < 6; ++k) {
    leps[k] += double(C[k]) * lsig[k];
    lep[k] -= double(C[k]) * lsig[k];
    lC[k] += double(eps[k] - ep[k]) * lsig[k];
  }
  T args[6 + NHM + 2];
  args[6 + nh] = ec[0];
  args[7 + nh] = ec[1];
  for (int i = n_it - 1; i >= 0; --i) {
    // recompute iterate i: sig_i, args_i, f_i, g_i, den_i
    T sgi[6];
    for (int k = 0; k < 6; ++k) sgi[k] = C[k] * (eps[k] - it_ep[i][k]);
    for (int a = 0; a < nh; ++a) {
      T s = T(0);
      for (int b = 0; b < nh; ++b) s += law.H[a][b] * it_al[i][b];
      args[6 + a] = -s;
    }
    for (int k = 0; k < 6; ++k) args[k] = sgi[k];
    const T fv = Y::f(mdl, args);
    T gr[6 + NHM];
    Y::grad(mdl, args, gr);
    double den = 0.0;
    for (int k = 0; k < 6; ++k) den += double(gr[k]) * double(C[k]) * double(gr[k]);
    double Hg[NHM];
    for (int a = 0; a < nh; ++a) {
      double s = 0.0;
      for (int b = 0; b < nh; ++b) s += double(law.H[a][b]) * double(gr[6 + b]);
      Hg[a] = s;
      den += double(gr[6 + a]) * s;
    }
    const double ddf = double(it_ddf[i]);
    // ep_{i+1} = ep_i + ddf g_s, al_{i+1} = al_i + ddf g_h  (lep, lal carry over to ep_i, al_i)
    double lddf = 0.0, lg[6 + NHM];
    for (int k = 0; k < 6; ++k) {
      lddf += lep[k] * double(gr[k]);
      lg[k] = ddf * lep[k];
    }
    for (int a = 0; a < nh; ++a) {
      lddf += lal[a] * double(gr[6 + a]);
      lg[6 + a] = ddf * lal[a];
    }
    // ddf = f / den
    const double lf = lddf / den;
    const double lden = -lddf * double(fv) / (den * den);
    // den = g_s^T C g_s + g_h^T H g_h
    for (int k = 0; k < 6; ++k) {
      lg[k] += 2.0 * double(C[k]) * double(gr[k]) * lden;
      lC[k] += double(gr[k]) * double(gr[k]) * lden;
    }
    for (int a = 0; a < nh; ++a) {
      double s = 0.0;
      for (int b = 0; b < nh; ++b) s += double(law.H[b][a]) * double(gr[6 + b]);
      lg[6 + a] += (Hg[a] + s) * lden;
    }
    // (f, g) = F(args)
    T lgT[6 + NHM], largs[6 + NHM + 2];
    for (int k = 0; k < 6 + nh; ++k) lgT[k] = T(lg[k]);
    for (int k = 0; k < 8 + nh; ++k) largs[k] = T(0);
    Y::vjp(mdl, args, T(lf), lgT, largs);
    // args = (sig_i, -H al_i, radius, area)
    for (int a = 0; a < nh; ++a) {
      double s = 0.0;
      for (int b = 0; b < nh; ++b) s += double(law.H[b][a]) * double(largs[6 + b]);
      lal[a] -= s;
    }
    lec[0] += double(largs[6 + nh]);
    lec[1] += double(largs[7 + nh]);
    // sig_i = C (eps - ep_i)
    for (int k = 0; k < 6; ++k) {
      const double ls = double(largs[k]);
      leps[k] += double(C[k]) * ls;
      lep[k] -= double(C[k]) * ls;
      lC[k] += double(eps[k] - it_ep[i][k]) * ls;
    }
  }
  for (int k = 0; k < 6; ++k) lep0[k] += lep[k];
  for (int a = 0; a < nh; ++a) lal0[a] += lal[a];
}

// Element forward (pure): end forces f[12] = (f_I[6], f_J[6]) and, for
// plastic elements, the committed history after the step.
template <class T, class Y, class M>
DL_HD void elem_forward(const M &mdl, const PlastLaw<T> &law, const ElemIn<T> &in, T f[12], ElemHist<T> *hout,
                        bool *overflow) {
  const ElemKin<T> k = elem_kin<T>(in.xi, in.xj, in.Ri, in.Rj, in.qNi, in.qNj, in.invL0);
  const T il = T(in.invL0);
  const int G = in.G;
  for (int q = 0; q < 12; ++q) f[q] = T(0);
  const Q4<T> epair = qexp((T(-0.5) * T(adj_gxi(G, G - 1))) * k.phi);
  if (overflow) *overflow = false;
  for (int g = 0; g < G; ++g) {
    const T xg = T(adj_gxi(G, g));
    const T Wg = T(adj_gw(G, g));
    const Q4<T> eg = xg > T(0) ? epair : (xg < T(0) ? qconj(epair) : Q4<T>{T(1), T(0), T(0), T(0)});
    T eps[6];
    Q4<T> qg;
    gp_strain_e(k, eg, il, in.g0[g], in.k0[g], eps, &qg);
    T sig[6];
    if (Y::kPlastic && in.plastic) {
      T ep[6], al[kAdjMaxNh];
      double dd = 0.0;
      int nit = 0;
      bool ovf = false, act = false;
      rm_forward<T, Y>(mdl, law, in.nh, in.ec, eps, in.C, in.ep[g], in.al[g], in.epsc[g], sig, ep, al, dd, act, nit,
                       ovf);
      if (overflow && ovf) *overflow = true;
      if (hout) {
        for (int q = 0; q < 6; ++q) {
          hout->ep[g][q] = ep[q];
          hout->epsc[g][q] = eps[q];
        }
        for (int a = 0; a < in.nh; ++a) hout->al[g][a] = al[a];
        hout->dediss[g] = dd;
      }
    } else {
      for (int q = 0; q < 6; ++q) sig[q] = in.C[q] * eps[q];
      if (hout) hout->dediss[g] = 0.0;
    }
    const double wgt = adj_gw(G, g) * 0.5 * in.L0;
    const V3<T> nn = qrot(qg, V3<T>{sig[0], sig[1], sig[2]});
    const V3<T> mm = qrot(qg, V3<T>{sig[3], sig[4], sig[5]});
    const V3<T> pxn = cross(k.phiP, nn);
    const T hw = T(0.5) * Wg;
    const T wI = T(wgt) * (T(0.5) * (T(1) - xg));
    const T wJ = T(wgt) * (T(0.5) * (T(1) + xg));
    f[0] -= hw * nn.x; f[1] -= hw * nn.y; f[2] -= hw * nn.z;
    f[3] += -hw * mm.x - wI * pxn.x;
    f[4] += -hw * mm.y - wI * pxn.y;
    f[5] += -hw * mm.z - wI * pxn.z;
    f[6] += hw * nn.x; f[7] += hw * nn.y; f[8] += hw * nn.z;
    f[9] += hw * mm.x - wJ * pxn.x;
    f[10] += hw * mm.y - wJ * pxn.y;
    f[11] += hw * mm.z - wJ * pxn.z;
  }
}

// adjoint outputs of one element
struct ElemAdjOut {
  V3<double> lxi, lxj, lthi, lthj;  // node translations, node rotations (spatial tangent)
  double lC[6];
  double lec[2];
};

// Forward prefix of the element VJP, shared by the Gauss points (as
// elem_kin: the FP64 relative rotation and chord, then the element-precision
// kinematics and the half-pair exponential).
template <class T>
struct ElemPrefix {
  Q4<double> LI, LJ, qIJ, qh, Lr;
  bool flip;
  Q4<T> qIJt;
  V3<double> pp;
  ElemKin<T> k;
  T il, smax;
  Q4<T> epair;
};

// One Gauss point's constants, committed history and history adjoint.
template <class T>
struct GpIn {
  T g0[3], k0[3];
  T ep[6], al[kAdjMaxNh], epsc[6];
};
struct GpHistAdj {
  double ep[6], al[kAdjMaxNh], epsc[6];
};

// Adjoints of the element-precision kinematic quantities and of the section
// constants, summed over the Gauss points.
template <class T>
struct ElemGpAdj {
  V3<T> lphi, ld, ldme3, lppT;
  Q4<T> lqr, lepair;
  double lC[6], lec[2];
};

template <class T>
DL_HD void gp_adj_zero(ElemGpAdj<T> &a) {
  a.lphi = a.ld = a.ldme3 = a.lppT = vzero<T>();
  a.lqr = a.lepair = qzero<T>();
  for (int q = 0; q < 6; ++q) a.lC[q] = 0.0;
  a.lec[0] = a.lec[1] = 0.0;
}

template <class T>
DL_HD void elem_vjp_prefix(const ElemIn<T> &in, ElemPrefix<T> &p) {
  p.LI = qmul(in.Ri, in.qNi);
  p.LJ = qmul(in.Rj, in.qNj);
  p.qIJ = qmul(qconj(p.LI), p.LJ);
  p.flip = p.qIJ.w < 0.0;
  if (p.flip) p.qIJ = Q4<double>{-p.qIJ.w, -p.qIJ.x, -p.qIJ.y, -p.qIJ.z};
  p.qIJt = cvtq<T>(p.qIJ);
  const V3<T> phi = qlog(p.qIJt);
  p.qh = qhalf(p.qIJ);
  p.Lr = qmul(p.LI, p.qh);
  p.pp = in.invL0 * (in.xj - in.xi);
  const V3<double> dd = qrot(qconj(p.Lr), p.pp);
  p.k.phi = phi;
  p.k.d = cvt<T>(dd);
  p.k.dme3 = V3<T>{static_cast<T>(dd.x), static_cast<T>(dd.y), static_cast<T>(dd.z - 1.0)};
  p.k.phiP = cvt<T>(p.pp);
  p.k.qr = cvtq<T>(p.Lr);
  p.il = T(in.invL0);
  p.smax = T(-0.5) * T(adj_gxi(in.G, in.G - 1));
  p.epair = qexp(p.smax * phi);
}

// Gauss point g of the element VJP: recomputes its strain and stress (with
// the return-map iterates), then reverses the end-force accumulation, the
// stress (return map) and the strain into acc.  lh: on entry the adjoint of
// the point's history after the step, on exit that of the history before it.
template <class T, class Y, class M>
DL_HD void elem_vjp_gp(const M &mdl, const PlastLaw<T> &law, const ElemIn<T> &in, const ElemPrefix<T> &p, int g,
                       const GpIn<T> &gi, const double lf[12], GpHistAdj *lh, double ldiss, ElemGpAdj<T> &acc) {
  const int G = in.G;
  const ElemKin<T> &k = p.k;
  const T xg = T(adj_gxi(G, g));
  const T Wg = T(adj_gw(G, g));
  const Q4<T> eg = xg > T(0) ? p.epair : (xg < T(0) ? qconj(p.epair) : Q4<T>{T(1), T(0), T(0), T(0)});
  T eps[6];
  Q4<T> qg;
  gp_strain_e(k, eg, p.il, gi.g0, gi.k0, eps, &qg);
  // stress resultants (recomputed, with the iterates for the reverse sweep)
  T sig[6], ep[6], al[kAdjMaxNh];
  T it_ep[kAdjMaxIter][6], it_al[kAdjMaxIter][AdjNhCap<Y>::value], it_ddf[kAdjMaxIter];
  double dd_g = 0.0;
  int nit = 0;
  bool ovf = false, act = false;
  const bool plastic = Y::kPlastic && in.plastic;
  if (plastic) {
    rm_forward<T, Y>(mdl, law, in.nh, in.ec, eps, in.C, gi.ep, gi.al, gi.epsc, sig, ep, al, dd_g, act, nit, ovf,
                     it_ep, it_al, it_ddf);
  } else {
    for (int q = 0; q < 6; ++q) sig[q] = in.C[q] * eps[q];
  }
  const double wgt = adj_gw(G, g) * 0.5 * in.L0;
  const V3<T> sn{sig[0], sig[1], sig[2]}, sm{sig[3], sig[4], sig[5]};
  const V3<T> nn = qrot(qg, sn);
  const T hw = T(0.5) * Wg;
  const T wI = T(wgt) * (T(0.5) * (T(1) - xg));
  const T wJ = T(wgt) * (T(0.5) * (T(1) + xg));
  // f accumulation reverse
  const V3<T> lfIt{T(lf[0]), T(lf[1]), T(lf[2])}, lfIr{T(lf[3]), T(lf[4]), T(lf[5])};
  const V3<T> lfJt{T(lf[6]), T(lf[7]), T(lf[8])}, lfJr{T(lf[9]), T(lf[10]), T(lf[11])};
  V3<T> lnn = hw * (lfJt - lfIt);
  const V3<T> lmm = hw * (lfJr - lfIr);
  const V3<T> lpxn = T(-1) * (wI * lfIr + wJ * lfJr);
  // pxn = phiP x nn
  acc.lppT = acc.lppT + cross(nn, lpxn);
  lnn = lnn + cross(lpxn, k.phiP);
  // nn = qrot(qg, sn), mm = qrot(qg, sm)
  Q4<T> lqg = qzero<T>();
  V3<T> lsn = vzero<T>(), lsm = vzero<T>();
  qrot_vjp(qg, sn, lnn, lqg, lsn);
  qrot_vjp(qg, sm, lmm, lqg, lsm);
  // stress resultants reverse
  double lsig[6] = {double(lsn.x), double(lsn.y), double(lsn.z), double(lsm.x), double(lsm.y), double(lsm.z)};
  double leps[6] = {0, 0, 0, 0, 0, 0};
  const int nh = Y::kNh >= 0 ? Y::kNh : in.nh;
  if (plastic) {
    double lep0[6] = {0, 0, 0, 0, 0, 0}, lal0[kAdjMaxNh], lepsc_old[6] = {0, 0, 0, 0, 0, 0};
    for (int a = 0; a < nh; ++a) lal0[a] = 0.0;
    // epsc after the step = eps
    for (int q = 0; q < 6; ++q) leps[q] += lh->epsc[q];
    rm_reverse<T, Y>(mdl, law, in.nh, in.ec, eps, in.C, gi.ep, gi.epsc, sig, ep, act ? 1.0 : 0.0, nit, it_ep,
                     it_al, it_ddf, lsig, lh->ep, lh->al, ldiss, leps, lep0, lal0, lepsc_old, acc.lC, acc.lec);
    for (int q = 0; q < 6; ++q) {
      lh->ep[q] = lep0[q];
      lh->epsc[q] = lepsc_old[q];
    }
    for (int a = 0; a < nh; ++a) lh->al[a] = lal0[a];
  } else {
    for (int q = 0; q < 6; ++q) {
      leps[q] += double(in.C[q]) * lsig[q];
      acc.lC[q] += double(eps[q]) * lsig[q];
    }
  }
  // qg = qr conj(eg)
  Q4<T> lceg = qzero<T>();
  qmul_vjp(k.qr, qconj(eg), lqg, acc.lqr, lceg);
  Q4<T> leg = qconj(lceg);
  // eps_t = (dme3 - g0) + qrot_delta(eg, d); eps_r = phi il - k0
  const V3<T> lepst{T(leps[0]), T(leps[1]), T(leps[2])};
  acc.ldme3 = acc.ldme3 + lepst;
  qrot_delta_vjp(eg, k.d, lepst, leg, acc.ld);
  acc.lphi = acc.lphi + p.il * V3<T>{T(leps[3]), T(leps[4]), T(leps[5])};
  if (xg > T(0)) acc.lepair = qadd(acc.lepair, leg);
  else if (xg < T(0)) acc.lepair = qadd(acc.lepair, qconj(leg));
}

// Reverse of the prefix from the summed Gauss-point adjoints: adjoints of
// the end translations and rotations; the section adjoints are copied.
template <class T>
DL_HD void elem_vjp_suffix(const ElemIn<T> &in, const ElemPrefix<T> &p, const ElemGpAdj<T> &acc, ElemAdjOut &out) {
  for (int q = 0; q < 6; ++q) out.lC[q] = acc.lC[q];
  out.lec[0] = acc.lec[0];
  out.lec[1] = acc.lec[1];
  // epair = qexp(smax phi)
  const V3<T> lphi = acc.lphi + p.smax * qexp_vjp(p.smax * p.k.phi, acc.lepair);
  // d = cvt(dd), dme3 = dd - e3, phiP = cvt(pp), qr = cvt(Lr), phi = qlog(cvt(qIJ))
  V3<double> ldd = cvt<double>(acc.ld) + cvt<double>(acc.ldme3);
  V3<double> lpp = cvt<double>(acc.lppT);
  Q4<double> lLr = cvtq<double>(acc.lqr);
  Q4<double> lqIJ = cvtq<double>(qlog_vjp(p.qIJt, lphi));
  // dd = qrot(conj(Lr), pp)
  Q4<double> lcLr = qzero<double>();
  qrot_vjp(qconj(p.Lr), p.pp, ldd, lcLr, lpp);
  lLr = qadd(lLr, qconj(lcLr));
  // pp = invL0 (xj - xi)
  out.lxj = in.invL0 * lpp;
  out.lxi = (-in.invL0) * lpp;
  // Lr = LI qh
  Q4<double> lLI = qzero<double>(), lqh = qzero<double>();
  qmul_vjp(p.LI, p.qh, lLr, lLI, lqh);
  // qh = qhalf(qIJ)
  lqIJ = qadd(lqIJ, qhalf_vjp(p.qIJ, lqh));
  if (p.flip) lqIJ = qscale(-1.0, lqIJ);
  // qIJ = conj(LI) LJ (before the flip)
  Q4<double> lcLI = qzero<double>(), lLJ = qzero<double>();
  qmul_vjp(qconj(p.LI), p.LJ, lqIJ, lcLI, lLJ);
  lLI = qadd(lLI, qconj(lcLI));
  // L = R qN
  Q4<double> lRi = qzero<double>(), lRj = qzero<double>(), dummy = qzero<double>();
  qmul_vjp(in.Ri, in.qNi, lLI, lRi, dummy);
  qmul_vjp(in.Rj, in.qNj, lLJ, lRj, dummy);
  out.lthi = rot_tangent(in.Ri, lRi);
  out.lthj = rot_tangent(in.Rj, lRj);
}

// Element VJP.  lf: adjoint of the end forces; lh: on entry the adjoint of the
// history after the step, on exit that of the history before it (plastic);
// ldiss[g]: adjoint of the dissipation increment of Gauss point g.
template <class T, class Y, class M>
DL_HD void elem_vjp(const M &mdl, const PlastLaw<T> &law, const ElemIn<T> &in, const double lf[12],
                    ElemHistAdj *lh, const double ldiss[kAdjMaxG], ElemAdjOut &out) {
  ElemPrefix<T> p;
  elem_vjp_prefix(in, p);
  ElemGpAdj<T> acc;
  gp_adj_zero(acc);
  for (int g = 0; g < in.G; ++g) {
    GpIn<T> gi;
    GpHistAdj gh;
    for (int q = 0; q < 3; ++q) {
      gi.g0[q] = in.g0[g][q];
      gi.k0[q] = in.k0[g][q];
    }
    for (int q = 0; q < 6; ++q) {
      gi.ep[q] = in.ep[g][q];
      gi.epsc[q] = in.epsc[g][q];
      gh.ep[q] = lh->ep[g][q];
      gh.epsc[q] = lh->epsc[g][q];
    }
    for (int a = 0; a < in.nh; ++a) {
      gi.al[a] = in.al[g][a];
      gh.al[a] = lh->al[g][a];
    }
    elem_vjp_gp<T, Y>(mdl, law, in, p, g, gi, lf, &gh, ldiss[g], acc);
    for (int q = 0; q < 6; ++q) {
      lh->ep[g][q] = gh.ep[q];
      lh->epsc[g][q] = gh.epsc[q];
    }
    for (int a = 0; a < in.nh; ++a) lh->al[g][a] = gh.al[a];
  }
  elem_vjp_suffix(in, p, acc, out);
}

// ---------------------------------------------------------------------------
// node: pure forward and VJP
// ---------------------------------------------------------------------------
struct NodeIn {
  V3<double> x;
  Q4<double> R;
  double v[6];
  double mass;          // translational mass
  Q4<double> P;         // principal frame of the rotational inertia S = P D P^T
  double D[3];
  unsigned mask;        // Dirichlet (acceleration) bits 0..5
  double aPre[6];       // prescribed accelerations of the masked DOFs
  double fx[6];         // external load
  int gyro;
  double dt;
};

// Inverse of the free block of M (rows/columns whose bit is clear in rmask),
// zero in the constrained rows/columns.  The constrained rows/columns are
// replaced by identity rows/columns first, so one 3x3 cofactor inverse with
// fixed indices serves every constraint pattern (no indexed local arrays).
DL_HD void inv_free_block(const double M[3][3], unsigned rmask, double Mi[3][3]) {
  double A[3][3];
  for (int i = 0; i < 3; ++i)
    for (int j = 0; j < 3; ++j) {
      const bool fi = !(rmask & (1u << i)), fj = !(rmask & (1u << j));
      A[i][j] = (fi && fj) ? M[i][j] : (i == j ? 1.0 : 0.0);
    }
  const double c00 = A[1][1] * A[2][2] - A[1][2] * A[2][1];
  const double c01 = A[1][2] * A[2][0] - A[1][0] * A[2][2];
  const double c02 = A[1][0] * A[2][1] - A[1][1] * A[2][0];
  const double id = 1.0 / (A[0][0] * c00 + A[0][1] * c01 + A[0][2] * c02);
  double B[3][3];
  B[0][0] = c00 * id;
  B[0][1] = (A[0][2] * A[2][1] - A[0][1] * A[2][2]) * id;
  B[0][2] = (A[0][1] * A[1][2] - A[0][2] * A[1][1]) * id;
  B[1][0] = c01 * id;
  B[1][1] = (A[0][0] * A[2][2] - A[0][2] * A[2][0]) * id;
  B[1][2] = (A[0][2] * A[1][0] - A[0][0] * A[1][2]) * id;
  B[2][0] = c02 * id;
  B[2][1] = (A[0][1] * A[2][0] - A[0][0] * A[2][1]) * id;
  B[2][2] = (A[0][0] * A[1][1] - A[0][1] * A[1][0]) * id;
  for (int i = 0; i < 3; ++i)
    for (int j = 0; j < 3; ++j) {
      const bool fi = !(rmask & (1u << i)), fj = !(rmask & (1u << j));
      Mi[i][j] = (fi && fj) ? B[i][j] : 0.0;
    }
}

DL_HD void node_mass_matrix(Q4<double> R, Q4<double> P, const double D[3], double M[3][3]) {
  double Rm[3][3];
  qmat(qmul(R, P), Rm);
  for (int i = 0; i < 3; ++i)
    for (int j = 0; j < 3; ++j)
      M[i][j] = Rm[i][0] * D[0] * Rm[j][0] + Rm[i][1] * D[1] * Rm[j][1] + Rm[i][2] * D[2] * Rm[j][2];
}

// Node forward (pure, matrix form of node_update with R <- exp(dt omega) R).
// fint: summed element end forces.  Outputs x, R, v after the step.
DL_HD void node_forward(const NodeIn &in, const double fint[6], V3<double> &xo, Q4<double> &Ro, double vo[6]) {
  double r[6], a[6];
  for (int k = 0; k < 6; ++k) {
    r[k] = in.fx[k] - fint[k];
    a[k] = in.aPre[k];
  }
  double M[3][3];
  node_mass_matrix(in.R, in.P, in.D, M);
  const V3<double> w0{in.v[3], in.v[4], in.v[5]};
  if (in.gyro) {
    const V3<double> gy = cross(w0, m3_mul(M, w0));
    r[3] -= gy.x;
    r[4] -= gy.y;
    r[5] -= gy.z;
  }
  for (int k = 0; k < 3; ++k)
    if (!(in.mask & (1u << k))) a[k] = r[k] / in.mass;
  const unsigned rm = (in.mask >> 3) & 7u;
  if (rm != 7u) {
    double b[3] = {r[3], r[4], r[5]};
    for (int i = 0; i < 3; ++i)
      if (!(rm & (1u << i)))
        for (int j = 0; j < 3; ++j)
          if (rm & (1u << j)) b[i] -= M[i][j] * a[3 + j];
    double Mi[3][3];
    inv_free_block(M, rm, Mi);
    for (int i = 0; i < 3; ++i)
      if (!(rm & (1u << i))) a[3 + i] = Mi[i][0] * b[0] + Mi[i][1] * b[1] + Mi[i][2] * b[2];
  }
  for (int k = 0; k < 6; ++k) vo[k] = in.v[k] + in.dt * a[k];
  xo = in.x + in.dt * V3<double>{vo[0], vo[1], vo[2]};
  Ro = qnormalize(qmul(qexp_small(in.dt * V3<double>{vo[3], vo[4], vo[5]}), in.R));
}

// Node VJP.  Inputs: the node state before the step (in), the velocity after
// it (v1), the adjoints of x, R (tangent), v after the step (lx1, lth1, lv1) and
// an extra adjoint of the internal force (lfseed, e.g. from an objective).
// Outputs: adjoints of x, R, v before the step, of the internal force (lf),
// of the mass (lmass) and of the inertia S in the reference frame (lS,
// symmetric, packed xx yy zz xy xz yz).
DL_HD void node_vjp(const NodeIn &in, const double v1[6], V3<double> lx1, V3<double> lth1, const double lv1_in[6],
                    const double lfseed[6], V3<double> &lx0, V3<double> &lth0, double lv0[6], double lf[6],
                    double &lmass, double lS[6]) {
  const double dt = in.dt;
  double lv1[6];
  for (int k = 0; k < 6; ++k) lv1[k] = lv1_in[k];
  // x1 = x0 + dt v1
  lx0 = lx1;
  lv1[0] += dt * lx1.x;
  lv1[1] += dt * lx1.y;
  lv1[2] += dt * lx1.z;
  // R1 = exp(dt w1) R0: mu0 = Q^T mu1, lw1 += dt J_l(dt w1)^T mu1
  const V3<double> w1{v1[3], v1[4], v1[5]};
  const V3<double> phi = dt * w1;
  const Q4<double> Q = qexp_small(phi);
  lth0 = qrot(qconj(Q), lth1);
  const V3<double> lphi = jl_t(phi, lth1);
  lv1[3] += dt * lphi.x;
  lv1[4] += dt * lphi.y;
  lv1[5] += dt * lphi.z;
  // v1 = v0 + dt a
  double la[6];
  for (int k = 0; k < 6; ++k) {
    lv0[k] = lv1[k];
    la[k] = (in.mask & (1u << k)) ? 0.0 : dt * lv1[k];
  }
  // accelerations of the step (constrained components are prescribed)
  double a[6];
  for (int k = 0; k < 6; ++k) a[k] = (in.mask & (1u << k)) ? in.aPre[k] : (v1[k] - in.v[k]) / dt;
  // translations: a = (fx - f) / m
  lmass = 0.0;
  for (int k = 0; k < 3; ++k) {
    lf[k] = -la[k] / in.mass + lfseed[k];
    lmass -= la[k] * a[k] / in.mass;
  }
  // rotations: M_ff a_f = r_f - M_fc a_c, r = fx - f - w0 x (M w0)
  double M[3][3], Mi[3][3];
  node_mass_matrix(in.R, in.P, in.D, M);
  const unsigned rm = (in.mask >> 3) & 7u;
  inv_free_block(M, rm, Mi);
  const V3<double> lal{la[3], la[4], la[5]};
  const V3<double> lr = m3_tmul(Mi, lal);  // zero in constrained rows
  lf[3] = -lr.x + lfseed[3];
  lf[4] = -lr.y + lfseed[4];
  lf[5] = -lr.z + lfseed[5];
  // dJ = sum G_ij dM_ij with G = -lr a^T (+ (w0 x lr) w0^T with the gyroscopic term)
  const V3<double> w0{in.v[3], in.v[4], in.v[5]};
  const V3<double> arot{a[3], a[4], a[5]};
  double Gm[3][3];
  const double lra[3] = {lr.x, lr.y, lr.z}, av[3] = {arot.x, arot.y, arot.z};
  for (int i = 0; i < 3; ++i)
    for (int j = 0; j < 3; ++j) Gm[i][j] = -lra[i] * av[j];
  if (in.gyro) {
    const V3<double> Mw = m3_mul(M, w0);
    const V3<double> wxl = cross(w0, lr);
    // r -= w0 x (M w0):  lw0 += lr x (M w0) + M (w0 x lr)
    const V3<double> lw = cross(lr, Mw) + m3_mul(M, wxl);
    lv0[3] += lw.x;
    lv0[4] += lw.y;
    lv0[5] += lw.z;
    const double wv[3] = {w0.x, w0.y, w0.z}, xl[3] = {wxl.x, wxl.y, wxl.z};
    for (int i = 0; i < 3; ++i)
      for (int j = 0; j < 3; ++j) Gm[i][j] += xl[i] * wv[j];
  }
  // M = R S R^T:  dM = [dth] M - M [dth] + R dS R^T
  double B[3][3];
  for (int i = 0; i < 3; ++i)
    for (int j = 0; j < 3; ++j) {
      double s = 0.0;
      for (int q = 0; q < 3; ++q) s += M[i][q] * Gm[j][q] - Gm[q][i] * M[q][j];
      B[i][j] = s;
    }
  lth0 = lth0 + V3<double>{B[1][2] - B[2][1], B[2][0] - B[0][2], B[0][1] - B[1][0]};
  double Rm[3][3], X[3][3];
  qmat(in.R, Rm);
  for (int i = 0; i < 3; ++i)
    for (int j = 0; j < 3; ++j) {
      double s = 0.0;
      for (int p = 0; p < 3; ++p)
        for (int q = 0; q < 3; ++q) s += Rm[p][i] * Gm[p][q] * Rm[q][j];
      X[i][j] = s;
    }
  lS[0] = X[0][0];
  lS[1] = X[1][1];
  lS[2] = X[2][2];
  lS[3] = 0.5 * (X[0][1] + X[1][0]);
  lS[4] = 0.5 * (X[0][2] + X[2][0]);
  lS[5] = 0.5 * (X[1][2] + X[2][1]);
}

}  // namespace dl
