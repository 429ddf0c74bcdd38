// Rod--rod penalty contact of one candidate element pair, restating the force
// path of RodContactModel (src/models/RodContactModel.cpp): closest points of
// the two lines (findClosestPoints_, :953-991), node projection
// (getClosestPoint_, :996-1026), the branch structure of computeContacts_
// (:451-738: segment-to-segment, one-sided and speculative node-to-segment,
// including the one-sided branch's projection of node iA of element B,
// :575), segment-to-segment penalty (computeSTS_, :1031-1152, force part) and
// node-to-segment penalty (computeNTS_, :1157-1208, force part).  FP64.
// Shared by the step kernels (device) and the host set-up (blacklist).
#pragma once

#include "rodkin.cuh"

namespace dl {

struct PairGeom {
  double A[2][3], B[2][3];
};

DL_HD double c_dot(const double *a, const double *b) { return a[0] * b[0] + a[1] * b[1] + a[2] * b[2]; }

DL_HD void c_closest(const PairGeom &g, double &uA, double &uB) {
  double d[3], tA[3], tB[3];
  for (int k = 0; k < 3; ++k) {
    d[k] = (g.B[1][k] + g.B[0][k]) - (g.A[1][k] + g.A[0][k]);
    tA[k] = g.A[1][k] - g.A[0][k];
    tB[k] = g.B[1][k] - g.B[0][k];
  }
  const double tAA = c_dot(tA, tA), tBB = c_dot(tB, tB), tAB = c_dot(tB, tA);
  double vA[3], vB[3];
  for (int k = 0; k < 3; ++k) {
    vA[k] = tB[k] * tAB - tA[k] * tBB;
    vB[k] = tA[k] * tAB - tB[k] * tAA;
  }
  const double den = tBB * tAA - tAB * tAB;
  uA = -1.0 * c_dot(d, vA) / den;
  uB = +1.0 * c_dot(d, vB) / den;
}

DL_HD double c_project(const double *S, const double M[2][3]) {
  double bM[3], tM[3];
  for (int k = 0; k < 3; ++k) {
    bM[k] = M[1][k] + M[0][k];
    tM[k] = M[1][k] - M[0][k];
  }
  return (2.0 * c_dot(S, tM) - c_dot(tM, bM)) / c_dot(tM, tM);
}

DL_HD bool c_contains(double u) { return u >= -1.0 && u <= 1.0; }

DL_HD void c_point(const double P[2][3], double u, double out[3]) {
  const double n0 = 0.5 * (1.0 - u), n1 = 0.5 * (1.0 + u);
  for (int k = 0; k < 3; ++k) out[k] = n0 * P[0][k] + n1 * P[1][k];
}

// STS: forces f[12] on (A0, A1, B0, B1)
DL_HD bool c_sts(double kp, double r, const PairGeom &g, double uA, double uB, double *f, double &gap) {
  double pA[3], pB[3], d[3];
  c_point(g.A, uA, pA);
  c_point(g.B, uB, pB);
  for (int c = 0; c < 3; ++c) d[c] = pB[c] - pA[c];
  const double dist = sqrt(c_dot(d, d));
  if (!(dist > 0.0)) return false;
  if (dist > 2.0 * r) return false;
  gap = dist - 2.0 * r;
  if (f) {
    const double NA0 = 0.5 * (1.0 - uA), NA1 = 0.5 * (1.0 + uA), NB0 = 0.5 * (1.0 - uB), NB1 = 0.5 * (1.0 + uB);
    for (int c = 0; c < 3; ++c) {
      const double s = kp * gap * (d[c] / dist);
      f[0 + c] -= NA0 * s;
      f[3 + c] -= NA1 * s;
      f[6 + c] += NB0 * s;
      f[9 + c] += NB1 * s;
    }
  }
  return true;
}

// NTS: slave node S against master segment M at uM; forces on (S, M0, M1)
DL_HD bool c_nts(double kp, double r, const double *S, const double M[2][3], double uM, double *fs, double *fm0,
                 double *fm1, double &gap) {
  double pM[3], d[3];
  c_point(M, uM, pM);
  for (int c = 0; c < 3; ++c) d[c] = pM[c] - S[c];
  const double dist = sqrt(c_dot(d, d));
  if (!(dist > 0.0)) return false;
  if (dist > 2.0 * r) return false;
  gap = dist - 2.0 * r;
  if (fs) {
    for (int c = 0; c < 3; ++c) {
      const double n = (S[c] - pM[c]) / dist;
      fs[c] += kp * gap * n;
      fm0[c] += kp * gap * (-0.5 * (1.0 - uM) * n);
      fm1[c] += kp * gap * (-0.5 * (1.0 + uM) * n);
    }
  }
  return true;
}

// One candidate pair (same nodes / blacklist already excluded).  Returns
// whether the contact is closed; adds forces to f[12] (A0, A1, B0, B1) when
// f != nullptr; gap = smallest distance - 2r of the closed evaluations;
// energy += 1/2 k gap^2 per closed evaluation.
DL_HD bool pair_contact(const PairGeom &g, double r, double ks, double kn, double *f, double &gapOut,
                        double &energy) {
  double uA = 0.0, uB = 0.0, gap = 0.0;
  c_closest(g, uA, uB);
  bool closed = false;
  gapOut = 0.0;
  if (c_contains(uA) && c_contains(uB)) {
    closed = c_sts(ks, r, g, uA, uB, f, gap);
    if (closed) {
      gapOut = gap;
      energy += 0.5 * ks * gap * gap;
    }
    return closed;
  }
  if (!c_contains(uA) && c_contains(uB)) {
    const int iA = (uA < -1.0) ? 0 : 1;
    uB = c_project(g.B[iA], g.A);  // the reference projects node iA of element B here
    if (!c_contains(uB)) return false;
    closed = c_nts(kn, r, g.A[iA], g.B, uB, f ? f + 3 * iA : nullptr, f ? f + 6 : nullptr, f ? f + 9 : nullptr, gap);
    if (closed) {
      gapOut = gap;
      energy += 0.5 * kn * gap * gap;
    }
    return closed;
  }
  if (!c_contains(uB) && c_contains(uA)) {
    const int iB = (uB < -1.0) ? 0 : 1;
    uA = c_project(g.B[iB], g.A);
    if (!c_contains(uA)) return false;
    closed = c_nts(kn, r, g.B[iB], g.A, uA, f ? f + 6 + 3 * iB : nullptr, f ? f : nullptr, f ? f + 3 : nullptr, gap);
    if (closed) {
      gapOut = gap;
      energy += 0.5 * kn * gap * gap;
    }
    return closed;
  }
  // speculative node-to-segment: both ends of A against B, then of B against A
  bool first = true;
  for (int iA = 0; iA < 2; ++iA) {
    const double u = c_project(g.A[iA], g.B);
    if (!c_contains(u)) continue;
    if (c_nts(kn, r, g.A[iA], g.B, u, f ? f + 3 * iA : nullptr, f ? f + 6 : nullptr, f ? f + 9 : nullptr, gap)) {
      closed = true;
      energy += 0.5 * kn * gap * gap;
      if (first || gap < gapOut) gapOut = gap;
      first = false;
    }
  }
  for (int iB = 0; iB < 2; ++iB) {
    const double u = c_project(g.B[iB], g.A);
    if (!c_contains(u)) continue;
    if (c_nts(kn, r, g.B[iB], g.A, u, f ? f + 6 + 3 * iB : nullptr, f ? f : nullptr, f ? f + 3 : nullptr, gap)) {
      closed = true;
      energy += 0.5 * kn * gap * gap;
      if (first || gap < gapOut) gapOut = gap;
      first = false;
    }
  }
  return closed;
}

// Distance between two segments (clamped closest points), for the candidate
// list: pairs further apart than 2r + margin cannot close before a rebuild.
DL_HD double segment_distance(const PairGeom &g) {
  double d1[3], d2[3], r0[3];
  for (int k = 0; k < 3; ++k) {
    d1[k] = g.A[1][k] - g.A[0][k];
    d2[k] = g.B[1][k] - g.B[0][k];
    r0[k] = g.A[0][k] - g.B[0][k];
  }
  const double a = c_dot(d1, d1), e = c_dot(d2, d2), f = c_dot(d2, r0);
  double s = 0.0, t = 0.0;
  const double c = c_dot(d1, r0), b = c_dot(d1, d2);
  const double den = a * e - b * b;
  if (den > 1e-300) {
    s = (b * f - c * e) / den;
    s = s < 0.0 ? 0.0 : (s > 1.0 ? 1.0 : s);
  }
  t = (b * s + f) / e;
  if (t < 0.0) {
    t = 0.0;
    s = -c / a;
    s = s < 0.0 ? 0.0 : (s > 1.0 ? 1.0 : s);
  } else if (t > 1.0) {
    t = 1.0;
    s = (b - c) / a;
    s = s < 0.0 ? 0.0 : (s > 1.0 ? 1.0 : s);
  }
  double dd[3];
  for (int k = 0; k < 3; ++k) dd[k] = (g.A[0][k] + d1[k] * s) - (g.B[0][k] + d2[k] * t);
  return sqrt(c_dot(dd, dd));
}

}  // namespace dl
