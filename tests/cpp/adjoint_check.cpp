// Host build of the adjoint building blocks (dynlattice_b200/csrc/adjoint.cuh)
// for finite-difference checks from Python.  Compiled by the tests with the
// yield policy that the engine generates for the model (dl_yield_source with
// host = 1), included as "yield_policy.inc".  T is double or float (-DACT=...).
#include <cmath>
#include <cstring>

#include "adjoint.cuh"

#ifndef ACT
#define ACT double
#endif

namespace dl {
#include "yield_policy.inc"
}

using namespace dl;
using T = ACT;

namespace {
struct Cfg {
  double qNi[4], qNj[4], invL0, L0;
  T g0[kAdjMaxG][3], k0[kAdjMaxG][3];
  int G, nh, plastic;
  T H[7][7];
  int max_iter;
  T prec;
} cfg;
struct Dummy {} mdl;

// packed differentiable inputs: xi 3, xj 3, Ri 4, Rj 4, C 6, ec 2,
// ep G*6, al G*nh, epsc G*6
ElemIn<T> unpack(const double *p) {
  ElemIn<T> in;
  in.xi = V3<double>{p[0], p[1], p[2]};
  in.xj = V3<double>{p[3], p[4], p[5]};
  in.Ri = Q4<double>{p[6], p[7], p[8], p[9]};
  in.Rj = Q4<double>{p[10], p[11], p[12], p[13]};
  for (int k = 0; k < 6; ++k) in.C[k] = T(p[14 + k]);
  in.ec[0] = T(p[20]);
  in.ec[1] = T(p[21]);
  int o = 22;
  for (int g = 0; g < cfg.G; ++g)
    for (int k = 0; k < 6; ++k) in.ep[g][k] = T(p[o++]);
  for (int g = 0; g < cfg.G; ++g)
    for (int a = 0; a < cfg.nh; ++a) in.al[g][a] = T(p[o++]);
  for (int g = 0; g < cfg.G; ++g)
    for (int k = 0; k < 6; ++k) in.epsc[g][k] = T(p[o++]);
  in.qNi = Q4<double>{cfg.qNi[0], cfg.qNi[1], cfg.qNi[2], cfg.qNi[3]};
  in.qNj = Q4<double>{cfg.qNj[0], cfg.qNj[1], cfg.qNj[2], cfg.qNj[3]};
  in.invL0 = cfg.invL0;
  in.L0 = cfg.L0;
  in.G = cfg.G;
  in.nh = cfg.nh;
  in.plastic = cfg.plastic;
  for (int g = 0; g < cfg.G; ++g)
    for (int k = 0; k < 3; ++k) {
      in.g0[g][k] = cfg.g0[g][k];
      in.k0[g][k] = cfg.k0[g][k];
    }
  return in;
}
PlastLaw<T> law() { return PlastLaw<T>{cfg.H, cfg.max_iter, cfg.prec}; }
}  // namespace

extern "C" {

int ac_setup(const double *qNi, const double *qNj, double invL0, double L0, const double *g0, const double *k0,
             int G, int nh, int plastic, const double *H, int max_iter, double prec) {
  std::memcpy(cfg.qNi, qNi, sizeof cfg.qNi);
  std::memcpy(cfg.qNj, qNj, sizeof cfg.qNj);
  cfg.invL0 = invL0;
  cfg.L0 = L0;
  cfg.G = G;
  cfg.nh = nh;
  cfg.plastic = plastic;
  for (int g = 0; g < G; ++g)
    for (int k = 0; k < 3; ++k) {
      cfg.g0[g][k] = T(g0[g * 3 + k]);
      cfg.k0[g][k] = T(k0[g * 3 + k]);
    }
  for (int i = 0; i < 7; ++i)
    for (int j = 0; j < 7; ++j) cfg.H[i][j] = T(H ? H[i * 7 + j] : 0.0);
  cfg.max_iter = max_iter;
  cfg.prec = T(prec);
  return 0;
}

// f[12]; hist: ep G*6, al G*nh, epsc G*6, dediss G
int ac_elem_forward(const double *p, double *f, double *hist) {
  ElemIn<T> in = unpack(p);
  T ff[12];
  ElemHist<T> h;
  bool ovf = false;
  elem_forward<T, YieldAdj>(mdl, law(), in, ff, &h, &ovf);
  for (int k = 0; k < 12; ++k) f[k] = double(ff[k]);
  int o = 0;
  for (int g = 0; g < cfg.G; ++g)
    for (int k = 0; k < 6; ++k) hist[o++] = cfg.plastic ? double(h.ep[g][k]) : 0.0;
  for (int g = 0; g < cfg.G; ++g)
    for (int a = 0; a < cfg.nh; ++a) hist[o++] = cfg.plastic ? double(h.al[g][a]) : 0.0;
  for (int g = 0; g < cfg.G; ++g)
    for (int k = 0; k < 6; ++k) hist[o++] = cfg.plastic ? double(h.epsc[g][k]) : 0.0;
  for (int g = 0; g < cfg.G; ++g) hist[o++] = h.dediss[g];
  return ovf ? 1 : 0;
}

// out: lxi 3, lxj 3, lthi 3, lthj 3, lC 6, lec 2, lep G*6, lal G*nh, lepsc G*6
int ac_elem_vjp(const double *p, const double *lf, const double *lhist, double *out) {
  ElemIn<T> in = unpack(p);
  ElemHistAdj lh;
  double ldiss[kAdjMaxG];
  int o = 0;
  for (int g = 0; g < cfg.G; ++g)
    for (int k = 0; k < 6; ++k) lh.ep[g][k] = lhist[o++];
  for (int g = 0; g < cfg.G; ++g)
    for (int a = 0; a < cfg.nh; ++a) lh.al[g][a] = lhist[o++];
  for (int g = 0; g < cfg.G; ++g)
    for (int k = 0; k < 6; ++k) lh.epsc[g][k] = lhist[o++];
  for (int g = 0; g < cfg.G; ++g) ldiss[g] = lhist[o++];
  ElemAdjOut r;
  elem_vjp<T, YieldAdj>(mdl, law(), in, lf, &lh, ldiss, r);
  const V3<double> v[4] = {r.lxi, r.lxj, r.lthi, r.lthj};
  o = 0;
  for (int i = 0; i < 4; ++i) {
    out[o++] = v[i].x;
    out[o++] = v[i].y;
    out[o++] = v[i].z;
  }
  for (int k = 0; k < 6; ++k) out[o++] = r.lC[k];
  out[o++] = r.lec[0];
  out[o++] = r.lec[1];
  for (int g = 0; g < cfg.G; ++g)
    for (int k = 0; k < 6; ++k) out[o++] = cfg.plastic ? lh.ep[g][k] : 0.0;
  for (int g = 0; g < cfg.G; ++g)
    for (int a = 0; a < cfg.nh; ++a) out[o++] = cfg.plastic ? lh.al[g][a] : 0.0;
  for (int g = 0; g < cfg.G; ++g)
    for (int k = 0; k < 6; ++k) out[o++] = cfg.plastic ? lh.epsc[g][k] : 0.0;
  return 0;
}

// node: p = x 3, R 4, v 6, fint 6, mass, P 4, D 3; cfgi = mask, gyro; dt
static NodeIn node_unpack(const double *p, const double *aPre, const double *fx, int mask, int gyro, double dt) {
  NodeIn in;
  in.x = V3<double>{p[0], p[1], p[2]};
  in.R = Q4<double>{p[3], p[4], p[5], p[6]};
  for (int k = 0; k < 6; ++k) in.v[k] = p[7 + k];
  in.mass = p[19];
  in.P = Q4<double>{p[20], p[21], p[22], p[23]};
  for (int k = 0; k < 3; ++k) in.D[k] = p[24 + k];
  in.mask = static_cast<unsigned>(mask);
  for (int k = 0; k < 6; ++k) {
    in.aPre[k] = aPre[k];
    in.fx[k] = fx[k];
  }
  in.gyro = gyro;
  in.dt = dt;
  return in;
}

// out: x 3, R 4, v 6
int ac_node_forward(const double *p, const double *aPre, const double *fx, int mask, int gyro, double dt,
                    double *out) {
  NodeIn in = node_unpack(p, aPre, fx, mask, gyro, dt);
  V3<double> xo;
  Q4<double> Ro;
  double vo[6];
  node_forward(in, p + 13, xo, Ro, vo);
  out[0] = xo.x; out[1] = xo.y; out[2] = xo.z;
  out[3] = Ro.w; out[4] = Ro.x; out[5] = Ro.y; out[6] = Ro.z;
  for (int k = 0; k < 6; ++k) out[7 + k] = vo[k];
  return 0;
}

// adj = lx1 3, lth1 3, lv1 6, lfseed 6; out = lx0 3, lth0 3, lv0 6, lf 6, lmass, lS 6
int ac_node_vjp(const double *p, const double *aPre, const double *fx, int mask, int gyro, double dt,
                const double *adj, double *out) {
  NodeIn in = node_unpack(p, aPre, fx, mask, gyro, dt);
  V3<double> xo;
  Q4<double> Ro;
  double v1[6];
  node_forward(in, p + 13, xo, Ro, v1);
  V3<double> lx0, lth0;
  double lv0[6], lf[6], lm, lS[6];
  node_vjp(in, v1, V3<double>{adj[0], adj[1], adj[2]}, V3<double>{adj[3], adj[4], adj[5]}, adj + 6, adj + 12, lx0,
           lth0, lv0, lf, lm, lS);
  out[0] = lx0.x; out[1] = lx0.y; out[2] = lx0.z;
  out[3] = lth0.x; out[4] = lth0.y; out[5] = lth0.z;
  for (int k = 0; k < 6; ++k) {
    out[6 + k] = lv0[k];
    out[12 + k] = lf[k];
  }
  out[18] = lm;
  for (int k = 0; k < 6; ++k) out[19 + k] = lS[k];
  return 0;
}

// yield policy: f, grad and vjp at args
int ac_yield(const double *args, int nargs, int ngrad, double *fout, double *gout, double lf, const double *lg,
             double *la) {
  T a[32], g[16], lgt[16], lat[32];
  for (int i = 0; i < nargs; ++i) a[i] = T(args[i]);
  *fout = double(YieldAdj::f(mdl, a));
  YieldAdj::grad(mdl, a, g);
  for (int k = 0; k < ngrad; ++k) {
    gout[k] = double(g[k]);
    lgt[k] = T(lg[k]);
  }
  for (int i = 0; i < nargs; ++i) lat[i] = T(0);
  YieldAdj::vjp(mdl, a, T(lf), lgt, lat);
  for (int i = 0; i < nargs; ++i) la[i] = double(lat[i]);
  return 0;
}
}
