// Device code of one explicit step, shared by the ahead-of-time build
// (kernels.cu, nvcc) and the runtime-compiled elastoplastic kernels (NVRTC,
// jit.cpp); contains no host code and no standard headers.
//
// One explicit step (LeapFrogModule::solve, LeapFrogModule.cpp:44-84, with
// ExplicitModule::getForce/getAcce/updateVec, ExplicitModule.cpp:339-419) is
// two phases over HBM-resident structure-of-arrays data:
//   element phase: per element, gather the two node states, evaluate the rod
//     kinematics, strains, stress resultants (elastic or cutting-plane return
//     map with history commit) and write the two end-force vectors;
//   node phase: per node, sum its incident end forces in a fixed order (CSR),
//     add loads, solve the node-block mass (translational scalar, rotational
//     R P D P^T R^T) with acceleration constraints, and update v, x and the
//     rotation quaternion by the exponential map.
// The persistent kernel runs many steps in one cooperative launch with a
// bounded grid barrier between the phases; k_element/k_node launch one phase
// each (stream mode).  Kernels are templated on the element precision T and on
// the yield-function policy Y.
#pragma once

#include "contact.cuh"
#include "devtypes.cuh"
#include "rodkin.cuh"

namespace dl {

constexpr double kDblEpsilon = 2.220446049250313e-16;  // DBL_EPSILON

// Gauss points/weights of Gauss1..Gauss3 on [-1, 1] (ascending)
__constant__ double c_gxi[3][3] = {{0.0, 0.0, 0.0},
                                   {-0.57735026918962576451, 0.57735026918962576451, 0.0},
                                   {-0.77459666924148337704, 0.0, 0.77459666924148337704}};
__constant__ double c_gw[3][3] = {{2.0, 0.0, 0.0},
                                  {1.0, 1.0, 0.0},
                                  {0.55555555555555555556, 0.88888888888888888889,
                                   0.55555555555555555556}};

// ---------------------------------------------------------------------------
// expression interpreter (programs from expr.cpp; uniform control flow)
// ---------------------------------------------------------------------------
__device__ __forceinline__ float x_pow(float a, float b) { return powf(a, b); }
__device__ __forceinline__ double x_pow(double a, double b) { return pow(a, b); }
__device__ __forceinline__ float x_fmod(float a, float b) { return fmodf(a, b); }
__device__ __forceinline__ double x_fmod(double a, double b) { return fmod(a, b); }

template <class T>
__device__ __forceinline__ void run_prog(const DevProg<T> &p, const T *args, T *r) {
  for (int i = 0; i < p.n_ops; ++i) {
    const ExprOp o = p.ops[i];
    const T a = r[o.a], b = r[o.b], c = r[o.c];
    T v;
    switch (o.op) {
      case XO_CONST: v = p.consts[o.a | (o.b << 8)]; break;
      case XO_ARG: v = args[o.a]; break;
      case XO_ADD: v = a + b; break;
      case XO_SUB: v = a - b; break;
      case XO_MUL: v = a * b; break;
      case XO_DIV: v = a / b; break;
      case XO_POW: v = x_pow(a, b); break;
      case XO_SQUARE: v = a * a; break;
      case XO_NEG: v = -a; break;
      case XO_ABS: v = fabs(a); break;
      case XO_SQRT: v = sqrt(a); break;
      case XO_EXP: v = exp(a); break;
      case XO_LOG: v = log(a); break;
      case XO_SIN: v = sin(a); break;
      case XO_COS: v = cos(a); break;
      case XO_TAN: v = tan(a); break;
      case XO_ATAN: v = atan(a); break;
      case XO_FLOOR: v = floor(a); break;
      case XO_CEIL: v = ceil(a); break;
      case XO_SIGN: v = T((a > T(0)) - (a < T(0))); break;
      case XO_MIN: v = a < b ? a : b; break;
      case XO_MAX: v = a > b ? a : b; break;
      case XO_MOD: v = x_fmod(a, b); break;
      case XO_LT: v = a < b ? T(1) : T(0); break;
      case XO_LE: v = a <= b ? T(1) : T(0); break;
      case XO_GT: v = a > b ? T(1) : T(0); break;
      case XO_GE: v = a >= b ? T(1) : T(0); break;
      case XO_EQ: v = a == b ? T(1) : T(0); break;
      case XO_NE: v = a != b ? T(1) : T(0); break;
      case XO_AND: v = (a != T(0) && b != T(0)) ? T(1) : T(0); break;
      case XO_OR: v = (a != T(0) || b != T(0)) ? T(1) : T(0); break;
      case XO_NOT: v = a == T(0) ? T(1) : T(0); break;
      case XO_SELECT: v = a != T(0) ? b : c; break;
      default: v = T(0); break;
    }
    r[o.dst] = v;
  }
}


// Yield-function policy of the ahead-of-time build: interprets the compiled
// register program (expr.cpp).  The runtime-compiled build replaces it with
// straight-line code generated from the same expressions (YieldJit).
struct YieldInterp {
  static constexpr bool kPlastic = true;
  static constexpr int kNh = -1;  // hardening count known only at run time
  static constexpr int kMinBlocks = 1;
  template <class T>
  __device__ static __forceinline__ T f(const DevModel<T> &m, const T *args, T *regs) {
    run_prog(m.yield, args, regs);
    return regs[m.yield.out0];
  }
  template <class T>
  __device__ static __forceinline__ void grad(const DevModel<T> &m, const T *args, T *gr, T *regs) {
    run_prog(m.grad, args, regs);
    for (int k = 0; k < 6 + m.nh; ++k) gr[k] = regs[m.grad.outs[k]];
  }
};

// Policy of elastic lattices: no return map is compiled in.
struct ElasticOnly {
  static constexpr bool kPlastic = false;
  static constexpr int kNh = 0;
  static constexpr int kMinBlocks = 2;
  template <class T>
  __device__ static __forceinline__ T f(const DevModel<T> &, const T *, T *) {
    return T(0);
  }
  template <class T>
  __device__ static __forceinline__ void grad(const DevModel<T> &, const T *, T *, T *) {}
};

// ---------------------------------------------------------------------------
// loads/stores
// ---------------------------------------------------------------------------
// Node state and end forces written in the other phase of the same persistent
// launch are read with plain (L1-cacheable) loads: the grid barrier's
// gpu-scope acquire makes the other blocks' writes visible, as for a
// cooperative-groups grid synchronisation.
__device__ __forceinline__ Q4<double> ldq(const double4 *p) {
  const double4 v = *p;
  return Q4<double>{v.x, v.y, v.z, v.w};
}
__device__ __forceinline__ V3<double> ldx(const double4 *p) {
  const double4 v = *p;
  return V3<double>{v.x, v.y, v.z};
}
__device__ __forceinline__ Q4<double> toq(float4 v) { return Q4<double>{v.x, v.y, v.z, v.w}; }
__device__ __forceinline__ Q4<double> toq(double4 v) { return Q4<double>{v.x, v.y, v.z, v.w}; }

// one end-force record (6 values) into its node-ordered slot
__device__ __forceinline__ void store_end(float *p, const float *f) {
  float2 *q = reinterpret_cast<float2 *>(p);
  q[0] = make_float2(f[0], f[1]);
  q[1] = make_float2(f[2], f[3]);
  q[2] = make_float2(f[4], f[5]);
}
__device__ __forceinline__ void store_end(double *p, const double *f) {
  double2 *q = reinterpret_cast<double2 *>(p);
  q[0] = make_double2(f[0], f[1]);
  q[1] = make_double2(f[2], f[3]);
  q[2] = make_double2(f[4], f[5]);
}
__device__ __forceinline__ void load_end(const float *p, double f[6]) {
  const float2 *q = reinterpret_cast<const float2 *>(p);
  const float2 a = q[0], b = q[1], c = q[2];
  f[0] += a.x; f[1] += a.y; f[2] += b.x; f[3] += b.y; f[4] += c.x; f[5] += c.y;
}
__device__ __forceinline__ void load_end(const double *p, double f[6]) {
  const double2 *q = reinterpret_cast<const double2 *>(p);
  const double2 a = q[0], b = q[1], c = q[2];
  f[0] += a.x; f[1] += a.y; f[2] += b.x; f[3] += b.y; f[4] += c.x; f[5] += c.y;
}

template <class T>
__device__ __forceinline__ double block_sum(double v) {
  __shared__ double s_part[32];
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  __syncthreads();
  if (lane == 0) s_part[w] = v;
  __syncthreads();
  double r = 0.0;
  if (threadIdx.x < 32) {
    r = (threadIdx.x < (blockDim.x + 31) / 32) ? s_part[threadIdx.x] : 0.0;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) r += __shfl_down_sync(0xffffffffu, r, o);
  }
  return r;  // valid in thread 0
}

// ---------------------------------------------------------------------------
// element phase
// ---------------------------------------------------------------------------
struct ElemEnergy {
  double pot = 0.0, diss = 0.0;
};

// Out-of-line paths that plain runs do not take (contact, plates, group
// output): kept out of the step kernels' register budget.

struct NodeExtra {
  double f[3];
  double energy;
};

// rod--rod contact force of this step (then cleared for the next one) and
// the rigid plates' node--plane penalty
template <class T>
__device__ __noinline__ NodeExtra node_contact(const DevModel<T> &m, int n, int64_t step, double xx, double xy,
                                               double xz, bool energy, bool last, bool walk) {
  NodeExtra o{{0.0, 0.0, 0.0}, 0.0};
  // the node's ends of closed pairs, in the index's fixed order; walked only
  // when a pair of the node closed in this step (walk: its stamp)
  if (walk && m.c_ptr)
    for (uint32_t i = m.c_ptr[n]; i < m.c_ptr[n + 1]; ++i) {
      const int v = m.c_ent[i];
      if (!m.pclosed[v >> 2]) continue;
      const double *f = m.pforce + static_cast<size_t>(v >> 2) * 12 + (v & 3) * 3;
      o.f[0] += f[0];
      o.f[1] += f[1];
      o.f[2] += f[2];
    }
  if (walk && m.j_ptr)
    for (uint32_t i = m.j_ptr[n]; i < m.j_ptr[n + 1]; ++i) {
      const int v = m.j_ent[i];
      if (!m.jclosed[v >> 1]) continue;
      const double *f = m.jforce + static_cast<size_t>(v >> 1) * 6 + (v & 1) * 3;
      o.f[0] += f[0];
      o.f[1] += f[1];
      o.f[2] += f[2];
    }
  for (int pl = 0; pl < m.n_plates; ++pl) {
    const double tk = m.t0 + static_cast<double>(step - m.tstep0) * m.dt;
    const double g = (xx - (m.plate_p0[pl][0] + m.plate_v[pl][0] * tk)) * m.plate_n[pl][0] +
                     (xy - (m.plate_p0[pl][1] + m.plate_v[pl][1] * tk)) * m.plate_n[pl][1] +
                     (xz - (m.plate_p0[pl][2] + m.plate_v[pl][2] * tk)) * m.plate_n[pl][2] - m.c_radius;
    if (g < 0.0) {
      const double kg = m.plate_k[pl] * g;
      for (int c2 = 0; c2 < 3; ++c2) o.f[c2] += kg * m.plate_n[pl][c2];
      if (energy) o.energy += 0.5 * kg * g;
      if (last)
        for (int c2 = 0; c2 < 3; ++c2) atomicAdd(m.plate_force + pl * 3 + c2, kg * m.plate_n[pl][c2]);
    }
  }
  return o;
}

template <class T>
__device__ __noinline__ void store_fint_last(const DevModel<T> &m, int n, double f0, double f1, double f2, double f3,
                                             double f4, double f5) {
  const int N = m.N;
  m.fint_last[n] = f0;
  m.fint_last[N + n] = f1;
  m.fint_last[2 * N + n] = f2;
  m.fint_last[3 * N + n] = f3;
  m.fint_last[4 * N + n] = f4;
  m.fint_last[5 * N + n] = f5;
}

// Stress resultants at one Gauss point: ElasticRodMaterial::getStress
// (ElasticRodMaterial.cpp:369-373) or the cutting-plane return map of
// ElastoPlasticRodMaterial::getStress (ElastoPlasticRodMaterial.cpp:198-269)
// followed by the commit of ElastoPlasticRodMaterial::applyDeform (:271-307).
// History modes of the material update: HM_COMMIT (explicit step: return map,
// history committed in place; with commit = false the elastic predictor
// only), HM_TRIAL (return map from the committed history, nothing written)
// and HM_STORE (return map, the resulting history written to HistOut: the
// predictor-corrector's trial that is committed once its step is accepted).
enum { HM_COMMIT = 0, HM_TRIAL = 1, HM_STORE = 2 };
template <class T>
struct HistOut {
  T *ep, *alpha, *epsc;  // layouts of DevModel::ep, alpha, epsc
  double *ediss;
};

// EN: every step of the launch reports energies (known at compile time):
// the point's dissipated energy is then loaded before the iterations, so
// that its latency overlaps them instead of ending the element's chain.
template <class T, class Y, bool X, int HM = HM_COMMIT, bool EN = false>
__device__ __forceinline__ void material(const DevModel<T> &m, int e, int g, const T eps[6],
                                         const T Cd[6], T sig[6], bool commit, bool energy,
                                         double wgt, ElemEnergy &en, int64_t tslot = -1,
                                         const HistOut<T> *ho = nullptr, int64_t bslot = -1) {
  const int E = m.E;
  if (!Y::kPlastic || !m.plastic) {
#pragma unroll
    for (int k = 0; k < 6; ++k) sig[k] = Cd[k] * eps[k];
    if (energy) {
      double s = 0.0;
#pragma unroll
      for (int k = 0; k < 6; ++k) s += double(eps[k]) * double(sig[k]);
      en.pot += wgt * 0.5 * s;
    }
    return;
  }
  // hardening count: a compile-time constant in the specialised kernels, so
  // that all history arrays below live in registers
  constexpr int NHC = Y::kNh;
  const int nh = NHC >= 0 ? NHC : m.nh;
  constexpr int NHMAX = NHC >= 0 ? NHC : 7;
  T ep[6], ep0[6], al[NHMAX > 0 ? NHMAX : 1];
#pragma unroll
  for (int k = 0; k < 6; ++k) ep0[k] = ep[k] = m.ep[(g * 6 + k) * E + e];
#pragma unroll
  for (int a = 0; a < NHMAX; ++a)
    if (a < nh) al[a] = m.alpha[(g * nh + a) * E + e];
  T args[16];
  args[6 + nh] = m.ec[e];
  args[7 + nh] = m.ec[E + e];
  constexpr bool ed_early = HM == HM_COMMIT && EN;
  const double ed_in = ed_early ? m.ediss[g * E + e] : 0.0;
  T regs[kMaxExprRegs];
  T dflow = T(0);
  int it = 0;
  // branch tape of a differentiated run: the iteration count to impose
  size_t bidx = 0;
  int it_imposed = -1;
  if (X && HM == HM_COMMIT && m.br && bslot >= 0) {
    bidx = (static_cast<size_t>(bslot) * m.G + g) * E + e;
    if (m.br_mode == 2) it_imposed = m.br[bidx];
  }
  for (;;) {
#pragma unroll
    for (int k = 0; k < 6; ++k) sig[k] = Cd[k] * (eps[k] - ep[k]);
    if (HM == HM_COMMIT && !commit) break;
#pragma unroll
    for (int a = 0; a < NHMAX; ++a) {
      if (a >= nh) break;
      T s = T(0);
#pragma unroll
      for (int b = 0; b < NHMAX; ++b)
        if (b < nh) s += m.H[a][b] * al[b];
      args[6 + a] = -s;
    }
#pragma unroll
    for (int k = 0; k < 6; ++k) args[k] = sig[k];
    const T fv = Y::f(m, args, regs);
    if (!(it < m.max_iter)) {
      atomicOr(m.err, 0x1u);
      break;
    }
    if (X && it_imposed >= 0 ? it >= it_imposed : fv < m.prec) break;
    T gr[13];
    Y::grad(m, args, gr, regs);
    T den = T(0);
#pragma unroll
    for (int k = 0; k < 6; ++k) den += gr[k] * Cd[k] * gr[k];
#pragma unroll
    for (int a = 0; a < NHMAX; ++a) {
      if (a >= nh) break;
      T s = T(0);
#pragma unroll
      for (int b = 0; b < NHMAX; ++b)
        if (b < nh) s += m.H[a][b] * gr[6 + b];
      den += gr[6 + a] * s;
    }
    const T ddf = fv / den;
#pragma unroll
    for (int k = 0; k < 6; ++k) ep[k] += ddf * gr[k];
#pragma unroll
    for (int a = 0; a < NHMAX; ++a)
      if (a < nh) al[a] += ddf * gr[6 + a];
    dflow += ddf;
    ++it;
  }
  if (HM == HM_COMMIT && !commit) return;
  if (HM == HM_TRIAL) return;
  if (X && HM == HM_COMMIT && m.br && bslot >= 0 && m.br_mode == 1) m.br[bidx] = static_cast<uint8_t>(it < 255 ? it : 255);
  // applyDeform: dissipation with the previous committed total strain
  double dd = 0.0;
  if (fabs(double(dflow)) > kDblEpsilon) {
#pragma unroll
    for (int k = 0; k < 6; ++k) {
      const T eold = m.epsc[(g * 6 + k) * E + e];
      const double so = double(Cd[k]) * double(eold - ep0[k]);
      dd += (so + double(sig[k])) / 2.0 * double(ep[k] - ep0[k]);
    }
    if (HM == HM_COMMIT) {
      if (ed_early) m.ediss[g * E + e] = ed_in + dd;
      else m.ediss[g * E + e] += dd;
    }
  }
  if (HM == HM_STORE) {
    const double ed = m.ediss[g * E + e] + dd;
    ho->ediss[g * E + e] = ed;
#pragma unroll
    for (int k = 0; k < 6; ++k) {
      ho->ep[(g * 6 + k) * E + e] = ep[k];
      ho->epsc[(g * 6 + k) * E + e] = eps[k];
    }
#pragma unroll
    for (int a = 0; a < NHMAX; ++a)
      if (a < nh) ho->alpha[(g * nh + a) * E + e] = al[a];
    if (energy) {
      double s = 0.0;
#pragma unroll
      for (int k = 0; k < 6; ++k) s += double(eps[k] - ep[k]) * double(sig[k]);
      en.pot += wgt * 0.5 * s;
      en.diss += wgt * ed;
    }
    return;
  }
  if (it > 0) {
#pragma unroll
    for (int k = 0; k < 6; ++k) m.ep[(g * 6 + k) * E + e] = ep[k];
#pragma unroll
    for (int a = 0; a < NHMAX; ++a)
      if (a < nh) m.alpha[(g * nh + a) * E + e] = al[a];
  }
#pragma unroll
  for (int k = 0; k < 6; ++k) m.epsc[(g * 6 + k) * E + e] = eps[k];
  if (X && m.tp_ep && tslot >= 0) {  // adjoint recomputation: history after this step
    const size_t o6 = static_cast<size_t>(tslot) * m.G * 6 * E, oh = static_cast<size_t>(tslot) * m.G * nh * E;
#pragma unroll
    for (int k = 0; k < 6; ++k) {
      m.tp_ep[o6 + (g * 6 + k) * E + e] = ep[k];
      m.tp_epsc[o6 + (g * 6 + k) * E + e] = eps[k];
    }
#pragma unroll
    for (int a = 0; a < NHMAX; ++a)
      if (a < nh) m.tp_al[oh + (g * nh + a) * E + e] = al[a];
  }
  if (energy) {
    double s = 0.0;
#pragma unroll
    for (int k = 0; k < 6; ++k) s += double(eps[k] - ep[k]) * double(sig[k]);
    en.pot += wgt * 0.5 * s;
    en.diss += wgt * (ed_early ? ed_in + dd : m.ediss[g * E + e]);
  }
}

// Internal force of one element (SpecialCosseratRodModel::assemble_,
// SpecialCosseratRodModel.cpp:899-949, with Line3D::getXi, Line3D.cpp:141-162):
//   f_n += w [ N'_n n ; N'_n m - N_n phi' x n ],  n = Lambda sigma_n, m = Lambda sigma_m.
// Gauss point g of an element: strain, stress resultants (with the history
// update of the history mode) and its contribution to the two end forces
// (SpecialCosseratRodModel::assemble_, SpecialCosseratRodModel.cpp:899-949,
// with Line3D::getXi, Line3D.cpp:141-162):
//   f_n += w [ N'_n n ; N'_n m - N_n phi' x n ],  n = Lambda sigma_n, m = Lambda sigma_m.
template <class T, class Y, bool X, int HM, bool EN = false>
__device__ __forceinline__ void gp_force(const DevModel<T> &m, int e, int g, int G, const ElemKin<T> &k,
                                         const Q4<T> &epair, T il, double L0, const T Cd[6], bool commit,
                                         bool energy, ElemEnergy &en, int64_t tslot, const HistOut<T> *ho,
                                         T f[12], int64_t bslot = -1) {
  const int E = m.E;
  const T xg = T(c_gxi[G - 1][g]);
  const T Wg = T(c_gw[G - 1][g]);
  const Q4<T> eg = xg > T(0) ? epair : (xg < T(0) ? qconj(epair) : Q4<T>{T(1), T(0), T(0), T(0)});
  T g0[3], k0[3];
#pragma unroll
  for (int q = 0; q < 3; ++q) {
    g0[q] = m.g0[(g * 3 + q) * E + e];
    k0[q] = m.k0[(g * 3 + q) * E + e];
  }
  T eps[6];
  Q4<T> qg;
  gp_strain_e(k, eg, il, g0, k0, eps, &qg);
  T sig[6];
  const double wgt = c_gw[G - 1][g] * 0.5 * L0;
  material<T, Y, X, HM, EN>(m, e, g, eps, Cd, sig, commit, energy, wgt, en, tslot, ho, bslot);
  const V3<T> nn = qrot(qg, V3<T>{sig[0], sig[1], sig[2]});
  const V3<T> mm = qrot(qg, V3<T>{sig[3], sig[4], sig[5]});
  const V3<T> pxn = cross(k.phiP, nn);
  const T hw = T(0.5) * Wg;                      // w N'_J = W/2
  const T wI = T(wgt) * (T(0.5) * (T(1) - xg));  // w N_I
  const T wJ = T(wgt) * (T(0.5) * (T(1) + xg));  // w N_J
  f[0] -= hw * nn.x; f[1] -= hw * nn.y; f[2] -= hw * nn.z;
  f[3] += -hw * mm.x - wI * pxn.x;
  f[4] += -hw * mm.y - wI * pxn.y;
  f[5] += -hw * mm.z - wI * pxn.z;
  f[6] += hw * nn.x; f[7] += hw * nn.y; f[8] += hw * nn.z;
  f[9] += hw * mm.x - wJ * pxn.x;
  f[10] += hw * mm.y - wJ * pxn.y;
  f[11] += hw * mm.z - wJ * pxn.z;
}

// The gathered end states, kinematics and section constants of element e.
template <class T>
struct ElemPre {
  int2 slot;
  ElemKin<T> k;
  T il;
  double L0;
  T Cd[6];
};
template <class T>
__device__ __forceinline__ void elem_pre(const DevModel<T> &m, int e, const double4 *P, const double4 *Q,
                                         ElemPre<T> &p) {
  const int E = m.E;
  const int2 c = m.conn[e];
  p.slot = m.eslot[e];
  const V3<double> xi = ldx(P + c.x), xj = ldx(P + c.y);
  const Q4<double> Ri = ldq(Q + c.x), Rj = ldq(Q + c.y);
  const Q4<double> qNi = toq(m.qN[e]), qNj = toq(m.qN[E + e]);
  const double invL0 = m.invL0[e];
  p.k = elem_kin<T>(xi, xj, Ri, Rj, qNi, qNj, invL0);
  p.il = T(invL0);
  p.L0 = double(m.L0[e]);
#pragma unroll
  for (int q = 0; q < 6; ++q) p.Cd[q] = m.C[q * E + e];
}

// Elements of 3 or 4 nodes: node positions, the reference rotation and the
// local rotation vectors (gathered from P/Q, the node state to use), and per
// Gauss point the strains minus the reference values (in T), with the point's
// weight and shape data.
struct ElemPreN {
  V3<double> x[kMaxElemNodes];
  Q4<double> Lr;
  V3<double> psi[kMaxElemNodes];
};
template <class T>
__device__ __forceinline__ void elem_pre_n(const DevModel<T> &m, int e, const double4 *P, const double4 *Q,
                                           ElemPreN &p) {
  const int E = m.E, n = m.nen;
  Q4<double> L[kMaxElemNodes];
  for (int a = 0; a < n; ++a) {
    const int nd = m.conn_n[a * E + e];
    p.x[a] = ldx(P + nd);
    L[a] = qmul(ldq(Q + nd), toq(m.qN[a * E + e]));
  }
  line_ref(L, n, p.Lr, p.psi);
}
template <class T>
__device__ __forceinline__ GpKinN gp_eps_n(const DevModel<T> &m, int e, int g, const ElemPreN &p, T eps[6],
                                           double &w, double N[kMaxElemNodes], double dN[kMaxElemNodes]) {
  const int E = m.E, n = m.nen;
  const double *sh = m.shp + (static_cast<size_t>(e) * m.G + g) * (n + 1);
  w = sh[0];
  for (int a = 0; a < n; ++a) {
    N[a] = m.Nq[a][g];
    dN[a] = sh[1 + a];
  }
  const GpKinN k = gp_kin_n(p.x, p.Lr, p.psi, n, N, dN);
  const double *s0 = m.s0_n + static_cast<size_t>(g) * 6 * E + e;
  eps[0] = T(k.gme3.x - s0[0]);
  eps[1] = T(k.gme3.y - s0[E]);
  eps[2] = T(k.gme3.z - s0[2 * E]);
  eps[3] = T(k.K.x - s0[3 * E]);
  eps[4] = T(k.K.y - s0[4 * E]);
  eps[5] = T(k.K.z - s0[5 * E]);
  return k;
}

// Internal force of an element of 3 or 4 nodes (SpecialCosseratRodModel::
// getStrains_/assemble_, SpecialCosseratRodModel.cpp:694-744, 899-949, with
// Line3D, Line3D.cpp:117-273): kinematics in FP64 (gp_kin_n), material and
// end forces in T,
//   f_a += w [ N_a' n ; N_a' m - N_a phi' x n ],  n = Lambda sigma_n, m = Lambda sigma_m.
// Out of line, so that the kernels' two-node paths keep their register
// allocation.  P/Q: the node positions and rotations to use.
template <class T, class Y, bool X, int HM>
__device__ __noinline__ void element_force_n(const DevModel<T> &m, int e, bool commit, bool energy,
                                             ElemEnergy &en, int64_t tslot, const double4 *P, const double4 *Q,
                                             const HistOut<T> *ho, int64_t bslot) {
  const int E = m.E, n = m.nen, G = m.G;
  ElemPreN p;
  elem_pre_n(m, e, P, Q, p);
  T Cd[6];
  for (int q = 0; q < 6; ++q) Cd[q] = m.C[q * E + e];
  T f[kMaxElemNodes][6];
  for (int a = 0; a < n; ++a)
    for (int q = 0; q < 6; ++q) f[a][q] = T(0);
  for (int g = 0; g < G; ++g) {
    T eps[6];
    double w, N[kMaxElemNodes], dN[kMaxElemNodes];
    const GpKinN k = gp_eps_n(m, e, g, p, eps, w, N, dN);
    T sig[6];
    material<T, Y, X, HM>(m, e, g, eps, Cd, sig, commit, energy, w, en, tslot, ho, bslot);
    const Q4<T> qg = cvtq<T>(k.L);
    const V3<T> nn = qrot(qg, V3<T>{sig[0], sig[1], sig[2]});
    const V3<T> mm = qrot(qg, V3<T>{sig[3], sig[4], sig[5]});
    const V3<T> pxn = cross(cvt<T>(k.phiP), nn);
    for (int a = 0; a < n; ++a) {
      const T wg = T(w * dN[a]), wn = T(w * N[a]);
      f[a][0] += wg * nn.x;
      f[a][1] += wg * nn.y;
      f[a][2] += wg * nn.z;
      f[a][3] += wg * mm.x - wn * pxn.x;
      f[a][4] += wg * mm.y - wn * pxn.y;
      f[a][5] += wg * mm.z - wn * pxn.z;
    }
  }
  for (int a = 0; a < n; ++a) store_end(m.ef + static_cast<size_t>(m.eslot_n[a * E + e]) * 6, f[a]);
}

// Internal force of one element: the end states, kinematics and the sum of
// its Gauss points' contributions into the two node-ordered end slots.
// HM != HM_COMMIT (predictor-corrector): the node state is read from pos/rot
// and the history is handled as material() describes.
// GC: the Gauss-point count when known at compile time (0: m.G); with a
// constant count the point loop unrolls and the points' independent
// strain/stress chains interleave.
template <class T, class Y, bool X, int HM = HM_COMMIT, int GC = 0, bool EN = false>
__device__ __forceinline__ void element_force(const DevModel<T> &m, int e, bool commit,
                                              bool energy, ElemEnergy &en, bool lat_energy_step = false,
                                              int64_t tslot = -1, const double4 *pos = nullptr,
                                              const double4 *rot = nullptr, const HistOut<T> *ho = nullptr,
                                              int64_t bslot = -1) {
  // elements of 3 or 4 nodes (no batches: no per-lattice energies); compiled
  // into the extended kernels and the predictor-corrector's history modes
  // only: the plain step kernels never see them (the launch picks the
  // extended variant), and a call site would cost them registers
  if (GC == 0 && (X || HM != HM_COMMIT) && m.nen > 2) {
    element_force_n<T, Y, X, HM>(m, e, commit, energy, en, tslot, HM == HM_COMMIT ? m.pos : pos,
                                 HM == HM_COMMIT ? m.rot : rot, ho, bslot);
    return;
  }
  const double pot0 = en.pot, diss0 = en.diss;
  ElemPre<T> p;
  elem_pre(m, e, HM == HM_COMMIT ? m.pos : pos, HM == HM_COMMIT ? m.rot : rot, p);
  T f[12];
#pragma unroll
  for (int q = 0; q < 12; ++q) f[q] = T(0);
  const int G = GC > 0 ? GC : m.G;
  // exp(-xi phi/2) of the largest positive Gauss abscissa; its conjugate serves -xi
  const Q4<T> epair = qexp((T(-0.5) * T(c_gxi[G - 1][G - 1])) * p.k.phi);
  if (GC == 2) {
    // each point from zero, then their sum: the same operations as the
    // half-element path, so both give the same bits
    T f1[12];
#pragma unroll
    for (int q = 0; q < 12; ++q) f1[q] = T(0);
    gp_force<T, Y, X, HM, EN>(m, e, 0, 2, p.k, epair, p.il, p.L0, p.Cd, commit, energy, en, tslot, ho, f, bslot);
    gp_force<T, Y, X, HM, EN>(m, e, 1, 2, p.k, epair, p.il, p.L0, p.Cd, commit, energy, en, tslot, ho, f1, bslot);
#pragma unroll
    for (int q = 0; q < 12; ++q) f[q] += f1[q];
  } else {
    for (int g = 0; g < G; ++g)
      gp_force<T, Y, X, HM, EN>(m, e, g, G, p.k, epair, p.il, p.L0, p.Cd, commit, energy, en, tslot, ho, f, bslot);
  }
  store_end(m.ef + static_cast<size_t>(p.slot.x) * 6, f);
  store_end(m.ef + static_cast<size_t>(p.slot.y) * 6, f + 6);
  if (energy && lat_energy_step && m.lat_energy) {
    atomicAdd(m.lat_energy + m.elat[e] * 5 + 1, en.pot - pot0);
    atomicAdd(m.lat_energy + m.elat[e] * 5 + 2, en.diss - diss0);
  }
}

// Half of a two-point element on one lane of an adjacent lane pair: both
// lanes gather the end states and form the kinematics, each lane evaluates
// Gauss point g = lane (the same instructions, so the pair does not
// diverge), the pair sums its end forces by shuffles and each lane writes one
// end slot.  Explicit step only (history committed in place).
template <class T, class Y, bool EN = false>
__device__ __forceinline__ void element_force_half(const DevModel<T> &m, int e, int lane, bool energy,
                                                   ElemEnergy &en, bool lat_energy_step) {
  const double pot0 = en.pot, diss0 = en.diss;
  ElemPre<T> p;
  elem_pre(m, e, m.pos, m.rot, p);
  T f[12];
#pragma unroll
  for (int q = 0; q < 12; ++q) f[q] = T(0);
  const Q4<T> epair = qexp((T(-0.5) * T(c_gxi[1][1])) * p.k.phi);
  gp_force<T, Y, false, HM_COMMIT, EN>(m, e, lane, 2, p.k, epair, p.il, p.L0, p.Cd, true, energy, en, -1, nullptr, f);
  const unsigned pm = 3u << ((threadIdx.x & 31) & ~1u);
#pragma unroll
  for (int q = 0; q < 12; ++q) f[q] += __shfl_xor_sync(pm, f[q], 1);
  T mine[6];  // selected, not indexed by the lane: f stays in registers
#pragma unroll
  for (int q = 0; q < 6; ++q) mine[q] = lane ? f[6 + q] : f[q];
  store_end(m.ef + static_cast<size_t>(lane ? p.slot.y : p.slot.x) * 6, mine);
  if (energy && lat_energy_step && m.lat_energy) {
    atomicAdd(m.lat_energy + m.elat[e] * 5 + 1, en.pot - pot0);
    atomicAdd(m.lat_energy + m.elat[e] * 5 + 2, en.diss - diss0);
  }
}

// Contact of one candidate pair at the positions of the step's start; its
// closed flag and node forces go to the pair's slots, which the node phase
// sums per node in a fixed order (internal force, translations only:
// RodContactModel adds its contributions to fint, RodContactModel.cpp:709).
template <class T>
__device__ __noinline__ void contact_pair(const DevModel<T> &m, int p, int64_t step, bool energy, double &econ) {
  const int4 q = m.c_quad[p];  // the end nodes directly: one dependent load less than pair -> elements -> nodes
  PairGeom g;
  const double4 a0 = m.pos[q.x], a1 = m.pos[q.y], b0 = m.pos[q.z], b1 = m.pos[q.w];
  g.A[0][0] = a0.x; g.A[0][1] = a0.y; g.A[0][2] = a0.z;
  g.A[1][0] = a1.x; g.A[1][1] = a1.y; g.A[1][2] = a1.z;
  g.B[0][0] = b0.x; g.B[0][1] = b0.y; g.B[0][2] = b0.z;
  g.B[1][0] = b1.x; g.B[1][1] = b1.y; g.B[1][2] = b1.z;
  double f[12];
#pragma unroll
  for (int k = 0; k < 12; ++k) f[k] = 0.0;
  double gap = 0.0, en = 0.0;
  // every closed evaluation of pair_contact (segment to segment, node to
  // segment) has two points of the segments within 2r: a pair whose segments
  // are further apart (with a margin far above the distance's rounding) is
  // open, and its branch logic is skipped
  const bool apart = segment_distance(g) > 2.0 * m.c_radius * (1.0 + 1e-6);
  const bool closed = !apart && pair_contact(g, m.c_radius, m.c_ks, m.c_kn, f, gap, en);
  if (energy) {
    econ += en;
    m.pair_gap[p] = closed ? gap : 1e300;
  }
  m.pclosed[p] = closed ? 1 : 0;
  if (!closed) return;
  if (m.cstamp) m.cstamp[q.x] = m.cstamp[q.y] = m.cstamp[q.z] = m.cstamp[q.w] = step;
  double *o = m.pforce + static_cast<size_t>(p) * 12;
#pragma unroll
  for (int k = 0; k < 12; ++k) o[k] = f[k];
}

// Joint contact of one candidate pair at the positions of the step's start
// (JointContactModel::computeContact_, JointContactModel.cpp:318-340): with
// n = (x_B - x_A)/d, f_int(A) -= k (2r - d) n and f_int(B) += k (2r - d) n
// when d <= 2r; its energy is -k (2r - d)^2 / 2.  No force at d = 0.
template <class T>
__device__ __noinline__ void joint_pair(const DevModel<T> &m, int p, int64_t step, bool energy, double &econ) {
  const int2 pr = m.jpairs[p];
  const double4 a = m.pos[pr.x], b = m.pos[pr.y];
  const double dx = b.x - a.x, dy = b.y - a.y, dz = b.z - a.z;
  const double d = sqrt(dx * dx + dy * dy + dz * dz);
  const double r2 = 2.0 * m.j_radius;
  const bool closed = d <= r2;
  if (energy) m.jpair_gap[p] = closed ? d - r2 : 1e300;
  const double g = r2 - d;
  if (closed && energy) econ -= 0.5 * m.j_k * g * g;
  const bool force = closed && d > 0.0;
  m.jclosed[p] = force ? 1 : 0;
  if (!force) return;
  if (m.cstamp) m.cstamp[pr.x] = m.cstamp[pr.y] = step;
  const double s = m.j_k * g / d;
  double *o = m.jforce + static_cast<size_t>(p) * 6;
  o[0] = -s * dx;
  o[1] = -s * dy;
  o[2] = -s * dz;
  o[3] = s * dx;
  o[4] = s * dy;
  o[5] = s * dz;
}

// ---------------------------------------------------------------------------
// node phase
// ---------------------------------------------------------------------------
struct NodeOut {
  double ekin = 0.0;
  double wext = 0.0;
  double econtact = 0.0;
  int64_t last_step = -1;
};

__device__ __forceinline__ double scale_of(const double *scales, int n_scales, int64_t row, int s) {
  return s < 0 ? 1.0 : scales[row * n_scales + s];
}

// masked solve of M a = r for the free components (constrained ones preset in a);
// out of line: only nodes with partially constrained rotations call it
static __device__ __noinline__ void solve3_masked(const double M[3][3], const double r[3], double a[3],
                                              unsigned mask) {
  int fr[3], nf = 0;
  for (int i = 0; i < 3; ++i)
    if (!(mask & (1u << i))) fr[nf++] = i;
  if (nf == 0) return;
  double A[3][3], b[3];
  for (int i = 0; i < nf; ++i) {
    b[i] = r[fr[i]];
    for (int j = 0; j < 3; ++j)
      if (mask & (1u << j)) b[i] -= M[fr[i]][j] * a[j];
    for (int j = 0; j < nf; ++j) A[i][j] = M[fr[i]][fr[j]];
  }
  if (nf == 1) {
    a[fr[0]] = b[0] / A[0][0];
  } else if (nf == 2) {
    const double det = A[0][0] * A[1][1] - A[0][1] * A[1][0];
    a[fr[0]] = (b[0] * A[1][1] - A[0][1] * b[1]) / det;
    a[fr[1]] = (A[0][0] * b[1] - A[1][0] * b[0]) / det;
  } else {
    const double c00 = A[1][1] * A[2][2] - A[1][2] * A[2][1];
    const double c01 = A[1][2] * A[2][0] - A[1][0] * A[2][2];
    const double c02 = A[1][0] * A[2][1] - A[1][1] * A[2][0];
    const double det = A[0][0] * c00 + A[0][1] * c01 + A[0][2] * c02;
    const double id = 1.0 / det;
    const double inv[3][3] = {
        {c00 * id, (A[0][2] * A[2][1] - A[0][1] * A[2][2]) * id, (A[0][1] * A[1][2] - A[0][2] * A[1][1]) * id},
        {c01 * id, (A[0][0] * A[2][2] - A[0][2] * A[2][0]) * id, (A[0][2] * A[1][0] - A[0][0] * A[1][2]) * id},
        {c02 * id, (A[0][1] * A[2][0] - A[0][0] * A[2][1]) * id, (A[0][0] * A[1][1] - A[0][1] * A[1][0]) * id}};
    for (int i = 0; i < 3; ++i) a[fr[i]] = inv[i][0] * b[0] + inv[i][1] * b[1] + inv[i][2] * b[2];
  }
}

template <class T, bool X, bool EN = false>
__device__ __forceinline__ void node_update(const DevModel<T> &m, int n, int64_t step, bool energy,
                                            const SampleSpec &smp, int64_t sidx, NodeOut &out) {
  const int N = m.N;
  // independent loads first (node state and constants), then the slot run
  double v[6];
#pragma unroll
  for (int k = 0; k < 6; ++k) v[k] = m.vel[k * N + n];
  const Q4<double> R = ldq(m.rot + n);
  V3<double> x = ldx(m.pos + n);
  const Q4<double> P = toq(m.iframe[n]);
  const auto Dv = m.idiag[n];
  const auto Di = m.idinv[n];
  const double im = m.imass[n];
  const double mn = EN ? m.mass[n] : 0.0;  // E_kin on every step (EN): loaded with the state
  const int i0 = m.slot_ptr[n], i1 = m.slot_ptr[n + 1];
  const int b0 = m.bc_ptr[n], b1 = m.bc_ptr[n + 1];
  // the step of the node's last closed contact pair (rod or joint contact)
  const int64_t cst = (X && m.cstamp) ? m.cstamp[n] : step;
  if (X && m.xbuild) {  // the candidate lists cover motion up to half the margin
    const double dx = x.x - m.xbuild[3 * n], dy = x.y - m.xbuild[3 * n + 1], dz = x.z - m.xbuild[3 * n + 2];
    if (dx * dx + dy * dy + dz * dz > m.half_margin * m.half_margin) atomicOr(m.err, 0x20u);
  }
  double f[6] = {0, 0, 0, 0, 0, 0};
  // a node of a rigid tie group (the HingeModel's constraints, condensed):
  // the group's end forces and contact summed over its members in the
  // group's fixed order, so that every member computes the same update; the
  // first member (the master) records the group's energies
  int t0 = 0, t1 = 0;
  if (X && m.tie_ptr) {
    t0 = m.tie_ptr[n];
    t1 = m.tie_ptr[n + 1];
  }
  const bool rec = !(X && t1 > t0) || m.tie_nodes[t0] == n;
  if (X && t1 > t0) {
    for (int t = t0; t < t1; ++t) {
      const int q = m.tie_nodes[t];
      for (int i = m.slot_ptr[q]; i < m.slot_ptr[q + 1]; ++i) load_end(m.ef + static_cast<size_t>(i) * 6, f);
      if (m.c_ptr || m.j_ptr || m.n_plates) {
        const NodeExtra ex = node_contact(m, q, step, x.x, x.y, x.z, energy && rec, rec && step == out.last_step,
                                          !m.cstamp || m.cstamp[q] == step);
        f[0] += ex.f[0];
        f[1] += ex.f[1];
        f[2] += ex.f[2];
        if (rec) out.econtact += ex.energy;
      }
    }
  } else {
    for (int i = i0; i < i1; ++i) load_end(m.ef + static_cast<size_t>(i) * 6, f);
    if (X && (m.c_ptr || m.j_ptr || m.n_plates)) {
      const NodeExtra ex = node_contact(m, n, step, x.x, x.y, x.z, energy, step == out.last_step, cst == step);
      f[0] += ex.f[0];
      f[1] += ex.f[1];
      f[2] += ex.f[2];
      out.econtact += ex.energy;
    }
  }
  if (X && m.grp_hist && m.grp_flag[n]) atomicAdd(m.grp_hist + (step - m.grp_step0), f[m.grp_dof]);
  // boundary conditions at this step (scale table row)
  double fx[6] = {0, 0, 0, 0, 0, 0};
  double a[6] = {0, 0, 0, 0, 0, 0};
  unsigned mask = 0u;
  const int64_t row = step - m.scale_step0;
  bool loaded = false;
  for (int b = b0; b < b1; ++b) {
    const BcTerm t = m.bc[b];
    const double val = t.factor * scale_of(m.scales, m.n_scales, row, t.scale);
    // compare-and-select over the six DOFs keeps fx/a in registers
#pragma unroll
    for (int k = 0; k < 6; ++k) {
      if (t.dof != k) continue;
      if (t.kind == BCD_NEUMANN) {
        fx[k] += val;
      } else {
        a[k] = val;
      }
    }
    if (t.kind == BCD_NEUMANN) loaded = true;
    else mask |= 1u << t.dof;
  }
  double r[6];
#pragma unroll
  for (int k = 0; k < 6; ++k) r[k] = fx[k] - f[k];
  // rotational inertia M = R P D P^T R^T with R the current rotation
  const double D[3] = {double(Dv.x), double(Dv.y), double(Dv.z)};
  const double Dinv[3] = {double(Di.x), double(Di.y), double(Di.z)};
  const Q4<double> RP = qmul(R, P);
  const Q4<double> RPc = qconj(RP);
  const V3<double> w0{v[3], v[4], v[5]};
  if (m.gyro) {  // SpecialCosseratRodModel::assembleGyro_ (:951-967): omega x (M omega)
    V3<double> wl = qrot(RPc, w0);
    V3<double> Mw = qrot(RP, V3<double>{D[0] * wl.x, D[1] * wl.y, D[2] * wl.z});
    if (m.madd) {  // M is the explicit module's matrix, Mass models included
      Mw.x += m.madd[3 * N + n] * w0.x;
      Mw.y += m.madd[4 * N + n] * w0.y;
      Mw.z += m.madd[5 * N + n] * w0.z;
    }
    V3<double> gy = cross(w0, Mw);
    r[3] -= gy.x;
    r[4] -= gy.y;
    r[5] -= gy.z;
  }
  if (X && m.fint_last && step == out.last_step)  // internal force of this step (GroupOutput "resp")
    store_fint_last(m, n, fx[0] - r[0], fx[1] - r[1], fx[2] - r[2], fx[3] - r[3], fx[4] - r[4], fx[5] - r[5]);
  // added point masses (MassModel, MassModel.cpp:77-99): the explicit
  // module's mass matrix is the sum of all GET_MATRIX2 contributions, m +
  // madd per translational DOF and R P D P^T R^T + diag(madd) for the
  // rotations (then solved in full)
  const bool madd = m.madd != nullptr;
#pragma unroll
  for (int k = 0; k < 3; ++k)
    if (!(mask & (1u << k))) a[k] = madd ? r[k] / (m.mass[n] + m.madd[k * N + n]) : r[k] * im;
  const unsigned rm = (mask >> 3) & 7u;
  // lumped mass (ExplicitModule LUMPED, ExplicitModule.cpp:339-357): the
  // diagonal of R P D P^T R^T (+ added masses), one DOF at a time
  double dg[3] = {0.0, 0.0, 0.0};
  if (X && m.lumped) {
    double Rm[3][3];
    qmat(RP, Rm);
#pragma unroll
    for (int i = 0; i < 3; ++i) {
      dg[i] = Rm[i][0] * Rm[i][0] * D[0] + Rm[i][1] * Rm[i][1] * D[1] + Rm[i][2] * Rm[i][2] * D[2];
      if (madd) dg[i] += m.madd[(3 + i) * N + n];
      if (!(rm & (1u << i))) a[3 + i] = r[3 + i] / dg[i];
    }
  } else if (rm == 0u && !madd) {
    V3<double> rl = qrot(RPc, V3<double>{r[3], r[4], r[5]});
    V3<double> al = qrot(RP, V3<double>{rl.x * Dinv[0], rl.y * Dinv[1], rl.z * Dinv[2]});
    a[3] = al.x;
    a[4] = al.y;
    a[5] = al.z;
  } else if (rm != 7u) {
    double Rm[3][3], M3[3][3];
    qmat(RP, Rm);
    for (int i = 0; i < 3; ++i)
      for (int j = 0; j < 3; ++j)
        M3[i][j] = Rm[i][0] * D[0] * Rm[j][0] + Rm[i][1] * D[1] * Rm[j][1] + Rm[i][2] * D[2] * Rm[j][2];
    if (madd)
      for (int i = 0; i < 3; ++i) M3[i][i] += m.madd[(3 + i) * N + n];
    double rr[3] = {r[3], r[4], r[5]};
    double ar[3] = {a[3], a[4], a[5]};
    solve3_masked(M3, rr, ar, rm);
    a[3] = ar[0];
    a[4] = ar[1];
    a[5] = ar[2];
  }
  const double dt = m.dtn ? m.dtn[n] : m.dt;
#pragma unroll
  for (int k = 0; k < 6; ++k) v[k] += dt * a[k];
  const V3<double> du{dt * v[0], dt * v[1], dt * v[2]};
  x = x + du;
  const V3<double> dr{dt * v[3], dt * v[4], dt * v[5]};
  Q4<double> Rn;
  if (m.so3) {  // ExplicitModule::updateVec (:362-392): R <- exp(dt omega) R
    Rn = qnormalize(qmul(qexp_small(dr), R));
  } else {
    V3<double> th = qlog(R);
    Rn = qexp(th + dr);
  }
  if (loaded && rec)
    out.wext += fx[0] * du.x + fx[1] * du.y + fx[2] * du.z + fx[3] * dr.x + fx[4] * dr.y + fx[5] * dr.z;
  if (energy && rec) {  // E_kin = 1/2 v^T M v, M from the rotation at the start of the step
    const V3<double> wn{v[3], v[4], v[5]};
    double ek;
    if (X && m.lumped) {
      ek = 0.5 * ((EN ? mn : m.mass[n]) * (v[0] * v[0] + v[1] * v[1] + v[2] * v[2]) + dg[0] * v[3] * v[3] +
                  dg[1] * v[4] * v[4] + dg[2] * v[5] * v[5]);
      if (madd)
#pragma unroll
        for (int k = 0; k < 3; ++k) ek += 0.5 * m.madd[k * N + n] * v[k] * v[k];
    } else {
      const V3<double> wl = qrot(RPc, wn);
      ek = 0.5 * ((EN ? mn : m.mass[n]) * (v[0] * v[0] + v[1] * v[1] + v[2] * v[2]) + D[0] * wl.x * wl.x +
                  D[1] * wl.y * wl.y + D[2] * wl.z * wl.z);
      if (madd)  // the reference's E_kin uses the global mass matrix (LatticeModel.cpp:122-129, 223-250)
#pragma unroll
        for (int k = 0; k < 6; ++k) ek += 0.5 * m.madd[k * N + n] * v[k] * v[k];
    }
    out.ekin += ek;
    if (m.lat_energy && step == out.last_step) atomicAdd(m.lat_energy + m.nlat[n] * 5 + 0, ek);
  }
  bool finite = true;
#pragma unroll
  for (int k = 0; k < 6; ++k) finite = finite && isfinite(v[k]);
  if (!finite) atomicOr(m.err, 0x2u);
#pragma unroll
  for (int k = 0; k < 6; ++k) m.vel[k * N + n] = v[k];
  m.pos[n] = make_double4(x.x, x.y, x.z, 0.0);
  m.rot[n] = make_double4(Rn.w, Rn.x, Rn.y, Rn.z);
  if (X && m.tp_pos) {  // adjoint recomputation: node state after this step
    const size_t sl = static_cast<size_t>(step - m.tp_step0);
    m.tp_pos[sl * N + n] = make_double4(x.x, x.y, x.z, 0.0);
    m.tp_rot[sl * N + n] = make_double4(Rn.w, Rn.x, Rn.y, Rn.z);
#pragma unroll
    for (int k = 0; k < 6; ++k) m.tp_vel[(sl * 6 + k) * N + n] = v[k];
  }
  if (sidx >= 0 && smp.n_watch > 0) {
    const int slot = smp.watch_slot[n];
    if (slot >= 0) {
      double *o = smp.rows + (sidx * smp.n_watch + slot) * 13;
      o[0] = x.x; o[1] = x.y; o[2] = x.z;
      o[3] = Rn.w; o[4] = Rn.x; o[5] = Rn.y; o[6] = Rn.z;
#pragma unroll
      for (int k = 0; k < 6; ++k) o[7 + k] = v[k];
    }
  }
}

// ---------------------------------------------------------------------------
// grid barrier with a bounded wait
// ---------------------------------------------------------------------------
__device__ __forceinline__ unsigned ld_acquire(const unsigned *p) {
  unsigned v;
  asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
  return v;
}

__device__ __forceinline__ unsigned long long global_ns() {
  unsigned long long t;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
  return t;
}

// Launch-constant parameters of the grid barrier, read once per launch.
struct BarrierState {
  unsigned add0;                // block 0's arrival increment
  unsigned long long limit_ns;  // bound of one wait
};
__device__ __forceinline__ BarrierState barrier_begin(const GridBarrier *b) {
  const unsigned expect = gridDim.x + b->phantom;
  const unsigned lim = b->limit_us;
  return BarrierState{0x80000000u - (expect - 1u), lim ? 1000ull * lim : 2000000000ull};
}

// Returns false when the barrier was abandoned (its wait ran out here or in
// another block).  One atomic per block: the arrival (after a fence that
// publishes the block's writes) returns the word before it; the block then
// polls with acquire loads until bit 31 differs from that value.
static __device__ bool grid_barrier(GridBarrier *b, const BarrierState &bs, uint32_t *err) {
  __shared__ int s_ok;
  __syncthreads();
  if (threadIdx.x == 0) {
    int ok = 1;
    const unsigned inc = blockIdx.x == 0 ? bs.add0 : 1u;
    __threadfence();  // the block's writes (ordered by __syncthreads) before the arrival
    const unsigned old = atomicAdd(&b->count, inc);
    unsigned polls = 0;
    unsigned long long t0 = 0;
    while (((ld_acquire(&b->count) ^ old) & 0x80000000u) == 0u) {
      if ((++polls & 63u) == 0u) {  // the abort flag and the clock now and then
        if (ld_acquire(&b->abort)) {
          ok = 0;
          break;
        }
        const unsigned long long t = global_ns();
        if (t0 == 0) {
          t0 = t;
        } else if (t - t0 > bs.limit_ns) {
          atomicOr(err, 0x4u);
          atomicExch(&b->abort, 1u);
          ok = 0;
          break;
        }
      }
    }
    __threadfence();
    s_ok = ok;
  }
  __syncthreads();
  return s_ok != 0;
}

// ---------------------------------------------------------------------------
// kernels
// ---------------------------------------------------------------------------
__device__ __forceinline__ int64_t sample_index(const SampleSpec &smp, const StepCtx &c, int64_t step) {
  if (smp.every <= 0 || step % smp.every != 0) return -1;
  const int64_t idx = c.sample_base + step / smp.every - c.step0 / smp.every - 1;
  return idx < smp.capacity ? idx : -1;
}

template <class T, class Y, bool X, bool EN = false>
__device__ __forceinline__ void element_phase(const DevModel<T> &m, const SampleSpec &smp, const StepCtx &c,
                                              int64_t step, int gtid, int gstride) {
  const int64_t sidx = sample_index(smp, c, step);
  const bool last = (step == c.step0 + c.nsteps);
  const bool energy = EN || (sidx >= 0) || last;
  ElemEnergy en;
  const int64_t tslot = (X && m.tp_ep) ? step - m.tp_step0 : -1;
  const int64_t bslot = (X && m.br) ? step - m.br_step0 - 1 : -1;
  // two-point elements of two nodes take the compile-time point count;
  // elements of 3 or 4 nodes run in the extended kernels, through the
  // generic path below
  if (m.G == 2 && !(X && m.nen > 2)) {
    const int E = m.E;
    bool split = false;
    if constexpr (!X && sizeof(T) == 4) {  // the FP64 kernel spills more with the extra path
      if (E > gstride && E - gstride <= gstride / 2) {
        // one element per thread, then the rest as half elements on lane
        // pairs: the longest thread does one element and a half instead of two
        split = true;
        element_force<T, Y, X, HM_COMMIT, 2, EN>(m, gtid, true, energy, en, last, tslot);
        const int e2 = gstride + (gtid >> 1);
        if (e2 < E) element_force_half<T, Y, EN>(m, e2, gtid & 1, energy, en, last);
      }
    }
    if (!split)
      for (int e = gtid; e < E; e += gstride)
        element_force<T, Y, X, HM_COMMIT, 2, EN>(m, e, true, energy, en, last, tslot, nullptr, nullptr, nullptr,
                                                 bslot);
  } else {
    for (int e = gtid; e < m.E; e += gstride)
      element_force<T, Y, X, HM_COMMIT, 0, EN>(m, e, true, energy, en, last, tslot, nullptr, nullptr, nullptr, bslot);
  }
  double econ = 0.0;
  if (X) {
    for (int p = gtid; p < m.n_pairs; p += gstride) contact_pair(m, p, step, energy, econ);
    for (int p = gtid; p < m.n_jpairs; p += gstride) joint_pair(m, p, step, energy, econ);
  }
  if (energy) {
    double p = block_sum<T>(en.pot);
    double d = block_sum<T>(en.diss);
    double q = (X && (m.n_pairs || m.n_jpairs)) ? block_sum<T>(econ) : 0.0;
    if (threadIdx.x == 0) {
      if (sidx >= 0) {
        atomicAdd(smp.energy + sidx * 5 + 1, p);
        atomicAdd(smp.energy + sidx * 5 + 2, d);
        if (q != 0.0) atomicAdd(smp.energy + sidx * 5 + 4, q);
      }
      if (last) {
        atomicAdd(c.last_energy + 1, p);
        atomicAdd(c.last_energy + 2, d);
        if (q != 0.0) atomicAdd(c.last_energy + 4, q);
      }
    }
  }
}

template <class T, bool X, bool EN = false>
__device__ __forceinline__ void node_phase(const DevModel<T> &m, const SampleSpec &smp, const StepCtx &c,
                                           int64_t step, int gtid, int gstride) {
  const int64_t sidx = sample_index(smp, c, step);
  const bool last = (step == c.step0 + c.nsteps);
  const bool energy = EN || (sidx >= 0) || last;
  NodeOut out;
  out.last_step = c.step0 + c.nsteps;
  for (int n = gtid; n < m.N; n += gstride) node_update<T, X, EN>(m, n, step, energy, smp, sidx, out);
  double k = energy ? block_sum<T>(out.ekin) : 0.0;
  // external work: only models with loads (c.wstep is null without them)
  double w = c.wstep ? block_sum<T>(out.wext) : 0.0;
  double q = (X && energy && m.n_plates) ? block_sum<T>(out.econtact) : 0.0;
  if (threadIdx.x == 0) {
    if (w != 0.0) atomicAdd(c.wstep + (step - c.step0 - 1), w);
    if (sidx >= 0) atomicAdd(smp.energy + sidx * 5 + 0, k);
    if (last) atomicAdd(c.last_energy + 0, k);
    if (q != 0.0) {
      if (sidx >= 0) atomicAdd(smp.energy + sidx * 5 + 4, q);
      if (last) atomicAdd(c.last_energy + 4, q);
    }
    if (sidx >= 0 && blockIdx.x == 0) smp.steps[sidx] = step;
  }
}

// Threads per block of a full persistent grid.  The plain FP32-element
// kernel runs 320 threads at two blocks per SM (96 registers): 94,720
// resident threads, one node per thread for a 20^3 BCC lattice's 81,261
// nodes, and few enough elements left over after one per thread to run them
// as half elements (element_phase).  The FP64 kernel and the extended
// variants (contact, plates, adjoint tape) spill more at fewer registers and
// keep 256.
template <class T, bool X>
struct PersistShape {
  static constexpr int kThreads = (sizeof(T) == 4 && !X) ? 320 : 256;
};

// X: the extended-features variant (contact, rigid plates, adjoint tape,
// per-step group force, group output of the last step); plain runs take the
// X = false kernels, which carry none of that code.  EN: every step reports
// energies (a launch of one step, whose only step is its last): the energy
// code then has no branches and its loads are issued with the others; the
// state arithmetic is the same code as in the EN = false kernel.
template <class T, class Y, bool X, bool EN = false>
__global__ void __launch_bounds__(PersistShape<T, X>::kThreads, Y::kMinBlocks)
    k_persistent(const __grid_constant__ DevModel<T> m, const __grid_constant__ SampleSpec smp, const StepCtx c,
                 GridBarrier *bar) {
  const BarrierState bs = barrier_begin(bar);
  if (blockIdx.x == 0 && threadIdx.x < 5) c.next_energy[threadIdx.x] = 0.0;
  // Items (elements, nodes) in chunks of 32 per warp, the chunks dealt to
  // the blocks round robin: a warp's items stay contiguous (Morton order, for
  // the gathers), while every block takes chunks from all over the lattice,
  // so the costly regions (return-map iterations in the impact zone) are
  // shared by all blocks instead of falling to a few, which the others would
  // wait for at the grid barrier.
  const int gtid = ((threadIdx.x >> 5) * gridDim.x + blockIdx.x) * 32 + (threadIdx.x & 31);
  const int gstride = gridDim.x * blockDim.x;
  for (int s = 0; s < c.nsteps; ++s) {
    const int64_t step = c.step0 + s + 1;
    element_phase<T, Y, X, EN>(m, smp, c, step, gtid, gstride);
    if (!grid_barrier(bar, bs, m.err)) return;
    node_phase<T, X, EN>(m, smp, c, step, gtid, gstride);
    // the launch's end orders its last node phase before whatever follows
    // on the stream: no barrier after the last step
    if (s + 1 < c.nsteps && !grid_barrier(bar, bs, m.err)) return;
  }
}

template <class T, class Y, bool X>
__global__ void __launch_bounds__(256, Y::kMinBlocks)
    k_element(const __grid_constant__ DevModel<T> m, const __grid_constant__ SampleSpec smp, const StepCtx c,
              int64_t step) {
  element_phase<T, Y, X>(m, smp, c, step, blockIdx.x * blockDim.x + threadIdx.x, gridDim.x * blockDim.x);
}

template <class T, bool X>
__global__ void __launch_bounds__(256, 2)
    k_node(const __grid_constant__ DevModel<T> m, const __grid_constant__ SampleSpec smp, const StepCtx c,
           int64_t step) {
  node_phase<T, X>(m, smp, c, step, blockIdx.x * blockDim.x + threadIdx.x, gridDim.x * blockDim.x);
}

template <class T, class Y>
__global__ void k_internal_force(const __grid_constant__ DevModel<T> m) {
  ElemEnergy en;
  for (int e = blockIdx.x * blockDim.x + threadIdx.x; e < m.E; e += gridDim.x * blockDim.x) {
    if (m.nen > 2)
      element_force_n<T, Y, false, HM_COMMIT>(m, e, false, false, en, -1, m.pos, m.rot, nullptr, -1);
    else
      element_force<T, Y, false>(m, e, false, false, en);
  }
}

// Each node's internal force: the sum of its end-force slots, written to row
// n of fint (engine numbering), or to row perm[n] when perm is given (the
// caller's numbering).
template <class T>
__global__ void k_gather_force(const __grid_constant__ DevModel<T> m, double *fint, const int32_t *perm) {
  for (int n = blockIdx.x * blockDim.x + threadIdx.x; n < m.N; n += gridDim.x * blockDim.x) {
    double f[6] = {0, 0, 0, 0, 0, 0};
    for (int i = m.slot_ptr[n]; i < m.slot_ptr[n + 1]; ++i) load_end(m.ef + static_cast<size_t>(i) * 6, f);
    const size_t row = perm ? static_cast<size_t>(perm[n]) : static_cast<size_t>(n);
    for (int k = 0; k < 6; ++k) fint[row * 6 + k] = f[k];
  }
}

}  // namespace dl
