// Kernels of the reverse sweep of one explicit step (adjoint of step.cuh),
// shared by the ahead-of-time build (adjoint.cu, elastic lattices) and the
// runtime-compiled build (jit.cpp, elastoplastic lattices with the generated
// YieldAdj policy).  One reverse step k+1 -> k is two launches:
//   k_adj_node: per node, the complete adjoint of the state after step k+1
//     (node part from the previous reverse step plus the element-end
//     contributions) through the node update: adjoints of the state before
//     the step and of the step's internal force;
//   k_adj_elem: per element, the adjoint of its end forces through the
//     element (kinematics, strains, return map): contributions to the node
//     adjoints of the state before the step (node-ordered end slots), the
//     history adjoints (in place) and the section/yield-variable adjoints.
// The states come from the tape written by the recomputed forward segment.
#pragma once

#include "adjoint.cuh"
#include "devtypes.cuh"
#include "step.cuh"

namespace dl {

// elastic lattices: no return map in the adjoint either
struct AdjElastic {
  static constexpr bool kPlastic = false;
  static constexpr int kNh = 0;
  template <class T, class M>
  __device__ static T f(const M &, const T *) {
    return T(0);
  }
  template <class T, class M>
  __device__ static void grad(const M &, const T *, T *) {}
  template <class T, class M>
  __device__ static void vjp(const M &, const T *, T, const T *, T *) {}
};

// Reverse of the node update of one step for node n.
template <class T>
__device__ __forceinline__ void adj_node_one(const DevModel<T> &m, const AdjCtx<T> &a, int64_t step, int n) {
  const int N = m.N;
  const size_t s1 = static_cast<size_t>(step - m.tp_step0), s0 = s1 - 1;
  // complete adjoint of the state after the step
  double lx1[3] = {a.lx[n], a.lx[N + n], a.lx[2 * N + n]};
  double lt1[3] = {a.lth[n], a.lth[N + n], a.lth[2 * N + n]};
  for (int i = m.slot_ptr[n]; i < m.slot_ptr[n + 1]; ++i) {
    const double *q = a.aslot + static_cast<size_t>(i) * 6;
    for (int k = 0; k < 3; ++k) {
      lx1[k] += q[k];
      lt1[k] += q[3 + k];
    }
  }
  double lv1[6];
  for (int k = 0; k < 6; ++k) lv1[k] = a.lv[k * N + n];
  NodeIn in;
  const double4 x0 = m.tp_pos[s0 * N + n], r0 = m.tp_rot[s0 * N + n];
  in.x = V3<double>{x0.x, x0.y, x0.z};
  in.R = Q4<double>{r0.x, r0.y, r0.z, r0.w};
  double v1[6];
  for (int k = 0; k < 6; ++k) {
    in.v[k] = m.tp_vel[(s0 * 6 + k) * N + n];
    v1[k] = m.tp_vel[(s1 * 6 + k) * N + n];
  }
  in.mass = m.mass[n];
  const auto Pq = m.iframe[n];
  const auto Dv = m.idiag[n];
  in.P = Q4<double>{double(Pq.x), double(Pq.y), double(Pq.z), double(Pq.w)};
  in.D[0] = double(Dv.x);
  in.D[1] = double(Dv.y);
  in.D[2] = double(Dv.z);
  unsigned mask = 0u;
  for (int b = m.bc_ptr[n]; b < m.bc_ptr[n + 1]; ++b)
    if (m.bc[b].kind == BCD_DIRICHLET) mask |= 1u << m.bc[b].dof;
  in.mask = mask;
  in.dt = m.dt;
  in.gyro = m.gyro;
  for (int k = 0; k < 6; ++k) {
    in.aPre[k] = (v1[k] - in.v[k]) / m.dt;  // the prescribed accelerations of the masked DOFs
    in.fx[k] = 0.0;                           // loads do not enter the adjoint
  }
  double seed[6] = {0, 0, 0, 0, 0, 0};
  if (step == a.peak_step && a.peak_flag && a.peak_flag[n]) seed[a.peak_dof] = a.w_peak;
  V3<double> lx0, lth0;
  double lv0[6], lf[6], lm, lS[6];
  node_vjp(in, v1, V3<double>{lx1[0], lx1[1], lx1[2]}, V3<double>{lt1[0], lt1[1], lt1[2]}, lv1, seed, lx0, lth0,
           lv0, lf, lm, lS);
  a.lx[n] = lx0.x;
  a.lx[N + n] = lx0.y;
  a.lx[2 * N + n] = lx0.z;
  a.lth[n] = lth0.x;
  a.lth[N + n] = lth0.y;
  a.lth[2 * N + n] = lth0.z;
  for (int k = 0; k < 6; ++k) {
    a.lv[k * N + n] = lv0[k];
    a.lf[k * N + n] = lf[k];
    a.lS[k * N + n] += lS[k];
  }
  a.lmass[n] += lm;
}

template <class T>
__global__ void __launch_bounds__(256) k_adj_node(const __grid_constant__ DevModel<T> m, const AdjCtx<T> a,
                                                        int64_t step) {
  for (int n = blockIdx.x * blockDim.x + threadIdx.x; n < m.N; n += gridDim.x * blockDim.x)
    adj_node_one(m, a, step, n);
}

// sum over the P lanes of an element (lanes aligned to P, P a power of two)
__device__ __forceinline__ double lane_sum(double v, unsigned mask, int P) {
  for (int o = 1; o < P; o <<= 1) v += __shfl_xor_sync(mask, v, o);
  return v;
}
__device__ __forceinline__ float lane_sum(float v, unsigned mask, int P) {
  for (int o = 1; o < P; o <<= 1) v += __shfl_xor_sync(mask, v, o);
  return v;
}
template <class T>
__device__ __forceinline__ V3<T> lane_sum(V3<T> v, unsigned mask, int P) {
  return V3<T>{lane_sum(v.x, mask, P), lane_sum(v.y, mask, P), lane_sum(v.z, mask, P)};
}
template <class T>
__device__ __forceinline__ Q4<T> lane_sum(Q4<T> q, unsigned mask, int P) {
  return Q4<T>{lane_sum(q.w, mask, P), lane_sum(q.x, mask, P), lane_sum(q.y, mask, P), lane_sum(q.z, mask, P)};
}

// end states (from the tape) and end frames of element e
template <class T>
__device__ __forceinline__ void load_elem_kin(const DevModel<T> &m, int e, int2 c, size_t s0, ElemIn<T> &in) {
  const int N = m.N, E = m.E;
  const double4 xa = m.tp_pos[s0 * N + c.x], xb = m.tp_pos[s0 * N + c.y];
  const double4 ra = m.tp_rot[s0 * N + c.x], rb = m.tp_rot[s0 * N + c.y];
  in.xi = V3<double>{xa.x, xa.y, xa.z};
  in.xj = V3<double>{xb.x, xb.y, xb.z};
  in.Ri = Q4<double>{ra.x, ra.y, ra.z, ra.w};
  in.Rj = Q4<double>{rb.x, rb.y, rb.z, rb.w};
  in.qNi = toq(m.qN[e]);
  in.qNj = toq(m.qN[E + e]);
  in.invL0 = m.invL0[e];
}

// One thread per (element, Gauss point): every lane of an element recomputes
// the shared kinematic prefix, runs its own Gauss point (strain, return map
// and their reverse), the lanes' adjoints are summed with shuffles and the
// element's first lane reverses the prefix and writes the end slots and the
// section adjoints.  Each lane reads and writes its own point's history.
template <class T, class Y>
__global__ void __launch_bounds__(256) k_adj_elem(const __grid_constant__ DevModel<T> m, const AdjCtx<T> a,
                                                        int64_t step) {
  const int E = m.E, N = m.N, G = m.G;
  const int nh = Y::kNh >= 0 ? Y::kNh : m.nh;  // compile-time in the generated policies
  const int P = adj_lanes(G);
  const PlastLaw<T> law{m.H, m.max_iter, m.prec};
  const int lane = threadIdx.x & 31;
  const unsigned gmask = (P == 1 ? 1u : ((1u << P) - 1u)) << (lane & ~(P - 1));
  const int total = E * P;  // blockDim.x is a multiple of 32, so an element's lanes share a warp
  for (int t = blockIdx.x * blockDim.x + threadIdx.x; t < total; t += gridDim.x * blockDim.x) {
    const int e = t / P, g = t - e * P;
    const size_t s0 = static_cast<size_t>(step - m.tp_step0) - 1;
    const int2 c = m.conn[e];
    ElemIn<T> in;
    load_elem_kin(m, e, c, s0, in);
    in.L0 = double(m.L0[e]);
    for (int q = 0; q < 6; ++q) in.C[q] = m.C[q * E + e];
    in.ec[0] = m.ec[e];
    in.ec[1] = m.ec[E + e];
    in.G = G;
    in.nh = nh;
    in.plastic = m.plastic;
    double lf[12];
    for (int k = 0; k < 6; ++k) {
      lf[k] = a.lf[k * N + c.x];
      lf[6 + k] = a.lf[k * N + c.y];
    }
    ElemGpAdj<T> acc;
    gp_adj_zero(acc);
    const bool plastic = Y::kPlastic && m.plastic;
    if (g < G) {
      ElemPrefix<T> pre;
      elem_vjp_prefix(in, pre);
      GpIn<T> gi;
      GpHistAdj lh;
      for (int q = 0; q < 3; ++q) {
        gi.g0[q] = m.g0[(g * 3 + q) * E + e];
        gi.k0[q] = m.k0[(g * 3 + q) * E + e];
      }
      double ldiss = 0.0;
      if (plastic) {
        const size_t o6 = s0 * G * 6 * E, oh = s0 * G * nh * E;
        for (int q = 0; q < 6; ++q) {
          gi.ep[q] = m.tp_ep[o6 + (g * 6 + q) * E + e];
          gi.epsc[q] = m.tp_epsc[o6 + (g * 6 + q) * E + e];
          lh.ep[q] = a.lep[(g * 6 + q) * E + e];
          lh.epsc[q] = a.lepsc[(g * 6 + q) * E + e];
        }
        for (int q = 0; q < nh; ++q) {
          gi.al[q] = m.tp_al[oh + (g * nh + q) * E + e];
          lh.al[q] = a.lal[(g * nh + q) * E + e];
        }
        ldiss = a.w_diss * adj_gw(G, g) * 0.5 * in.L0;
      }
      elem_vjp_gp<T, Y>(m, law, in, pre, g, gi, lf, &lh, ldiss, acc);
      if (plastic) {
        for (int q = 0; q < 6; ++q) {
          a.lep[(g * 6 + q) * E + e] = lh.ep[q];
          a.lepsc[(g * 6 + q) * E + e] = lh.epsc[q];
        }
        for (int q = 0; q < nh; ++q) a.lal[(g * nh + q) * E + e] = lh.al[q];
      }
    }
    if (P > 1) {
      acc.lphi = lane_sum(acc.lphi, gmask, P);
      acc.ld = lane_sum(acc.ld, gmask, P);
      acc.ldme3 = lane_sum(acc.ldme3, gmask, P);
      acc.lppT = lane_sum(acc.lppT, gmask, P);
      acc.lqr = lane_sum(acc.lqr, gmask, P);
      acc.lepair = lane_sum(acc.lepair, gmask, P);
      for (int q = 0; q < 6; ++q) acc.lC[q] = lane_sum(acc.lC[q], gmask, P);
      acc.lec[0] = lane_sum(acc.lec[0], gmask, P);
      acc.lec[1] = lane_sum(acc.lec[1], gmask, P);
    }
    if (g == 0) {
      // the FP64 prefix again from reloaded end states: cheaper than
      // keeping it in registers across the Gauss-point work
      load_elem_kin(m, e, c, s0, in);
      ElemPrefix<T> pre;
      elem_vjp_prefix(in, pre);
      ElemAdjOut o;
      elem_vjp_suffix(in, pre, acc, o);
      const int2 sl = m.eslot[e];
      double *pa = a.aslot + static_cast<size_t>(sl.x) * 6;
      double *pb = a.aslot + static_cast<size_t>(sl.y) * 6;
      pa[0] = o.lxi.x; pa[1] = o.lxi.y; pa[2] = o.lxi.z;
      pa[3] = o.lthi.x; pa[4] = o.lthi.y; pa[5] = o.lthi.z;
      pb[0] = o.lxj.x; pb[1] = o.lxj.y; pb[2] = o.lxj.z;
      pb[3] = o.lthj.x; pb[4] = o.lthj.y; pb[5] = o.lthj.z;
      for (int q = 0; q < 6; ++q) a.lC[q * E + e] += o.lC[q];
      a.lec[e] += o.lec[0];
      a.lec[E + e] += o.lec[1];
    }
  }
}

}  // namespace dl
