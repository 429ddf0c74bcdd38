// Ahead-of-time kernels (nvcc, sm_100a) and host launchers.
//
// The step kernels themselves live in step.cuh; this file instantiates them
// with the interpreting yield policy and holds the small utility kernels
// (energy slots, external-work bookkeeping, state conversion).
#include <algorithm>
#include <cstdint>

#include "engine.hpp"
#include "rodkin.cuh"
#include "milne.cuh"

namespace dl {

__global__ void k_clear5(double *p) {
  if (threadIdx.x < 5) p[threadIdx.x] = 0.0;
}

__global__ void k_finish_wext(double *wstep, int n, double *wext_total, SampleSpec smp, int64_t step0,
                              int64_t sample_base, double *last_energy) {
  if (threadIdx.x != 0 || blockIdx.x != 0) return;
  double acc = *wext_total;
  for (int s = 0; s < n; ++s) {
    acc += wstep[s];
    wstep[s] = 0.0;
    const int64_t step = step0 + s + 1;
    if (smp.every > 0 && step % smp.every == 0) {
      const int64_t idx = sample_base + step / smp.every - step0 / smp.every - 1;
      if (idx < smp.capacity) smp.energy[idx * 5 + 3] = acc;
    }
  }
  *wext_total = acc;
  last_energy[3] = acc;
}


// ---------------------------------------------------------------------------
// state conversion between the internal layout and caller arrays in the
// original node numbering: u = x - X0, theta = log(R), v
// ---------------------------------------------------------------------------
__global__ void k_state_out(const double4 *pos, const double4 *rot, const double *vel, const double *X0,
                            const int32_t *node_old, int N, double *u, double *th, double *v) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < N; i += gridDim.x * blockDim.x) {
    const int n = node_old[i];
    const double4 p = pos[i];
    if (u) {
      u[n * 3] = p.x - X0[i * 3];
      u[n * 3 + 1] = p.y - X0[i * 3 + 1];
      u[n * 3 + 2] = p.z - X0[i * 3 + 2];
    }
    if (th) {
      const double4 q = rot[i];
      const V3<double> t = qlog(Q4<double>{q.x, q.y, q.z, q.w});
      th[n * 3] = t.x;
      th[n * 3 + 1] = t.y;
      th[n * 3 + 2] = t.z;
    }
    if (v)
      for (int k = 0; k < 6; ++k) v[n * 6 + k] = vel[k * N + i];
  }
}

__global__ void k_state_in(double4 *pos, double4 *rot, double *vel, const double *X0, const int32_t *node_old,
                           int N, const double *u, const double *th, const double *v) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < N; i += gridDim.x * blockDim.x) {
    const int n = node_old[i];
    if (u) pos[i] = make_double4(X0[i * 3] + u[n * 3], X0[i * 3 + 1] + u[n * 3 + 1], X0[i * 3 + 2] + u[n * 3 + 2], 0.0);
    if (th) {
      const Q4<double> q = qexp(V3<double>{th[n * 3], th[n * 3 + 1], th[n * 3 + 2]});
      rot[i] = make_double4(q.w, q.x, q.y, q.z);
    }
    if (v)
      for (int k = 0; k < 6; ++k) vel[k * N + i] = v[n * 6 + k];
  }
}

// ---------------------------------------------------------------------------
// host launchers
// ---------------------------------------------------------------------------
static int grid_for(int n, int threads) {
  int dev = 0, sms = 0;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  const int want = (n + threads - 1) / threads;
  const int cap = sms * 8;
  return want < 1 ? 1 : (want > cap ? cap : want);
}

int threads_for(int work) {
  static int sms = 0;
  if (sms == 0) {
    int dev = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    if (sms <= 0) sms = 1;
  }
  int tpb = 256;
  while (tpb > 32 && (work + tpb - 1) / tpb < sms) tpb /= 2;
  return tpb;
}

void set_persistent_caps(KernelSet &ks) {
  // the step kernels use a few hundred bytes of shared memory: the rest of
  // each SM's on-chip memory serves as L1 for the node gathers and slot runs
  for (const void *k : {ks.persistent, ks.persistent1, ks.persistent_x, ks.element, ks.node, ks.element_x, ks.node_x,
                        ks.milne})
    if (k && cudaFuncSetAttribute(k, cudaFuncAttributePreferredSharedMemoryCarveout,
                                  static_cast<int>(cudaSharedmemCarveoutMaxL1)) != cudaSuccess)
      cudaGetLastError();
  for (int i = 0; i < 4; ++i) {
    ks.persist_cap[i] = cooperative_blocks(ks.persistent, i == 3 ? ks.full_threads : 32 << i);
    ks.persist_cap1[i] = ks.persistent1 ? cooperative_blocks(ks.persistent1, i == 3 ? ks.full_threads : 32 << i) : 0;
    ks.persist_cap_x[i] = cooperative_blocks(ks.persistent_x, i == 3 ? ks.full_threads_x : 32 << i);
    ks.milne_cap[i] = ks.milne ? cooperative_blocks(ks.milne, 32 << i) : 0;
  }
  ks.persist_blocks = ks.persist_cap[3];
}

int cooperative_blocks(const void *kernel, int threads) {
  int dev = 0, sms = 0, occ = 0;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, kernel, threads, 0) != cudaSuccess) {
    cudaGetLastError();
    occ = 1;
  }
  if (occ < 1) occ = 1;
  return sms * occ;
}

template <class T, class Y>
static KernelSet aot_set() {
  KernelSet k;
  k.persistent = reinterpret_cast<const void *>(k_persistent<T, Y, false>);
  k.persistent1 = reinterpret_cast<const void *>(k_persistent<T, Y, false, true>);
  k.element = reinterpret_cast<const void *>(k_element<T, Y, false>);
  k.node = reinterpret_cast<const void *>(k_node<T, false>);
  k.persistent_x = reinterpret_cast<const void *>(k_persistent<T, Y, true>);
  k.element_x = reinterpret_cast<const void *>(k_element<T, Y, true>);
  k.node_x = reinterpret_cast<const void *>(k_node<T, true>);
  k.internal_force = reinterpret_cast<const void *>(k_internal_force<T, Y>);
  k.gather = reinterpret_cast<const void *>(k_gather_force<T>);
  k.milne = reinterpret_cast<const void *>(k_milne<T, Y>);
  k.full_threads = PersistShape<T, false>::kThreads;
  k.full_threads_x = PersistShape<T, true>::kThreads;
  set_persistent_caps(k);
  k.jit = false;
  return k;
}

template <class T>
KernelSet aot_kernels(bool plastic) {
  return plastic ? aot_set<T, YieldInterp>() : aot_set<T, ElasticOnly>();
}

template <class T>
cudaError_t launch_steps(const KernelSet &ks, const DevModel<T> &m, const SampleSpec &smp, const StepCtx &c,
                         int mode, GridBarrier *bar, cudaStream_t s) {
  if (c.nsteps <= 0) return cudaSuccess;
  // the extended kernels only when the model or the run uses their features
  const bool ext = m.c_ptr || m.j_ptr || m.n_plates > 0 || m.tp_pos || m.tp_ep || m.grp_hist || m.fint_last ||
                   m.br || m.lumped || m.tie_ptr || m.nen > 2;
  DevModel<T> mm = m;
  SampleSpec ss = smp;
  StepCtx cc = c;
  if (mode == EXEC_PERSISTENT || mode == EXEC_GRAPH) {
    GridBarrier *bb = bar;
    void *args[] = {&mm, &ss, &cc, &bb};
    // one element or node per thread at most: small models take few blocks,
    // which keeps the grid barriers short
    const int work = std::max(std::max(m.E, m.N), m.n_pairs);
    int tpb = ks.tpb_override > 0 ? ks.tpb_override : threads_for(work);
    if (tpb == 256) tpb = ext ? ks.full_threads_x : ks.full_threads;
    const int ci = tpb == 32 ? 0 : (tpb == 64 ? 1 : (tpb == 128 ? 2 : 3));
    const int want = std::max(1, (work + tpb - 1) / tpb);
    // a launch of one step reports its energies: the kernel with that known
    const bool one = !ext && c.nsteps == 1 && ks.persistent1 && ks.persist_cap1[ci] > 0;
    const int cap = ext ? ks.persist_cap_x[ci] : (one ? ks.persist_cap1[ci] : ks.persist_cap[ci]);
    const int blocks = std::min(cap > 0 ? cap : ks.persist_blocks, want);
    const void *kern = ext ? ks.persistent_x : (one ? ks.persistent1 : ks.persistent);
    return cudaLaunchCooperativeKernel(kern, dim3(blocks), dim3(tpb), args, 0, s);
  }
  const int eb = grid_for(m.E, 256), nb = grid_for(m.N, 256);
  k_clear5<<<1, 32, 0, s>>>(c.last_energy);
  k_clear5<<<1, 32, 0, s>>>(c.next_energy);
  for (int i = 0; i < c.nsteps; ++i) {
    int64_t step = c.step0 + i + 1;
    void *args[] = {&mm, &ss, &cc, &step};
    cudaError_t e = cudaLaunchKernel(ext ? ks.element_x : ks.element, dim3(eb), dim3(256), args, 0, s);
    if (e != cudaSuccess) return e;
    e = cudaLaunchKernel(ext ? ks.node_x : ks.node, dim3(nb), dim3(256), args, 0, s);
    if (e != cudaSuccess) return e;
  }
  return cudaGetLastError();
}

void milne_shape(const KernelSet &ks, int work, int *blocks, int *tpb) {
  const int t = ks.tpb_override > 0 ? ks.tpb_override : threads_for(work);
  const int ci = t == 32 ? 0 : (t == 64 ? 1 : (t == 128 ? 2 : 3));
  const int want = std::max(1, (work + t - 1) / t);
  const int cap = ks.milne_cap[ci] > 0 ? ks.milne_cap[ci] : 1;
  *blocks = std::min(cap, want);
  *tpb = t;
}

template <class T>
cudaError_t launch_milne(const KernelSet &ks, const DevModel<T> &m, const SampleSpec &smp, const StepCtx &c,
                         GridBarrier *bar, const MilneDev<T> &md, int blocks, int tpb, cudaStream_t s) {
  if (c.nsteps <= 0) return cudaSuccess;
  if (!ks.milne) return cudaErrorInvalidDeviceFunction;
  DevModel<T> mm = m;
  SampleSpec ss = smp;
  StepCtx cc = c;
  GridBarrier *bb = bar;
  MilneDev<T> dd = md;
  void *args[] = {&mm, &ss, &cc, &bb, &dd};
  return cudaLaunchCooperativeKernel(ks.milne, dim3(blocks), dim3(tpb), args, 0, s);
}

template <class T>
cudaError_t launch_internal_force(const KernelSet &ks, const DevModel<T> &m, double *fint, cudaStream_t s) {
  DevModel<T> mm = m;
  double *ff = fint;
  const int32_t *perm = nullptr;  // engine numbering
  void *a1[] = {&mm};
  cudaError_t e = cudaLaunchKernel(ks.internal_force, dim3(grid_for(m.E, 256)), dim3(256), a1, 0, s);
  if (e != cudaSuccess) return e;
  void *a2[] = {&mm, &ff, &perm};
  return cudaLaunchKernel(ks.gather, dim3(grid_for(m.N, 256)), dim3(256), a2, 0, s);
}

// Element tables of the reference's GET_TABLE action at the current state,
// as ParaViewModule writes them as cell data (ParaViewModule.cpp:585-616):
// per Gauss point the strain (SpecialCosseratRodModel::getStrainTable_,
// SpecialCosseratRodModel.cpp:428-478: Gamma - Gamma0, K - K0), the stress
// (getStressTable_, :482-532, with the output load case: C (eps - eps_p) from
// the committed plastic strain, ElastoPlasticRodMaterial.cpp:217-224) or the
// plastic strain (ElastoPlasticRodMaterial::getTable "plast_strain", :323-340),
// in the material frame or rotated by the point's rotation (spatial,
// getStrains_/getStresses_ :737-741, 763-770); the points' values are summed
// and the sum scaled by the point count (the table's weights, which
// ParaViewModule applies with scaleRows without inverting them).  out is
// [E][6] in internal element order.
template <class T>
__global__ void k_elem_table(const DevModel<T> m, int kind, int spatial, double *out) {
  for (int e = blockIdx.x * blockDim.x + threadIdx.x; e < m.E; e += gridDim.x * blockDim.x) {
    const int E = m.E;
    const int G = m.G;
    if (m.nen > 2) {  // elements of 3 or 4 nodes
      ElemPreN pn;
      elem_pre_n(m, e, m.pos, m.rot, pn);
      double acc[6] = {0, 0, 0, 0, 0, 0};
      for (int g = 0; g < G; ++g) {
        T eps[6];
        double w, N[kMaxElemNodes], dN[kMaxElemNodes];
        const GpKinN k = gp_eps_n(m, e, g, pn, eps, w, N, dN);
        const Q4<T> qg = cvtq<T>(k.L);
        T val[6];
        for (int q = 0; q < 6; ++q) {
          const T ep = m.plastic ? m.ep[(g * 6 + q) * E + e] : T(0);
          val[q] = kind == 0 ? eps[q] : (kind == 1 ? T(m.C[q * E + e]) * (eps[q] - ep) : ep);
        }
        if (spatial) {
          const V3<T> a = qrot(qg, V3<T>{val[0], val[1], val[2]});
          const V3<T> b = qrot(qg, V3<T>{val[3], val[4], val[5]});
          val[0] = a.x; val[1] = a.y; val[2] = a.z;
          val[3] = b.x; val[4] = b.y; val[5] = b.z;
        }
        for (int q = 0; q < 6; ++q) acc[q] += double(val[q]);
      }
      for (int q = 0; q < 6; ++q) out[static_cast<size_t>(e) * 6 + q] = acc[q] * G;
      continue;
    }
    ElemPre<T> p;
    elem_pre(m, e, m.pos, m.rot, p);
    const Q4<T> epair = qexp((T(-0.5) * T(c_gxi[G - 1][G - 1])) * p.k.phi);
    double acc[6] = {0, 0, 0, 0, 0, 0};
    for (int g = 0; g < G; ++g) {
      const T xg = T(c_gxi[G - 1][g]);
      const Q4<T> eg = xg > T(0) ? epair : (xg < T(0) ? qconj(epair) : Q4<T>{T(1), T(0), T(0), T(0)});
      T g0[3], k0[3];
      for (int q = 0; q < 3; ++q) {
        g0[q] = m.g0[(g * 3 + q) * E + e];
        k0[q] = m.k0[(g * 3 + q) * E + e];
      }
      T eps[6];
      Q4<T> qg;
      gp_strain_e(p.k, eg, p.il, g0, k0, eps, &qg);
      T val[6];
      for (int k = 0; k < 6; ++k) {
        const T ep = m.plastic ? m.ep[(g * 6 + k) * E + e] : T(0);
        val[k] = kind == 0 ? eps[k] : (kind == 1 ? p.Cd[k] * (eps[k] - ep) : ep);
      }
      if (spatial) {
        const V3<T> a = qrot(qg, V3<T>{val[0], val[1], val[2]});
        const V3<T> b = qrot(qg, V3<T>{val[3], val[4], val[5]});
        val[0] = a.x; val[1] = a.y; val[2] = a.z;
        val[3] = b.x; val[4] = b.y; val[5] = b.z;
      }
      for (int k = 0; k < 6; ++k) acc[k] += double(val[k]);
    }
    for (int k = 0; k < 6; ++k) out[static_cast<size_t>(e) * 6 + k] = acc[k] * G;
  }
}

template <class T>
cudaError_t launch_elem_table(const DevModel<T> &m, int kind, bool spatial, double *out, cudaStream_t s) {
  k_elem_table<T><<<grid_for(m.E, 256), 256, 0, s>>>(m, kind, spatial ? 1 : 0, out);
  return cudaGetLastError();
}

cudaError_t launch_finish_wext(double *wstep, int n, double *wext_total, const SampleSpec &smp,
                               int64_t step0, int64_t sample_base, double *last_energy, cudaStream_t s) {
  k_finish_wext<<<1, 32, 0, s>>>(wstep, n, wext_total, smp, step0, sample_base, last_energy);
  return cudaGetLastError();
}

cudaError_t launch_state_out(const double4 *pos, const double4 *rot, const double *vel, const double *X0,
                             const int32_t *node_old, int N, double *u, double *th, double *v, cudaStream_t s) {
  k_state_out<<<grid_for(N, 256), 256, 0, s>>>(pos, rot, vel, X0, node_old, N, u, th, v);
  return cudaGetLastError();
}

cudaError_t launch_state_in(double4 *pos, double4 *rot, double *vel, const double *X0, const int32_t *node_old,
                            int N, const double *u, const double *th, const double *v, cudaStream_t s) {
  k_state_in<<<grid_for(N, 256), 256, 0, s>>>(pos, rot, vel, X0, node_old, N, u, th, v);
  return cudaGetLastError();
}

#define DL_INSTANTIATE(T)                                                                              \
  template KernelSet aot_kernels<T>(bool);                                                                 \
  template cudaError_t launch_steps<T>(const KernelSet &, const DevModel<T> &, const SampleSpec &,     \
                                       const StepCtx &, int, GridBarrier *, cudaStream_t);            \
  template cudaError_t launch_internal_force<T>(const KernelSet &, const DevModel<T> &, double *,     \
                                                cudaStream_t);                                        \
  template cudaError_t launch_milne<T>(const KernelSet &, const DevModel<T> &, const SampleSpec &,     \
                                       const StepCtx &, GridBarrier *, const MilneDev<T> &, int, int, \
                                       cudaStream_t);                                                 \
  template cudaError_t launch_elem_table<T>(const DevModel<T> &, int, bool, double *, cudaStream_t);
DL_INSTANTIATE(float)
DL_INSTANTIATE(double)

}  // namespace dl
