// MilneDevice predictor-corrector with error-controlled time step
// (MilneDeviceModule::solve, MilneDeviceModule.cpp:41-118, order 1, with
// ExplicitModule::advance/commit/cancel, ExplicitModule.cpp:259-334), as one
// persistent cooperative launch over many accepted steps.  Shared by the
// ahead-of-time build (kernels.cu) and the runtime-compiled elastoplastic
// kernels (jit.cpp).
//
// One attempt of step n -> n+1 (t -> t + dt) is four phases separated by the
// bounded grid barrier:
//   A  element force at the current state (return map from the committed
//      history, nothing written);
//   A' node: a_cur = M^-1 (f_ext - f_int), prediction v_pre = v + dt a_cur,
//      x_pre = x + dt v, R_pre = exp(dt w) R  ->  pre buffers;
//   B  element force at the predicted state, the resulting history written
//      to the trial buffers (the reference commits the history of its last
//      force evaluation, which is this one);
//   B' node: a_pre with the same mass (rotation of the step's start) and
//      loads, correction v_new = v + dt a_pre, x_new = x + dt v_pre,
//      R_new = exp(dt w_pre) R  ->  pre buffers; per-block sums of the
//      squared prediction-correction differences (getQuality, :494-501).
// Then every block reduces the per-block sums in the same order, so all of
// them take the same accept/reject decision and the same next dt.  An
// accepted step's state and history are taken over at the start of the
// next attempt (the element and node threads that own them copy them), or
// at the end of the launch.  A rejected step leaves the current state and
// repeats with the smaller dt.
#pragma once

#include "step.cuh"

namespace dl {

// Loads and prescribed accelerations of node n from the block's scale values.
template <class T>
__device__ __forceinline__ unsigned milne_bcs(const DevModel<T> &m, int n, const double *scale, double fx[6],
                                              double a[6]) {
  unsigned mask = 0u;
  for (int b = m.bc_ptr[n]; b < m.bc_ptr[n + 1]; ++b) {
    const BcTerm t = m.bc[b];
    const double val = t.factor * (t.scale < 0 ? 1.0 : scale[t.scale]);
#pragma unroll
    for (int k = 0; k < 6; ++k) {
      if (t.dof != k) continue;
      if (t.kind == BCD_NEUMANN) {
        fx[k] += val;
      } else {
        a[k] = val;
      }
    }
    if (t.kind != BCD_NEUMANN) mask |= 1u << t.dof;
  }
  return mask;
}

// a = M^-1 (fx - f - w x (M w)) for the free components (getAcce,
// ExplicitModule.cpp:339-357); M from the rotation R of the step's start,
// the gyroscopic term with the velocity wg of the evaluated state.
template <class T>
__device__ __forceinline__ void milne_accel(const DevModel<T> &m, int n, const Q4<double> &R, const V3<double> &wg,
                                            const double f[6], const double fx[6], unsigned mask, double a[6]) {
  double r[6];
#pragma unroll
  for (int k = 0; k < 6; ++k) r[k] = fx[k] - f[k];
  const Q4<double> P = toq(m.iframe[n]);
  const auto Dv = m.idiag[n];
  const auto Di = m.idinv[n];
  const double D[3] = {double(Dv.x), double(Dv.y), double(Dv.z)};
  const double Dinv[3] = {double(Di.x), double(Di.y), double(Di.z)};
  const Q4<double> RP = qmul(R, P);
  const Q4<double> RPc = qconj(RP);
  if (m.gyro) {
    const V3<double> wl = qrot(RPc, wg);
    const V3<double> Mw = qrot(RP, V3<double>{D[0] * wl.x, D[1] * wl.y, D[2] * wl.z});
    const V3<double> gy = cross(wg, Mw);
    r[3] -= gy.x;
    r[4] -= gy.y;
    r[5] -= gy.z;
  }
  const double im = m.imass[n];
#pragma unroll
  for (int k = 0; k < 3; ++k)
    if (!(mask & (1u << k))) a[k] = r[k] * im;
  const unsigned rm = (mask >> 3) & 7u;
  if (rm == 0u) {
    const V3<double> rl = qrot(RPc, V3<double>{r[3], r[4], r[5]});
    const V3<double> al = qrot(RP, V3<double>{rl.x * Dinv[0], rl.y * Dinv[1], rl.z * Dinv[2]});
    a[3] = al.x;
    a[4] = al.y;
    a[5] = al.z;
  } else if (rm != 7u) {
    double Rm[3][3], M3[3][3];
    qmat(RP, Rm);
    for (int i = 0; i < 3; ++i)
      for (int j = 0; j < 3; ++j)
        M3[i][j] = Rm[i][0] * D[0] * Rm[j][0] + Rm[i][1] * D[1] * Rm[j][1] + Rm[i][2] * D[2] * Rm[j][2];
    double rr[3] = {r[3], r[4], r[5]};
    double ar[3] = {a[3], a[4], a[5]};
    solve3_masked(M3, rr, ar, rm);
    a[3] = ar[0];
    a[4] = ar[1];
    a[5] = ar[2];
  }
}

// R <- exp(dr) R on SO(3), or the additive rotation vector without dofs_SO3
// (ExplicitModule::updateVec, :362-392)
template <class T>
__device__ __forceinline__ Q4<double> milne_rotate(const DevModel<T> &m, const Q4<double> &R, const V3<double> &dr) {
  if (m.so3) return qnormalize(qmul(qexp_small(dr), R));
  return qexp(qlog(R) + dr);
}

__device__ __forceinline__ void milne_sum_forces(const float *ef, int i0, int i1, double f[6]) {
  for (int i = i0; i < i1; ++i) load_end(ef + static_cast<size_t>(i) * 6, f);
}
__device__ __forceinline__ void milne_sum_forces(const double *ef, int i0, int i1, double f[6]) {
  for (int i = i0; i < i1; ++i) load_end(ef + static_cast<size_t>(i) * 6, f);
}

template <class T, class Y>
__global__ void __launch_bounds__(256, Y::kMinBlocks)
    k_milne(const __grid_constant__ DevModel<T> m, const __grid_constant__ SampleSpec smp, const StepCtx c,
            GridBarrier *bar, const __grid_constant__ MilneDev<T> md) {
  __shared__ double s_scale[kMilneMaxScales];
  __shared__ double s_dec[3];
  const BarrierState bs = barrier_begin(bar);
  if (blockIdx.x == 0 && threadIdx.x < 5) c.next_energy[threadIdx.x] = 0.0;
  const int gtid = blockIdx.x * blockDim.x + threadIdx.x;
  const int gstride = gridDim.x * blockDim.x;
  const int N = m.N, E = m.E, G = m.G;
  const int nh = Y::kNh >= 0 ? Y::kNh : m.nh;
  const HistOut<T> ho{md.ep_new, md.alpha_new, md.epsc_new, md.ediss_new};
  double t = md.ctl->t, dt = md.ctl->dt;
  int64_t step = md.ctl->step, rejected = md.ctl->rejected;
  const double inv_rms = 1.0 / sqrt(6.0 * double(N));
  int64_t done = 0;
  int attempts = 0;
  bool acc_prev = false;
  // take over the trial history of an accepted step (each element's own thread)
  auto commit_history = [&]() {
    if constexpr (Y::kPlastic) {
      if (!m.plastic) return;
      for (int e = gtid; e < E; e += gstride)
        for (int g = 0; g < G; ++g) {
          for (int k = 0; k < 6; ++k) {
            m.ep[(g * 6 + k) * E + e] = md.ep_new[(g * 6 + k) * E + e];
            m.epsc[(g * 6 + k) * E + e] = md.epsc_new[(g * 6 + k) * E + e];
          }
          for (int a = 0; a < nh; ++a) m.alpha[(g * nh + a) * E + e] = md.alpha_new[(g * nh + a) * E + e];
          m.ediss[g * E + e] = md.ediss_new[g * E + e];
        }
    }
  };
  while (done < c.nsteps) {
    const int64_t snext = step + 1;
    const double tn = t + dt;
    const int64_t sidx = sample_index(smp, c, snext);
    const bool last = (done + 1 == c.nsteps);
    const bool energy = (sidx >= 0) || last;
    const double4 *pos_cur = acc_prev ? md.pos_pre : m.pos;
    const double4 *rot_cur = acc_prev ? md.rot_pre : m.rot;
    const double *vel_cur = acc_prev ? md.vel_pre : m.vel;
    // ---- A: force at the current state
    if (acc_prev) commit_history();
    {
      ElemEnergy en;
      for (int e = gtid; e < E; e += gstride)
        element_force<T, Y, false, HM_TRIAL>(m, e, true, false, en, false, -1, pos_cur, rot_cur, nullptr);
    }
    if (!grid_barrier(bar, bs, m.err)) return;
    // ---- A': loads at t + dt, prediction
    if (threadIdx.x == 0 && md.n_scales > 0) {
      double regs[kMaxExprRegs];
      const double args[3] = {tn, double(snext), dt};
      run_prog(md.scale_prog, args, regs);
      for (int s = 0; s < md.n_scales; ++s) s_scale[s] = regs[md.scale_prog.outs[s]];
    }
    if (blockIdx.x == 0 && threadIdx.x < 5 && energy) {  // energy slots of this attempt
      if (sidx >= 0) smp.energy[sidx * 5 + threadIdx.x] = 0.0;
      if (last) c.last_energy[threadIdx.x] = 0.0;
    }
    __syncthreads();
    for (int n = gtid; n < N; n += gstride) {
      double v[6];
#pragma unroll
      for (int k = 0; k < 6; ++k) v[k] = vel_cur[k * N + n];
      const V3<double> x = ldx(pos_cur + n);
      const Q4<double> R = ldq(rot_cur + n);
      if (acc_prev) {  // the accepted state becomes the current one
#pragma unroll
        for (int k = 0; k < 6; ++k) m.vel[k * N + n] = v[k];
        m.pos[n] = make_double4(x.x, x.y, x.z, 0.0);
        m.rot[n] = make_double4(R.w, R.x, R.y, R.z);
      }
      double f[6] = {0, 0, 0, 0, 0, 0}, fx[6] = {0, 0, 0, 0, 0, 0}, a[6] = {0, 0, 0, 0, 0, 0};
      milne_sum_forces(m.ef, m.slot_ptr[n], m.slot_ptr[n + 1], f);
      const unsigned mask = milne_bcs(m, n, s_scale, fx, a);
      milne_accel(m, n, R, V3<double>{v[3], v[4], v[5]}, f, fx, mask, a);
      const V3<double> xp = x + dt * V3<double>{v[0], v[1], v[2]};
      const Q4<double> Rp = milne_rotate(m, R, dt * V3<double>{v[3], v[4], v[5]});
#pragma unroll
      for (int k = 0; k < 6; ++k) md.vel_pre[k * N + n] = v[k] + dt * a[k];
      md.pos_pre[n] = make_double4(xp.x, xp.y, xp.z, 0.0);
      md.rot_pre[n] = make_double4(Rp.w, Rp.x, Rp.y, Rp.z);
    }
    if (!grid_barrier(bar, bs, m.err)) return;
    // ---- B: force at the predicted state, trial history
    {
      ElemEnergy en;
      for (int e = gtid; e < E; e += gstride)
        element_force<T, Y, false, HM_STORE>(m, e, true, energy, en, false, -1, md.pos_pre, md.rot_pre, &ho);
      if (energy) {
        const double p = block_sum<T>(en.pot);
        const double d = block_sum<T>(en.diss);
        if (threadIdx.x == 0) {
          if (sidx >= 0) {
            atomicAdd(smp.energy + sidx * 5 + 1, p);
            atomicAdd(smp.energy + sidx * 5 + 2, d);
          }
          if (last) {
            atomicAdd(c.last_energy + 1, p);
            atomicAdd(c.last_energy + 2, d);
          }
        }
      }
    }
    if (!grid_barrier(bar, bs, m.err)) return;
    // ---- B': correction and the error sums
    double su = 0.0, sv = 0.0, wx = 0.0, ek = 0.0;
    for (int n = gtid; n < N; n += gstride) {
      double v[6], vp[6];
#pragma unroll
      for (int k = 0; k < 6; ++k) {
        v[k] = m.vel[k * N + n];
        vp[k] = md.vel_pre[k * N + n];
      }
      const V3<double> x = ldx(m.pos + n);
      const Q4<double> R = ldq(m.rot + n), Rp = ldq(md.rot_pre + n);
      double f[6] = {0, 0, 0, 0, 0, 0}, fx[6] = {0, 0, 0, 0, 0, 0}, a[6] = {0, 0, 0, 0, 0, 0};
      milne_sum_forces(m.ef, m.slot_ptr[n], m.slot_ptr[n + 1], f);
      const unsigned mask = milne_bcs(m, n, s_scale, fx, a);
      milne_accel(m, n, R, V3<double>{vp[3], vp[4], vp[5]}, f, fx, mask, a);
      double vn[6];
#pragma unroll
      for (int k = 0; k < 6; ++k) vn[k] = v[k] + dt * a[k];
      const V3<double> du{dt * vp[0], dt * vp[1], dt * vp[2]};
      const V3<double> dr{dt * vp[3], dt * vp[4], dt * vp[5]};
      const V3<double> xn = x + du;
      const Q4<double> Rn = milne_rotate(m, R, dr);
      // getQuality: translations over lengthScale; rotation vectors (and
      // angular velocities) unscaled on SO(3).  x_pre - x_new is evaluated as
      // dt (v - v_pre), its exact value: the node positions are absolute
      // coordinates, whose rounding would swamp the difference, where the
      // reference subtracts displacements.
      const double ls = 1.0 / md.len_scale, lr = m.so3 ? 1.0 : ls;
      const V3<double> dx = (ls * dt) * V3<double>{v[0] - vp[0], v[1] - vp[1], v[2] - vp[2]};
      const V3<double> dth = lr * (qlog(Rp) - qlog(Rn));
      su += dot(dx, dx) + dot(dth, dth);
#pragma unroll
      for (int k = 0; k < 6; ++k) {
        const double dv = (k < 3 ? ls : lr) * (vp[k] - vn[k]);
        sv += dv * dv;
      }
      wx += fx[0] * du.x + fx[1] * du.y + fx[2] * du.z + fx[3] * dr.x + fx[4] * dr.y + fx[5] * dr.z;
      if (energy) {  // E_kin with the mass of the step's start
        const Q4<double> RPc = qconj(qmul(R, toq(m.iframe[n])));
        const auto Dv = m.idiag[n];
        const V3<double> wl = qrot(RPc, V3<double>{vn[3], vn[4], vn[5]});
        ek += 0.5 * (m.mass[n] * (vn[0] * vn[0] + vn[1] * vn[1] + vn[2] * vn[2]) + double(Dv.x) * wl.x * wl.x +
                     double(Dv.y) * wl.y * wl.y + double(Dv.z) * wl.z * wl.z);
      }
      bool finite = true;
#pragma unroll
      for (int k = 0; k < 6; ++k) finite = finite && isfinite(vn[k]);
      if (!finite) atomicOr(m.err, 0x2u);
#pragma unroll
      for (int k = 0; k < 6; ++k) md.vel_pre[k * N + n] = vn[k];
      md.pos_pre[n] = make_double4(xn.x, xn.y, xn.z, 0.0);
      md.rot_pre[n] = make_double4(Rn.w, Rn.x, Rn.y, Rn.z);
      if (sidx >= 0 && smp.n_watch > 0) {
        const int slot = smp.watch_slot[n];
        if (slot >= 0) {
          double *o = smp.rows + (sidx * smp.n_watch + slot) * 13;
          o[0] = xn.x; o[1] = xn.y; o[2] = xn.z;
          o[3] = Rn.w; o[4] = Rn.x; o[5] = Rn.y; o[6] = Rn.z;
#pragma unroll
          for (int k = 0; k < 6; ++k) o[7 + k] = vn[k];
        }
      }
    }
    {
      const double bu = block_sum<T>(su);
      const double bv = block_sum<T>(sv);
      const double bw = block_sum<T>(wx);
      const double bk = energy ? block_sum<T>(ek) : 0.0;
      if (threadIdx.x == 0) {
        md.partial[blockIdx.x * 3 + 0] = bu;
        md.partial[blockIdx.x * 3 + 1] = bv;
        md.partial[blockIdx.x * 3 + 2] = bw;
        if (energy) {
          if (sidx >= 0) atomicAdd(smp.energy + sidx * 5 + 0, bk);
          if (last) atomicAdd(c.last_energy + 0, bk);
        }
      }
    }
    if (!grid_barrier(bar, bs, m.err)) return;
    // ---- decision: the same sums in the same order in every block
    {
      double pu = 0.0, pv = 0.0, pw = 0.0;
      for (int b = threadIdx.x; b < gridDim.x; b += blockDim.x) {
        pu += md.partial[b * 3 + 0];
        pv += md.partial[b * 3 + 1];
        pw += md.partial[b * 3 + 2];
      }
      pu = block_sum<T>(pu);
      pv = block_sum<T>(pv);
      pw = block_sum<T>(pw);
      if (threadIdx.x == 0) {
        s_dec[0] = pu;
        s_dec[1] = pv;
        s_dec[2] = pw;
      }
      __syncthreads();
      pu = s_dec[0];
      pv = s_dec[1];
      pw = s_dec[2];
      __syncthreads();
      const double error = 0.5 * (sqrt(pu) * inv_rms + sqrt(pv) * inv_rms * dt);
      if (!isfinite(error) || ++attempts > kMilneMaxAttempts) {
        if (blockIdx.x == 0 && threadIdx.x == 0) atomicOr(m.err, 0x40u);
        return;
      }
      const double dt_opt = dt * sqrt(md.prec / error);  // (prec / error)^(1 / (order + 1)), order 1
      const bool accept = error <= md.prec || dt <= md.min_dt;
      if (accept) {
        const double dt_next = fmax(fmax(fmin(fmin(md.safety * dt_opt, md.incr * dt), md.max_dt), md.decr * dt),
                                    md.min_dt);
        t = tn;
        step = snext;
        ++done;
        attempts = 0;
        if (blockIdx.x == 0 && threadIdx.x == 0) {
          const double w = *md.wext + pw;
          *md.wext = w;
          if (sidx >= 0) {
            smp.energy[sidx * 5 + 3] = w;
            smp.steps[sidx] = snext;
            if (smp.times) smp.times[sidx] = tn;
          }
          if (last) c.last_energy[3] = w;
        }
        dt = dt_next;
      } else {
        dt = fmax(fmax(md.safety * dt_opt, md.decr * dt), md.min_dt);
        ++rejected;
      }
      acc_prev = accept;
    }
  }
  // the last accepted step becomes the current state
  if (acc_prev) {
    commit_history();
    for (int n = gtid; n < N; n += gstride) {
#pragma unroll
      for (int k = 0; k < 6; ++k) m.vel[k * N + n] = md.vel_pre[k * N + n];
      m.pos[n] = md.pos_pre[n];
      m.rot[n] = md.rot_pre[n];
    }
  }
  if (blockIdx.x == 0 && threadIdx.x == 0) {
    md.ctl->t = t;
    md.ctl->dt = dt;
    md.ctl->step = step;
    md.ctl->rejected = rejected;
  }
}

}  // namespace dl
