// Engine handle and C ABI (include/dynlattice.h).
//
// A handle owns the device arrays of one lattice in the layout of engine.hpp.
// dl_run advances the state with the persistent kernel (default) or with
// per-phase launches; host work per dl_run call is the per-step table of load
// scale functions for the steps of the call (JIVE LoadScale / Dirichlet /
// Neumann time dependence, evaluated in FP64 on the host as the reference
// does) and at most a few small copies.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <memory>
#include <mutex>
#include <stdexcept>
#include <string>
#include <vector>

#include "../../include/dynlattice.h"
#include "engine.hpp"
#include "jit.hpp"
#include "noalloc.hpp"
#include "output.hpp"
#include "pro.hpp"
#include "rodkin.cuh"
#include "setup.hpp"
#include "contact_build.hpp"

namespace dl {

thread_local std::string g_last_error;

#define DL_CUDA(call)                                                                        \
  do {                                                                                       \
    cudaError_t _e = (call);                                                                 \
    if (_e != cudaSuccess) {                                                                 \
      cudaGetLastError(); /* non-sticky errors must not leak into later calls */             \
      throw ::dl::CudaError(std::string(#call) + ": " + cudaGetErrorString(_e));             \
    }                                                                                        \
  } while (0)

cudaMemPool_t retained_pool() {
  static std::mutex mu;
  static std::vector<cudaMemPool_t> pools;
  int dev = 0;
  DL_CUDA(cudaGetDevice(&dev));
  std::lock_guard<std::mutex> lock(mu);
  if (static_cast<int>(pools.size()) <= dev) pools.resize(dev + 1, nullptr);
  if (!pools[dev]) {
    cudaMemPoolProps props{};
    props.allocType = cudaMemAllocationTypePinned;
    props.location.type = cudaMemLocationTypeDevice;
    props.location.id = dev;
    cudaMemPool_t pool = nullptr;
    DL_CUDA(cudaMemPoolCreate(&pool, &props));
    uint64_t keep = ~uint64_t(0);
    DL_CUDA(cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &keep));
    pools[dev] = pool;
  }
  return pools[dev];
}

void trim_retained_pool() { DL_CUDA(cudaMemPoolTrimTo(retained_pool(), 0)); }

// Per-step states of one checkpoint segment, recorded by the forward kernel
// and read by the reverse sweep: node positions, rotations, velocities and
// the plastic history of every Gauss point.
struct StateTape {
  PoolBuf pos, rot, vel, ep, al, epsc;
};

template <class T>
static void upload(DevBuf &b, const std::vector<T> &v) {
  b.alloc(v.size() * sizeof(T));
  if (!v.empty()) DL_CUDA(cudaMemcpy(b.p, v.data(), v.size() * sizeof(T), cudaMemcpyHostToDevice));
}
// convert a double host vector to T on upload
template <class T>
static void upload_as(DevBuf &b, const std::vector<double> &v) {
  std::vector<T> t(v.begin(), v.end());
  upload(b, t);
}

struct EngineBase {
  virtual ~EngineBase() = default;
  std::unique_ptr<HostLattice> host;
  int precision = DL_PLAIN_FP64;
  int device = 0;  // the CUDA device current when the handle was created
  cudaStream_t stream = nullptr;
  int exec_mode = EXEC_PERSISTENT;
  int64_t step = 0;
  double t = 0.0;
  // sampling
  int every = 0;
  std::vector<int32_t> watch;   // original numbering
  int64_t capacity = 0;
  int64_t n_samples = 0;
  dl_energies last{};
  virtual void run(int64_t nsteps) = 0;
  virtual void info(int32_t *jit, int32_t *blocks, const char **log) = 0;
  virtual void fetch_last_energies() = 0;
  virtual void set_sampling(int every, const std::vector<int32_t> &watch, int64_t capacity) = 0;
  virtual void get_samples(int64_t *n, int64_t *steps, double *rows, dl_energies *en, int64_t max) = 0;
  virtual void get_state(double *u, double *th, double *v) = 0;
  virtual void set_state(const double *u, const double *th, const double *v) = 0;
  virtual void internal_force(const double *u, const double *th, double *fint) = 0;
  virtual int internal_force_static(const double *u, const double *th, double *fint, const char **why) = 0;
  virtual void get_history(double *ep, double *hp, double *ed) = 0;
  virtual uint32_t error_word() = 0;
  virtual void group_sums(int n, const int32_t *nodes, double *resp, double *load) = 0;
  virtual void batch_energies(int lat, dl_energies *e) = 0;
  virtual void contact_pairs(int64_t *n, int32_t *pairs, double *gaps, int64_t max) = 0;
  virtual void joint_contact_pairs(int64_t *n, int32_t *pairs, double *gaps, int64_t max) = 0;
  virtual void element_table(const std::string &name, double *out) = 0;
  virtual void plate_reaction(double *out) = 0;
  virtual void contact_stats(int64_t *cand, int64_t *builds) = 0;
  virtual int64_t launch_count() = 0;
  virtual void set_tape_budget(int64_t bytes) = 0;
  virtual void autotune(int64_t steps, int32_t *best_mode, int32_t *best_tpb, double *best_ms) = 0;
  virtual void set_threads(int tpb) = 0;
  virtual void set_group_output(bool on) = 0;
  virtual void set_integrator(const dl_integrator_desc &d) = 0;
  virtual bool adaptive() const = 0;
  // external loads [N][6] (original numbering) at the current time
  void external_force(double *f) {
    HostLattice &h = *host;
    double dt = 0.0;
    get_time(nullptr, &dt, nullptr, nullptr);
    std::fill(f, f + static_cast<size_t>(h.N) * 6, 0.0);
    for (int ni = 0; ni < h.N; ++ni)
      for (int b = h.bc_ptr[ni]; b < h.bc_ptr[ni + 1]; ++b) {
        const BcTerm &bt = h.bc[b];
        if (bt.kind != BCD_NEUMANN) continue;
        double sc = 1.0;
        if (bt.scale >= 0) {
          const double vars[3] = {t, static_cast<double>(step), dt};
          sc = evalExpr(h.scales[bt.scale].expr.get(), vars);
        }
        f[static_cast<size_t>(h.node_old[ni]) * 6 + bt.dof] += bt.factor * sc;
      }
  }
  virtual void get_time(double *t, double *dt, int64_t *step, int64_t *rejected) = 0;
  std::vector<double> sample_t;  // time of each recorded sample
  virtual void adjoint_radius(int64_t nsteps, int K, int n_params, const int32_t *elem_param, int n_react,
                              const int32_t *react_nodes, int react_dof, double react_w, double *J,
                              double *grad) = 0;
  // failure-path hooks: bound of one grid-barrier wait and blocks the
  // barrier expects beyond the launch's own; clearing the error word
  virtual void set_barrier_test(uint32_t limit_us, uint32_t phantom) = 0;
  virtual void clear_error() = 0;
  // return-map branch tape of the next dl_adjoint_radius forward run
  int br_mode = 0;                 // 0 off, 1 record, 2 impose
  std::vector<uint8_t> br_host;    // recorded / imposed iteration counts [nsteps][G][E]
  int64_t br_peak_step = -1;       // peak step of the recorded run (relative to its start) ...
  double br_peak_sign = 1.0;       // ... and the sign of the group force there
};

template <class T>
struct Engine final : EngineBase {
  using T4 = typename Vec4<T>::type;
  DevModel<T> m;
  DevBuf pos, rot, vel, mass, imass, iframe, idiag, idinv, slot_ptr, bc_ptr, bc, madd;
  DevBuf conn, eslot, invL0, L0, qN, g0, k0, C, ec, ep, alpha, epsc, ediss, ef, cstamp;
  DevBuf conn_n, eslot_n, shp, s0_n;  // elements of 3 or 4 nodes
  DevBuf yops, yconsts, gops, gconsts, gouts;
  DevBuf err, wext_dev, scales, wstep, energy_slots, barrier;
  // adjoint: checkpoints, tape of one segment, adjoint state, objective group
  PoolBuf ck_pos, ck_rot, ck_vel, ck_ep, ck_al, ck_epsc, ck_ediss;
  // state tapes: two sets, so that the recomputation of one checkpoint
  // segment overlaps the reverse sweep over the next one
  StateTape tape[2];
  // the reverse sweep's stream (non-blocking, highest priority: it is the
  // critical path) and the events ordering it against the recomputation
  cudaStream_t rstream = nullptr;
  cudaEvent_t ev_ready[2] = {nullptr, nullptr}, ev_free[2] = {nullptr, nullptr}, ev_join = nullptr;
  DevBuf a_lx, a_lth, a_lv, a_lf, a_aslot, a_lep, a_lal, a_lepsc, a_lC, a_lec, a_lmass, a_lS;
  DevBuf grp_flag_dev, grp_hist_dev, br_dev, tie_ptr_dev, tie_nodes_dev;
  int64_t adj_launches = 0;
  int64_t tape_budget = -1;   // bytes for the adjoint's state tape (-1: half the free memory)
  double *pinned_scales = nullptr;
  double *pinned_energy = nullptr;  // [5] staging of dl_get_energies
  cudaEvent_t staged_event = nullptr;
  bool staged_event_pending = false;
  bool has_neumann = false;
  int64_t launches = 0;
  int last_slot = 0;
  DevBuf s_slot, s_rows, s_energy, s_steps, s_count;
  DevBuf X0dev, node_old_dev, xfer;
  DevBuf dtn_dev, nlat_dev, elat_dev, lat_energy;
  ContactList clist;
  JointList jlist;
  DevBuf pair_gap, jpair_gap, plate_force, fint_last;
  bool contact_on = false;
  bool joint_on = false;     // joint contact (JointContactModel)
  int64_t list_budget = 0;   // steps the current contact candidate list stays valid
  double plate_speed = 0.0;  // fastest rigid plate
  int64_t list_builds = 0;
  int64_t kernel_launches = 0;  // step and utility kernels issued by run()
  KernelSet kernels;
  std::string jit_log;
  int64_t scale_capacity = 0;
  // MilneDevice predictor-corrector (dl_set_integrator)
  dl_integrator_desc integ{};
  MilneDev<T> md{};
  DevBuf mi_pos, mi_rot, mi_vel, mi_ep, mi_al, mi_epsc, mi_ediss, mi_partial, mi_ctl, mi_ops, mi_consts, mi_outs;
  DevBuf s_times;
  double cur_dt = 0.0;      // the time step of the next step
  int64_t rejected = 0;

  explicit Engine(std::unique_ptr<HostLattice> hl, int prec) {
    host = std::move(hl);
    precision = prec;
    DL_CUDA(cudaGetDevice(&device));
    HostLattice &h = *host;
    const int N = h.N, E = h.E, G = h.G;
    m.N = N;
    m.E = E;
    m.G = G;
    m.nh = h.nh;
    m.plastic = h.plastic ? 1 : 0;
    m.gyro = h.gyro ? 1 : 0;
    m.lumped = h.lumped ? 1 : 0;
    if (h.ties) {
      upload(tie_ptr_dev, h.tie_ptr);
      upload(tie_nodes_dev, h.tie_nodes);
      m.tie_ptr = tie_ptr_dev.as<int32_t>();
      m.tie_nodes = tie_nodes_dev.as<int32_t>();
    }
    m.so3 = h.so3 ? 1 : 0;
    m.dt = h.dt;
    // nodes
    upload(pos, h.pos);
    upload(rot, h.rot);
    upload(vel, h.vel);
    upload(mass, h.mass);
    upload_as<T>(iframe, h.iframe);
    upload_as<T>(idiag, h.idiag);
    {
      std::vector<double> inv(h.idiag.size(), 0.0), im(h.mass.size());
      for (size_t i = 0; i < h.idiag.size(); ++i)
        if (i % 4 != 3) inv[i] = 1.0 / h.idiag[i];
      for (size_t i = 0; i < h.mass.size(); ++i) im[i] = 1.0 / h.mass[i];
      upload_as<T>(idinv, inv);
      upload(imass, im);
    }
    upload(slot_ptr, h.slot_ptr);
    upload(bc_ptr, h.bc_ptr);
    upload(bc, h.bc);
    if (!h.madd.empty()) {
      upload(madd, h.madd);
      m.madd = madd.as<double>();
    }
    m.pos = pos.as<double4>();
    m.rot = rot.as<double4>();
    m.vel = vel.as<double>();
    m.mass = mass.as<double>();
    m.iframe = iframe.as<T4>();
    m.idiag = idiag.as<T4>();
    m.idinv = idinv.as<T4>();
    m.imass = imass.as<double>();
    m.slot_ptr = slot_ptr.as<int32_t>();
    m.bc_ptr = bc_ptr.as<int32_t>();
    m.bc = bc.as<BcTerm>();
    // elements
    upload(conn, h.conn);
    upload(eslot, h.eslot);
    upload(invL0, h.invL0);
    {
      std::vector<double> l0(h.invL0.size());
      for (size_t i = 0; i < l0.size(); ++i) l0[i] = 1.0 / h.invL0[i];
      upload_as<T>(L0, l0);
    }
    upload_as<T>(qN, h.qN);
    upload_as<T>(g0, h.g0);
    upload_as<T>(k0, h.k0);
    upload_as<T>(C, h.C);
    upload_as<T>(ec, h.ec);
    m.conn = conn.as<int2>();
    m.eslot = eslot.as<int2>();
    m.invL0 = invL0.as<double>();
    m.L0 = L0.as<T>();
    m.qN = qN.as<T4>();
    m.g0 = g0.as<T>();
    m.k0 = k0.as<T>();
    m.C = C.as<T>();
    m.ec = ec.as<T>();
    m.nen = h.nen;
    if (h.nen > 2) {
      upload(conn_n, h.conn_n);
      upload(eslot_n, h.eslot_n);
      upload(shp, h.shp);
      m.conn_n = conn_n.as<int32_t>();
      m.eslot_n = eslot_n.as<int32_t>();
      m.shp = shp.as<double>();
      std::vector<double> s0(static_cast<size_t>(G) * 6 * E);
      for (int g = 0; g < G; ++g)
        for (int k = 0; k < 3; ++k)
          for (int e = 0; e < E; ++e) {
            s0[(static_cast<size_t>(g) * 6 + k) * E + e] = h.g0[(static_cast<size_t>(g) * 3 + k) * E + e];
            s0[(static_cast<size_t>(g) * 6 + 3 + k) * E + e] = h.k0[(static_cast<size_t>(g) * 3 + k) * E + e];
          }
      upload(s0_n, s0);
      m.s0_n = s0_n.as<double>();
    }
    for (int a = 0; a < 4; ++a)
      for (int g = 0; g < 4; ++g) m.Nq[a][g] = h.Nq[a][g];
    if (h.plastic) {
      const size_t NG = static_cast<size_t>(E) * G;
      ep.alloc(NG * 6 * sizeof(T));
      DL_CUDA(cudaMemset(ep.p, 0, ep.bytes));
      alpha.alloc(NG * std::max(1, h.nh) * sizeof(T));
      DL_CUDA(cudaMemset(alpha.p, 0, alpha.bytes));
      epsc.alloc(NG * 6 * sizeof(T));
      DL_CUDA(cudaMemset(epsc.p, 0, epsc.bytes));
      ediss.alloc(NG * sizeof(double));
      DL_CUDA(cudaMemset(ediss.p, 0, ediss.bytes));
      m.ep = ep.as<T>();
      m.alpha = alpha.as<T>();
      m.epsc = epsc.as<T>();
      m.ediss = ediss.as<double>();
      upload(yops, h.yield.ops);
      upload_as<T>(yconsts, h.yield.consts);
      upload(gops, h.grad.ops);
      upload_as<T>(gconsts, h.grad.consts);
      upload(gouts, h.grad.outputs);
      m.yield.ops = yops.as<ExprOp>();
      m.yield.consts = yconsts.as<T>();
      m.yield.n_ops = static_cast<int>(h.yield.ops.size());
      m.yield.out0 = h.yield.outputs[0];
      m.grad.ops = gops.as<ExprOp>();
      m.grad.consts = gconsts.as<T>();
      m.grad.n_ops = static_cast<int>(h.grad.ops.size());
      m.grad.outs = gouts.as<uint8_t>();
      for (int a = 0; a < 7; ++a)
        for (int b = 0; b < 7; ++b) m.H[a][b] = T(h.H[a][b]);
      m.max_iter = h.max_iter;
      m.prec = T(h.prec);
    }
    ef.alloc(static_cast<size_t>(E) * 6 * h.nen * sizeof(T));  // one 6-value slot per element node
    DL_CUDA(cudaMemset(ef.p, 0, ef.bytes));
    m.ef = ef.as<T>();
    err.alloc(sizeof(uint32_t));
    DL_CUDA(cudaMemset(err.p, 0, err.bytes));
    m.err = err.as<uint32_t>();
    {
      std::vector<double> x0i(static_cast<size_t>(N) * 3);
      for (int i = 0; i < N; ++i)
        for (int k = 0; k < 3; ++k) x0i[static_cast<size_t>(i) * 3 + k] = h.X0[static_cast<size_t>(h.node_old[i]) * 3 + k];
      upload(X0dev, x0i);
      upload(node_old_dev, h.node_old);
      xfer.alloc(static_cast<size_t>(N) * 12 * sizeof(double));
    }
    if (h.n_lat > 1) {
      upload(dtn_dev, h.dtn);
      upload(nlat_dev, h.nlat);
      upload(elat_dev, h.elat);
      lat_energy.alloc(static_cast<size_t>(h.n_lat) * 5 * sizeof(double));
      DL_CUDA(cudaMemset(lat_energy.p, 0, lat_energy.bytes));
      m.n_lat = h.n_lat;
      m.dtn = dtn_dev.as<double>();
      m.nlat = nlat_dev.as<int32_t>();
      m.elat = elat_dev.as<int32_t>();
      m.lat_energy = lat_energy.as<double>();
    }
    energy_slots.alloc(10 * sizeof(double));
    DL_CUDA(cudaMemset(energy_slots.p, 0, energy_slots.bytes));
    // rod--rod contact and rigid plates
    const dl_contact_desc &cd = h.contact;
    if (cd.enabled || cd.n_plates > 0) {
      if (!(cd.radius > 0.0)) throw std::invalid_argument("contact radius must be positive");
      if (cd.n_plates < 0 || cd.n_plates > 2) throw std::invalid_argument("at most two plates");
      m.c_radius = cd.radius;
      m.n_plates = cd.n_plates;
      for (int p = 0; p < cd.n_plates; ++p) {
        for (int k = 0; k < 3; ++k) {
          m.plate_n[p][k] = cd.plates[p].normal[k];
          m.plate_p0[p][k] = cd.plates[p].point0[k];
          m.plate_v[p][k] = cd.plates[p].velocity[k];
        }
        m.plate_k[p] = cd.plates[p].penalty;
        const double *pv = cd.plates[p].velocity;
        plate_speed = std::max(plate_speed, std::sqrt(pv[0] * pv[0] + pv[1] * pv[1] + pv[2] * pv[2]));
      }
      plate_force.alloc(6 * sizeof(double));
      DL_CUDA(cudaMemset(plate_force.p, 0, plate_force.bytes));
      m.plate_force = plate_force.as<double>();
      if (cd.enabled) {
        contact_on = true;
        m.c_ks = cd.penalty_sts;
        m.c_kn = cd.penalty_nts;
        clist.init(h, stream);
        clist.init_blacklist(m.pos, m.conn);
        m.half_margin = 0.5 * clist.margin;
      }
    }
    if (h.jcontact.enabled) {
      joint_on = true;
      m.j_radius = h.jcontact.radius;
      m.j_k = h.jcontact.penalty;
      jlist.init(h, stream);
      m.half_margin = 0.5 * list_margin();
    }
    if (contact_on || joint_on) {
      cstamp.alloc(static_cast<size_t>(N) * sizeof(int64_t));
      DL_CUDA(cudaMemset(cstamp.p, 0xff, cstamp.bytes));  // -1: no closed pair yet
      m.cstamp = cstamp.as<int64_t>();
    }
    wext_dev.alloc(sizeof(double));
    DL_CUDA(cudaMemset(wext_dev.p, 0, wext_dev.bytes));
    for (const BcTerm &bt : h.bc) has_neumann = has_neumann || (bt.kind == BCD_NEUMANN);
    if (has_neumann) {
      wstep.alloc(1024 * sizeof(double));
      DL_CUDA(cudaMemset(wstep.p, 0, wstep.bytes));
    }
    DL_CUDA(cudaEventCreateWithFlags(&staged_event, cudaEventDisableTiming));
    barrier.alloc(sizeof(GridBarrier));
    DL_CUDA(cudaMemset(barrier.p, 0, barrier.bytes));
    m.n_scales = static_cast<int>(h.scales.size());
    kernels = aot_kernels<T>(h.plastic);
    // elastoplastic lattices: compile the yield function into the kernels
    const char *nojit = std::getenv("DL_NO_JIT");
    if (h.plastic && !(nojit && nojit[0] == '1')) {
      const std::string code = emitYieldPolicy(h.yield_expr, h.grad_exprs, sizeof(T) == 4);
      const KernelSet *ks = jit_kernels(code, sizeof(T) == 4, &jit_log);
      if (ks) kernels = *ks;
    }
    set_sampling(0, {}, 0);
  }

  ~Engine() override {
    if (stream) cudaStreamSynchronize(stream);
    else cudaDeviceSynchronize();
    graph_release();
    if (rstream) cudaStreamSynchronize(rstream);
    if (own_stream) cudaStreamDestroy(own_stream);
    if (rstream) cudaStreamDestroy(rstream);
    for (cudaEvent_t ev : {ev_ready[0], ev_ready[1], ev_free[0], ev_free[1], ev_join})
      if (ev) cudaEventDestroy(ev);
    if (pinned_scales) cudaFreeHost(pinned_scales);
    if (pinned_energy) cudaFreeHost(pinned_energy);
    if (staged_event) cudaEventDestroy(staged_event);
  }

  void ensure_scale_table(int64_t nsteps) {
    if (m.n_scales == 0) return;
    if (nsteps > scale_capacity) {
      DL_CUDA(cudaStreamSynchronize(stream));
      staged_event_pending = false;
      scales.alloc(static_cast<size_t>(nsteps) * m.n_scales * sizeof(double));
      if (pinned_scales) cudaFreeHost(pinned_scales);
      pinned_scales = nullptr;
      DL_CUDA(cudaMallocHost(reinterpret_cast<void **>(&pinned_scales),
                             static_cast<size_t>(nsteps) * m.n_scales * sizeof(double)));
      scale_capacity = nsteps;
    }
  }

  void set_sampling(int ev, const std::vector<int32_t> &w, int64_t cap) override {
    HostLattice &h = *host;
    every = ev;
    watch = w;
    capacity = cap;
    n_samples = 0;
    if (stream) DL_CUDA(cudaStreamSynchronize(stream));
    std::vector<int32_t> slot(h.N, -1);
    for (size_t i = 0; i < w.size(); ++i) {
      if (w[i] < 0 || w[i] >= h.N) throw std::invalid_argument("watch node out of range");
      slot[h.node_new[w[i]]] = static_cast<int32_t>(i);
    }
    upload(s_slot, slot);
    s_rows.alloc(static_cast<size_t>(std::max<int64_t>(cap, 1)) * std::max<size_t>(w.size(), 1) * 13 * sizeof(double));
    s_energy.alloc(static_cast<size_t>(std::max<int64_t>(cap, 1)) * 5 * sizeof(double));
    DL_CUDA(cudaMemset(s_energy.p, 0, s_energy.bytes));
    s_steps.alloc(static_cast<size_t>(std::max<int64_t>(cap, 1)) * sizeof(int64_t));
    s_times.alloc(static_cast<size_t>(std::max<int64_t>(cap, 1)) * sizeof(double));
    sample_t.clear();
  }

  SampleSpec sample_spec() {
    SampleSpec s;
    s.every = every;
    s.n_watch = static_cast<int>(watch.size());
    s.watch_slot = s_slot.as<int32_t>();
    s.rows = s_rows.as<double>();
    s.energy = s_energy.as<double>();
    s.steps = s_steps.as<int64_t>();
    s.capacity = capacity;
    s.times = s_times.as<double>();
    return s;
  }

  // ---- CUDA graph of one launch (exec mode 2) -------------------------------
  // The launch sequence of a block of n steps (energy-slot clear, persistent
  // step kernel, external-work finisher) is captured per block and, when the
  // block has the shape of the previous one, applied to the instantiated
  // graph as an in-place update (new step number, sample base, energy slots)
  // instead of a new instantiation.
  cudaGraph_t graph = nullptr;
  cudaGraphExec_t graph_exec = nullptr;
  int graph_n = -1;
  int64_t graph_replays = 0;

  void graph_release() {
    if (graph_exec) cudaGraphExecDestroy(graph_exec);
    if (graph) cudaGraphDestroy(graph);
    graph_exec = nullptr;
    graph = nullptr;
    graph_n = -1;
  }

  cudaStream_t own_stream = nullptr;

  template <class F>
  void graph_launch(int n, F &&enqueue, const StepCtx &c, const SampleSpec &smp) {
    (void)c;
    (void)smp;
    if (!stream) {
      // the legacy default stream cannot be captured: work on a blocking
      // stream of the engine's own (ordered with the legacy stream)
      if (!own_stream) DL_CUDA(cudaStreamCreate(&own_stream));
      stream = own_stream;
      clist.stream = stream;
      jlist.stream = stream;
    }
    // capture this block's launch sequence; a graph of the same shape is
    // updated in place (new kernel arguments), otherwise instantiated
    cudaGraph_t g = nullptr;
    DL_CUDA(cudaStreamBeginCapture(stream, cudaStreamCaptureModeThreadLocal));
    try {
      enqueue();
    } catch (...) {
      cudaStreamEndCapture(stream, &g);
      if (g) cudaGraphDestroy(g);
      cudaGetLastError();
      throw;
    }
    DL_CUDA(cudaStreamEndCapture(stream, &g));
    bool updated = false;
    if (graph_exec && graph_n == n) {
      cudaGraphExecUpdateResultInfo info;
      if (cudaGraphExecUpdate(graph_exec, g, &info) == cudaSuccess) {
        updated = true;
      } else {
        cudaGetLastError();
      }
    }
    if (!updated) {
      if (graph_exec) cudaGraphExecDestroy(graph_exec);
      graph_exec = nullptr;
      const cudaError_t e = cudaGraphInstantiate(&graph_exec, g, 0);
      if (e != cudaSuccess) {
        cudaGetLastError();
        cudaGraphDestroy(g);
        graph_exec = nullptr;
        throw CudaError(std::string("cudaGraphInstantiate: ") + cudaGetErrorString(e));
      }
      graph_n = n;
    }
    if (graph) cudaGraphDestroy(graph);
    graph = g;
    DL_CUDA(cudaGraphLaunch(graph_exec, stream));
    ++graph_replays;
  }

  void set_threads(int tpb) override { kernels.tpb_override = tpb; }
  // Recording the internal force of each launch's last step costs a
  // store per node and selects the extended kernel variant, so it is off
  // until a caller asks for group sums.
  void set_group_output(bool on) override {
    if (on && !fint_last.p) {
      fint_last.alloc(static_cast<size_t>(host->N) * 6 * sizeof(double));
      DL_CUDA(cudaMemsetAsync(fint_last.p, 0, fint_last.bytes, stream));
    }
    m.fint_last = on ? fint_last.as<double>() : nullptr;
  }

  // ---- autotuner -------------------------------------------------------------
  // Times `steps` steps of a fresh copy of this lattice for each launch shape
  // (persistent launch with 32..256 threads per block, two launches per step)
  // and keeps the fastest for this handle.
  void autotune(int64_t steps, int32_t *best_mode, int32_t *best_tpb, double *best_ms) {
    const int cand[5][2] = {{EXEC_PERSISTENT, 256}, {EXEC_PERSISTENT, 128}, {EXEC_PERSISTENT, 64},
                            {EXEC_PERSISTENT, 32}, {EXEC_STREAM, 0}};
    cudaEvent_t a, b;
    DL_CUDA(cudaEventCreate(&a));
    DL_CUDA(cudaEventCreate(&b));
    double best = 1e300;
    int bm = exec_mode, bt = kernels.tpb_override;
    for (auto &cd : cand) {
      auto probe = std::make_unique<Engine<T>>(std::make_unique<HostLattice>(*host), precision);
      probe->stream = stream;
      probe->exec_mode = cd[0];
      probe->kernels.tpb_override = cd[1];
      probe->run(std::min<int64_t>(steps, 10));
      // calls of `steps` steps, as the caller will make them, 50 steps at least
      const int64_t reps = std::max<int64_t>(1, (50 + steps - 1) / steps);
      DL_CUDA(cudaEventRecord(a, stream));
      for (int64_t r = 0; r < reps; ++r) probe->run(steps);
      DL_CUDA(cudaEventRecord(b, stream));
      DL_CUDA(cudaEventSynchronize(b));
      float ms = 0.f;
      DL_CUDA(cudaEventElapsedTime(&ms, a, b));
      if (probe->error_word() & (DL_EW_TIMEOUT | DL_EW_NONFINITE)) continue;
      ms /= static_cast<float>(reps);
      if (ms < best) {
        best = ms;
        bm = cd[0];
        bt = cd[1];
      }
    }
    cudaEventDestroy(a);
    cudaEventDestroy(b);
    exec_mode = bm;
    kernels.tpb_override = bt;
    if (best_mode) *best_mode = bm;
    if (best_tpb) *best_tpb = bt;
    if (best_ms) *best_ms = best;
  }

  // Enqueue nsteps steps on the stream; no host synchronisation.  The load
  // scale table of the call is staged through pinned memory.
  void run(int64_t nsteps) override {
    HostLattice &h = *host;
    if (integ.kind == DL_INTEG_MILNE) {
      run_milne(nsteps);
      return;
    }
    const int64_t kChunk = 1 << 20;
    while (nsteps > 0) {
      int n = static_cast<int>(std::min<int64_t>(nsteps, kChunk));
      if (contact_on || joint_on) {
        if (list_budget <= 0) {
          // the candidate lists are valid while no node moves more than half the
          // margin: their lifetime in steps from the larger of the current maximum
          // node speed and the plate speeds (a plate sets resting nodes in
          // motion), with a factor 4 to spare for nodes that speed up during the
          // chunk (the step kernel flags a violation)
          clist.stream = stream;
          jlist.stream = stream;
          double vmax = plate_speed;
          if (contact_on) {
            vmax = std::max(vmax, clist.max_speed(m.vel));
          } else {
            vmax = std::max(vmax, node_max_speed(m.vel, h.N, jlist.scalars.as<unsigned long long>() + 3, stream));
            ++jlist.launches;
          }
          const double S = vmax > 0.0 ? 0.125 * list_margin() / (vmax * h.dt) : 1e9;
          list_budget = std::max<int64_t>(1, static_cast<int64_t>(std::min(S, 1e9)));
          if (contact_on) {
            clist.build(m.pos, m.conn, 2.0 * clist.radius + clist.margin);
            if (pair_gap.bytes < static_cast<size_t>(std::max(1, clist.n_pairs)) * sizeof(double))
              pair_gap.alloc(static_cast<size_t>(clist.capacity) * sizeof(double));
            m.pairs = clist.pairs.as<int2>();
            m.n_pairs = clist.n_pairs;
            m.xbuild = clist.xbuild.as<double>();
            m.pair_gap = pair_gap.as<double>();
            m.pclosed = clist.closed.as<uint8_t>();
            m.pforce = clist.force.as<double>();
            m.c_quad = reinterpret_cast<const int4 *>(clist.end_node.as<int32_t>());
            m.c_ptr = clist.ends.ptr.as<uint32_t>();
            m.c_ent = clist.ends.val_out.as<int32_t>();
          }
          if (joint_on) {
            jlist.build(m.pos);
            if (jpair_gap.bytes < static_cast<size_t>(std::max(1, jlist.n_pairs)) * sizeof(double))
              jpair_gap.alloc(static_cast<size_t>(jlist.capacity) * sizeof(double));
            m.jpairs = jlist.pairs.as<int2>();
            m.n_jpairs = jlist.n_pairs;
            m.jpair_gap = jpair_gap.as<double>();
            m.jclosed = jlist.closed.as<uint8_t>();
            m.jforce = jlist.force.as<double>();
            m.j_ptr = jlist.ends.ptr.as<uint32_t>();
            m.j_ent = jlist.ends.val_out.as<int32_t>();
            if (!contact_on) m.xbuild = jlist.xbuild.as<double>();
          }
          ++list_builds;
        }
        n = static_cast<int>(std::min<int64_t>(n, list_budget));
        list_budget -= n;
      }
      // step k uses t_k = t_{k-1} + dt and i = k (ExplicitModule::advance
      // advances time before the force evaluation, ExplicitModule.cpp:259-272)
      double tt = t;
      if (m.n_scales > 0) {
        ensure_scale_table(n);
        if (staged_event_pending) DL_CUDA(cudaEventSynchronize(staged_event));
        for (int s = 0; s < n; ++s) {
          tt += h.dt;
          const double vars[3] = {tt, static_cast<double>(step + s + 1), h.dt};
          for (int c = 0; c < m.n_scales; ++c)
            pinned_scales[static_cast<size_t>(s) * m.n_scales + c] = evalExpr(h.scales[c].expr.get(), vars);
        }
        DL_CUDA(cudaMemcpyAsync(scales.p, pinned_scales, static_cast<size_t>(n) * m.n_scales * sizeof(double),
                                cudaMemcpyHostToDevice, stream));
        DL_CUDA(cudaEventRecord(staged_event, stream));
        staged_event_pending = true;
        m.scales = scales.as<double>();
        m.scale_step0 = step + 1;
      } else {
        for (int s = 0; s < n; ++s) tt += h.dt;
      }
      m.t0 = t;
      m.tstep0 = step;
      if (m.plate_force) DL_CUDA(cudaMemsetAsync(m.plate_force, 0, plate_force.bytes, stream));
      if (has_neumann && static_cast<int64_t>(wstep.bytes) < static_cast<int64_t>(n * sizeof(double))) {
        // the previous launches have consumed (and cleared) the old buffer
        DL_CUDA(cudaStreamSynchronize(stream));
        wstep.alloc(static_cast<size_t>(n) * sizeof(double));
        DL_CUDA(cudaMemset(wstep.p, 0, wstep.bytes));
      }
      StepCtx c;
      c.step0 = step;
      c.nsteps = n;
      c.sample_base = n_samples;
      c.wstep = wstep.as<double>();
      c.last_energy = energy_slots.as<double>() + 5 * (launches & 1);
      c.next_energy = energy_slots.as<double>() + 5 * ((launches + 1) & 1);
      SampleSpec smp = sample_spec();
      auto enqueue = [&]() {
        if (m.lat_energy) DL_CUDA(cudaMemsetAsync(m.lat_energy, 0, lat_energy.bytes, stream));
        cudaError_t e = launch_steps<T>(kernels, m, smp, c, exec_mode, barrier.as<GridBarrier>(), stream);
        if (e != cudaSuccess) throw CudaError(std::string("step launch: ") + cudaGetErrorString(e));
        if (has_neumann) {
          e = launch_finish_wext(wstep.as<double>(), n, wext_dev.as<double>(), smp, step, n_samples, c.last_energy,
                                 stream);
          if (e != cudaSuccess) throw CudaError(std::string("finish launch: ") + cudaGetErrorString(e));
        }
      };
      if (exec_mode == EXEC_GRAPH) {
        graph_launch(n, enqueue, c, smp);
      } else {
        enqueue();
      }
      kernel_launches += (exec_mode != EXEC_STREAM) ? 1 : 2 + 2 * static_cast<int64_t>(n);
      if (has_neumann) ++kernel_launches;
      last_slot = static_cast<int>(launches & 1);
      ++launches;
      {
        double ts = t;
        for (int s = 0; s < n; ++s) {
          const int64_t k = step + s + 1;
          ts += h.dt;
          if (every > 0 && k % every == 0 && n_samples < capacity) {
            ++n_samples;
            sample_t.push_back(ts);
          }
        }
      }
      step += n;
      t = tt;
      nsteps -= n;
    }
  }

  // ---- MilneDevice ------------------------------------------------------------
  void set_integrator(const dl_integrator_desc &d) override {
    HostLattice &h = *host;
    if (d.kind != DL_INTEG_LEAPFROG && d.kind != DL_INTEG_MILNE) throw std::invalid_argument("unknown integrator");
    if (d.kind == DL_INTEG_LEAPFROG) {
      integ = d;
      return;
    }
    if (!(d.precision > 0.0)) throw std::invalid_argument("MilneDevice needs precision > 0");
    if (h.n_lat > 1) throw dl::UnsupportedError("MilneDevice runs single lattices, not batches");
    if (contact_on || joint_on || m.n_plates > 0)
      throw dl::UnsupportedError("MilneDevice runs without contact or plates");
    if (m.madd) throw dl::UnsupportedError("MilneDevice runs without added masses");
    if (m.lumped) throw dl::UnsupportedError("MilneDevice runs with the consistent mass");
    if (m.tie_ptr) throw dl::UnsupportedError("MilneDevice runs without rigid ties");
    if (!kernels.milne) throw dl::UnsupportedError("no predictor-corrector kernel in this build");
    if (h.scales.size() > static_cast<size_t>(kMilneMaxScales))
      throw dl::UnsupportedError("MilneDevice takes at most 32 load-scale functions");
    const int N = h.N, E = h.E, G = h.G;
    const int nhA = std::max(1, h.nh);
    if (integ.kind != DL_INTEG_MILNE) {
      mi_pos.alloc(static_cast<size_t>(N) * sizeof(double4));
      mi_rot.alloc(static_cast<size_t>(N) * sizeof(double4));
      mi_vel.alloc(static_cast<size_t>(N) * 6 * sizeof(double));
      if (h.plastic) {
        const size_t NG = static_cast<size_t>(E) * G;
        mi_ep.alloc(NG * 6 * sizeof(T));
        mi_al.alloc(NG * nhA * sizeof(T));
        mi_epsc.alloc(NG * 6 * sizeof(T));
        mi_ediss.alloc(NG * sizeof(double));
      }
      mi_ctl.alloc(sizeof(MilneCtl));
      // load scales as one device program of (t, i, deltaTime)
      if (!h.scales.empty()) {
        std::vector<ExprPtr> ex;
        for (const ScaleFn &f : h.scales) ex.push_back(f.expr);
        const ExprProgram prog = compileExprs(ex);
        if (prog.n_regs > kMaxExprRegs) throw dl::UnsupportedError("load-scale functions need too many registers");
        upload(mi_ops, prog.ops);
        upload(mi_consts, prog.consts);
        upload(mi_outs, prog.outputs);
        md.scale_prog.ops = mi_ops.as<ExprOp>();
        md.scale_prog.consts = mi_consts.as<double>();
        md.scale_prog.n_ops = static_cast<int>(prog.ops.size());
        md.scale_prog.outs = mi_outs.as<uint8_t>();
        md.scale_prog.out0 = prog.outputs.empty() ? 0 : prog.outputs[0];
      }
      md.n_scales = static_cast<int>(h.scales.size());
      cur_dt = h.dt;
      rejected = 0;
    }
    integ = d;
    md.pos_pre = mi_pos.as<double4>();
    md.rot_pre = mi_rot.as<double4>();
    md.vel_pre = mi_vel.as<double>();
    md.ep_new = mi_ep.as<T>();
    md.alpha_new = mi_al.as<T>();
    md.epsc_new = mi_epsc.as<T>();
    md.ediss_new = mi_ediss.as<double>();
    md.ctl = mi_ctl.as<MilneCtl>();
    md.wext = wext_dev.as<double>();
    md.prec = d.precision;
    md.min_dt = d.min_dt > 0.0 ? d.min_dt : h.dt / 100.0;
    md.max_dt = d.max_dt > 0.0 ? d.max_dt : h.dt * 100.0;
    md.safety = d.safety > 0.0 ? d.safety : 0.9;
    md.incr = d.increase > 0.0 ? d.increase : 1.2;
    md.decr = d.decrease > 0.0 ? d.decrease : 0.8;
    md.len_scale = d.length_scale > 0.0 ? d.length_scale : 1e-3;
    const MilneCtl ctl{t, cur_dt, step, rejected};
    DL_CUDA(cudaMemcpyAsync(mi_ctl.p, &ctl, sizeof ctl, cudaMemcpyHostToDevice, stream));
    DL_CUDA(cudaStreamSynchronize(stream));
  }

  void run_milne(int64_t nsteps) {
    const int64_t kChunk = 1 << 20;
    while (nsteps > 0) {
      const int n = static_cast<int>(std::min<int64_t>(nsteps, kChunk));
      int blocks = 0, tpb = 0;
      milne_shape(kernels, std::max(m.E, m.N), &blocks, &tpb);
      if (mi_partial.bytes < static_cast<size_t>(blocks) * 3 * sizeof(double))
        mi_partial.alloc(static_cast<size_t>(blocks) * 3 * sizeof(double));
      md.partial = mi_partial.as<double>();
      StepCtx c;
      c.step0 = step;
      c.nsteps = n;
      c.sample_base = n_samples;
      c.wstep = nullptr;
      c.last_energy = energy_slots.as<double>() + 5 * (launches & 1);
      c.next_energy = energy_slots.as<double>() + 5 * ((launches + 1) & 1);
      const SampleSpec smp = sample_spec();
      const cudaError_t e = launch_milne<T>(kernels, m, smp, c, barrier.as<GridBarrier>(), md, blocks, tpb, stream);
      if (e != cudaSuccess) throw CudaError(std::string("predictor-corrector launch: ") + cudaGetErrorString(e));
      ++kernel_launches;
      last_slot = static_cast<int>(launches & 1);
      ++launches;
      const int64_t s0 = n_samples;
      for (int s = 0; s < n; ++s) {
        const int64_t k = step + s + 1;
        if (every > 0 && k % every == 0 && n_samples < capacity) ++n_samples;
      }
      MilneCtl ctl{};
      DL_CUDA(cudaMemcpyAsync(&ctl, mi_ctl.p, sizeof ctl, cudaMemcpyDeviceToHost, stream));
      DL_CUDA(cudaStreamSynchronize(stream));
      step = ctl.step;
      t = ctl.t;
      cur_dt = ctl.dt;
      rejected = ctl.rejected;
      if (n_samples > s0) {
        std::vector<double> ts(static_cast<size_t>(n_samples - s0));
        DL_CUDA(cudaMemcpy(ts.data(), s_times.as<double>() + s0, ts.size() * sizeof(double), cudaMemcpyDeviceToHost));
        sample_t.insert(sample_t.end(), ts.begin(), ts.end());
      }
      nsteps -= n;
    }
  }

  bool adaptive() const override { return integ.kind == DL_INTEG_MILNE; }

  void get_time(double *tt, double *dt, int64_t *st, int64_t *rj) override {
    DL_CUDA(cudaStreamSynchronize(stream));
    const bool milne = integ.kind == DL_INTEG_MILNE;
    if (tt) *tt = t;
    if (dt) *dt = milne ? cur_dt : host->dt;
    if (st) *st = step;
    if (rj) *rj = milne ? rejected : 0;
  }

  void info(int32_t *jit, int32_t *blocks, const char **log) override {
    if (jit) *jit = kernels.jit ? 1 : 0;
    if (blocks) *blocks = kernels.persist_blocks;
    if (log) *log = jit_log.c_str();
  }

  void batch_energies(int lat, dl_energies *e) override {
    HostLattice &h = *host;
    if (lat < 0 || lat >= h.n_lat) throw std::invalid_argument("lattice index out of range");
    double le[5] = {0, 0, 0, 0, 0};
    DL_CUDA(cudaStreamSynchronize(stream));
    if (h.n_lat > 1) {
      DL_CUDA(cudaMemcpy(le, lat_energy.as<double>() + 5 * lat, sizeof le, cudaMemcpyDeviceToHost));
    } else {
      DL_CUDA(cudaMemcpy(le, energy_slots.as<double>() + 5 * last_slot, sizeof le, cudaMemcpyDeviceToHost));
    }
    e->kinetic = le[0];
    e->potential = le[1];
    e->dissipated = le[2];
    e->external_work = h.n_lat > 1 ? 0.0 : le[3];
    e->contact = 0.0;
  }

  void contact_pairs(int64_t *n, int32_t *pairs_out, double *gaps, int64_t max) override {
    HostLattice &h = *host;
    DL_CUDA(cudaStreamSynchronize(stream));
    std::vector<std::pair<std::pair<int, int>, double>> closed;
    if (contact_on && m.n_pairs > 0 && launches > 0) {
      std::vector<int2> pr(m.n_pairs);
      std::vector<double> gp(m.n_pairs);
      DL_CUDA(cudaMemcpy(pr.data(), m.pairs, pr.size() * sizeof(int2), cudaMemcpyDeviceToHost));
      DL_CUDA(cudaMemcpy(gp.data(), m.pair_gap, gp.size() * sizeof(double), cudaMemcpyDeviceToHost));
      for (int i = 0; i < m.n_pairs; ++i)
        if (gp[i] < 1e299) {
          const int a = h.elem_old[pr[i].x], b = h.elem_old[pr[i].y];
          closed.push_back({{std::min(a, b), std::max(a, b)}, gp[i]});
        }
      std::sort(closed.begin(), closed.end());
    }
    if (n) *n = static_cast<int64_t>(closed.size());
    for (int64_t i = 0; i < std::min<int64_t>(max, static_cast<int64_t>(closed.size())); ++i) {
      if (pairs_out) {
        pairs_out[2 * i] = closed[i].first.first;
        pairs_out[2 * i + 1] = closed[i].first.second;
      }
      if (gaps) gaps[i] = closed[i].second;
    }
  }

  void joint_contact_pairs(int64_t *n, int32_t *pairs_out, double *gaps, int64_t max) override {
    HostLattice &h = *host;
    DL_CUDA(cudaStreamSynchronize(stream));
    std::vector<std::pair<std::pair<int, int>, double>> closed;
    if (joint_on && m.n_jpairs > 0 && launches > 0) {
      std::vector<int2> pr(m.n_jpairs);
      std::vector<double> gp(m.n_jpairs);
      DL_CUDA(cudaMemcpy(pr.data(), m.jpairs, pr.size() * sizeof(int2), cudaMemcpyDeviceToHost));
      DL_CUDA(cudaMemcpy(gp.data(), m.jpair_gap, gp.size() * sizeof(double), cudaMemcpyDeviceToHost));
      for (int i = 0; i < m.n_jpairs; ++i)
        if (gp[i] < 1e299) {
          const int a = h.node_old[pr[i].x], b = h.node_old[pr[i].y];
          closed.push_back({{std::min(a, b), std::max(a, b)}, gp[i]});
        }
      std::sort(closed.begin(), closed.end());
    }
    if (n) *n = static_cast<int64_t>(closed.size());
    for (int64_t i = 0; i < std::min<int64_t>(max, static_cast<int64_t>(closed.size())); ++i) {
      if (pairs_out) {
        pairs_out[2 * i] = closed[i].first.first;
        pairs_out[2 * i + 1] = closed[i].first.second;
      }
      if (gaps) gaps[i] = closed[i].second;
    }
  }

  // Element table at the current state ([E][6], caller's element numbering):
  // "strain", "stress" (spatial), "mat_strain", "mat_stress" (material frame),
  // "plast_strain" (zeros for elastic models, whose material writes no rows).
  void element_table(const std::string &name, double *out) override {
    HostLattice &h = *host;
    int kind = 0;
    bool spatial = false;
    if (name == "strain") {
      spatial = true;
    } else if (name == "mat_strain") {
    } else if (name == "stress") {
      kind = 1;
      spatial = true;
    } else if (name == "mat_stress") {
      kind = 1;
    } else if (name == "plast_strain") {
      kind = 2;
    } else {
      throw std::invalid_argument("element table \"" + name +
                                  "\": supported are strain, stress, mat_strain, mat_stress, plast_strain");
    }
    DevBuf buf;
    buf.alloc(static_cast<size_t>(h.E) * 6 * sizeof(double));
    DL_CUDA(launch_elem_table<T>(m, kind, spatial, buf.as<double>(), stream));
    std::vector<double> tmp(static_cast<size_t>(h.E) * 6);
    DL_CUDA(cudaMemcpyAsync(tmp.data(), buf.p, buf.bytes, cudaMemcpyDeviceToHost, stream));
    DL_CUDA(cudaStreamSynchronize(stream));
    ++kernel_launches;
    for (int ei = 0; ei < h.E; ++ei)
      for (int k = 0; k < 6; ++k) out[static_cast<size_t>(h.elem_old[ei]) * 6 + k] = tmp[static_cast<size_t>(ei) * 6 + k];
  }

  // margin of the candidate lists (rod and joint contact are rebuilt together)
  double list_margin() const {
    if (contact_on && joint_on) return std::min(clist.margin, jlist.margin);
    return contact_on ? clist.margin : jlist.margin;
  }

  int64_t launch_count() override {
    return kernel_launches + clist.launches + clist.ends.launches + jlist.launches + jlist.ends.launches +
           adj_launches;
  }
  void set_tape_budget(int64_t bytes) override { tape_budget = bytes; }

  // ---- adjoint of the radius ----------------------------------------------
  // Forward run with checkpoints (state every K steps) and the per-step group
  // force, then the reverse sweep segment by segment: restore a checkpoint,
  // recompute its K steps with the state tape on, and step the adjoint back
  // through them (k_adj_node, k_adj_elem per step).  The handle ends in the
  // forward run's final state.
  void adjoint_radius(int64_t nsteps, int K, int n_params, const int32_t *elem_param, int n_react,
                      const int32_t *react_nodes, int react_dof, double react_w, double *J, double *grad) override {
    HostLattice &h = *host;
    if (h.n_lat > 1) throw std::invalid_argument("the adjoint works on single lattices, not batches");
    if (contact_on || joint_on || m.n_plates > 0)
      throw std::invalid_argument("the adjoint does not cover contact or plates");
    if (m.madd) throw std::invalid_argument("the adjoint does not cover added masses");
    if (m.lumped) throw dl::UnsupportedError("the adjoint differentiates the consistent mass only");
    if (m.tie_ptr) throw dl::UnsupportedError("the adjoint does not cover rigid ties");
    if (m.nen > 2) throw dl::UnsupportedError("the adjoint differentiates two-node elements");
    if (!m.so3) throw std::invalid_argument("the adjoint needs the SO(3) rotation update");
    if (integ.kind != DL_INTEG_LEAPFROG) throw dl::UnsupportedError("the adjoint differentiates LeapFrog runs");
    if (nsteps <= 0 || K < 0) throw std::invalid_argument("nsteps must be positive, checkpoint_every >= 0");
    const bool reverse = K > 0;  // checkpoint_every = 0: the objective only
    if (!reverse) K = static_cast<int>(std::min<int64_t>(nsteps, 1 << 30));
    if (react_dof < 0 || react_dof > 5) throw std::invalid_argument("react_dof must be 0..5");
    for (int e = 0; e < h.E; ++e)
      if (!h.ecircle[e]) throw std::invalid_argument("radius derivatives need circular sections");
    if (!elem_param && n_params != h.E) throw std::invalid_argument("without elem_param, n_params must be n_elems");
    AdjKernels ak;
    if (!reverse) {
    } else if (h.plastic) {
      const std::string src = emitYieldAdjPolicy(h.yield_expr, h.grad_exprs, sizeof(T) == 4, "__device__");
      std::string log;
      const AdjKernels *p = jit_adjoint_kernels(src, sizeof(T) == 4, &log);
      if (!p) throw std::runtime_error("adjoint kernels could not be compiled: " + log);
      ak = *p;
    } else {
      ak = aot_adj_kernels<T>();
    }
    const int N = h.N, E = h.E, G = h.G;
    const int nhA = std::max(1, h.nh);
    const size_t NG = static_cast<size_t>(E) * G;
    const size_t b_pos = static_cast<size_t>(N) * sizeof(double4), b_vel = static_cast<size_t>(N) * 6 * sizeof(double);
    const size_t b_ep = h.plastic ? NG * 6 * sizeof(T) : 0, b_al = h.plastic ? NG * nhA * sizeof(T) : 0;
    const size_t b_ediss = h.plastic ? NG * sizeof(double) : 0;
    // full tape when it fits the memory budget: every step's state is kept
    // during the forward run and nothing is recomputed; otherwise checkpoints
    // every K steps and one recomputation per segment
    const size_t slot_bytes = 2 * b_pos + b_vel + 2 * b_ep + b_al;
    size_t free_b = 0, total_b = 0;
    DL_CUDA(cudaMemGetInfo(&free_b, &total_b));
    const size_t budget = tape_budget < 0 ? free_b / 2 : static_cast<size_t>(tape_budget);
    const bool full = reverse && static_cast<size_t>(nsteps + 1) * slot_bytes <= budget;
    if (full) K = static_cast<int>(std::min<int64_t>(nsteps, 1 << 30));
    const int64_t C = (nsteps + K - 1) / K;
    auto ensure = [](DevBuf &b, size_t n) {
      if (b.bytes < n) b.alloc(n);
    };
    auto ensure_pool = [&](PoolBuf &b, size_t n) {
      if (b.bytes < n) b.alloc(n, stream);
    };
    // checkpoints 0..C-1 (segment starts) and C (final state)
    ensure_pool(ck_pos, (C + 1) * b_pos);
    ensure_pool(ck_rot, (C + 1) * b_pos);
    ensure_pool(ck_vel, (C + 1) * b_vel);
    if (h.plastic) {
      ensure_pool(ck_ep, (C + 1) * b_ep);
      ensure_pool(ck_al, (C + 1) * b_al);
      ensure_pool(ck_epsc, (C + 1) * b_ep);
      ensure_pool(ck_ediss, (C + 1) * b_ediss);
    }
    auto d2d = [&](void *dst, const void *src, size_t n) {
      if (n) DL_CUDA(cudaMemcpyAsync(dst, src, n, cudaMemcpyDeviceToDevice, stream));
    };
    auto at = [](PoolBuf &b, size_t off) { return static_cast<char *>(b.p) + off; };
    auto save = [&](int64_t c) {
      d2d(at(ck_pos, c * b_pos), pos.p, b_pos);
      d2d(at(ck_rot, c * b_pos), rot.p, b_pos);
      d2d(at(ck_vel, c * b_vel), vel.p, b_vel);
      if (h.plastic) {
        d2d(at(ck_ep, c * b_ep), ep.p, b_ep);
        d2d(at(ck_al, c * b_al), alpha.p, b_al);
        d2d(at(ck_epsc, c * b_ep), epsc.p, b_ep);
        d2d(at(ck_ediss, c * b_ediss), ediss.p, b_ediss);
      }
    };
    auto restore = [&](int64_t c) {
      d2d(pos.p, at(ck_pos, c * b_pos), b_pos);
      d2d(rot.p, at(ck_rot, c * b_pos), b_pos);
      d2d(vel.p, at(ck_vel, c * b_vel), b_vel);
      if (h.plastic) {
        d2d(ep.p, at(ck_ep, c * b_ep), b_ep);
        d2d(alpha.p, at(ck_al, c * b_al), b_al);
        d2d(epsc.p, at(ck_epsc, c * b_ep), b_ep);
        d2d(ediss.p, at(ck_ediss, c * b_ediss), b_ediss);
      }
    };
    // objective group
    const bool peak = n_react > 0 && react_w != 0.0;
    if (peak) {
      std::vector<uint8_t> flag(N, 0);
      for (int i = 0; i < n_react; ++i) {
        if (react_nodes[i] < 0 || react_nodes[i] >= N) throw std::invalid_argument("react node out of range");
        flag[h.node_new[react_nodes[i]]] = 1;
      }
      upload(grp_flag_dev, flag);
      ensure(grp_hist_dev, static_cast<size_t>(nsteps + 1) * sizeof(double));
      DL_CUDA(cudaMemsetAsync(grp_hist_dev.p, 0, static_cast<size_t>(nsteps + 1) * sizeof(double), stream));
    }
    // plain forward run (sampling off), checkpoints at segment starts
    const int every_saved = every;
    every = 0;
    double wext_saved = 0.0;
    DL_CUDA(cudaMemcpyAsync(&wext_saved, wext_dev.p, sizeof(double), cudaMemcpyDeviceToHost, stream));
    DL_CUDA(cudaStreamSynchronize(stream));
    const int64_t base = step;
    std::vector<double> t_ck(C + 1);
    if (peak) {
      m.grp_flag = grp_flag_dev.as<uint8_t>();
      m.grp_hist = grp_hist_dev.as<double>();
      m.grp_dof = react_dof;
      m.grp_step0 = base;
    }
    // branch tape: record or impose the cutting-plane iteration counts of
    // this forward run (elastoplastic lattices only)
    const bool branches = br_mode != 0 && h.plastic;
    if (branches && br_mode == 2 && reverse)
      throw std::invalid_argument("imposed branches evaluate the objective only (checkpoint_every = 0)");
    const size_t br_bytes = static_cast<size_t>(nsteps) * NG;
    if (branches) {
      if (br_mode == 2) {
        if (br_host.size() != br_bytes) throw std::invalid_argument("branch tape size does not match the run");
        upload(br_dev, br_host);
      } else {
        ensure(br_dev, br_bytes);
      }
      m.br = br_dev.as<uint8_t>();
      m.br_mode = br_mode;
      m.br_step0 = base;
    }
    auto tape_into = [&](DevModel<T> &mm, StateTape &tb, int64_t step0) {
      mm.tp_pos = tb.pos.as<double4>();
      mm.tp_rot = tb.rot.as<double4>();
      mm.tp_vel = tb.vel.as<double>();
      mm.tp_ep = h.plastic ? tb.ep.as<T>() : nullptr;
      mm.tp_al = h.plastic ? tb.al.as<T>() : nullptr;
      mm.tp_epsc = h.plastic ? tb.epsc.as<T>() : nullptr;
      mm.tp_step0 = step0;
    };
    auto tape_on = [&](StateTape &tb, int64_t step0) { tape_into(m, tb, step0); };
    auto tape_off = [&]() {
      m.tp_pos = nullptr;
      m.tp_rot = nullptr;
      m.tp_vel = nullptr;
      m.tp_ep = m.tp_al = m.tp_epsc = nullptr;
    };
    auto tape_slot0 = [&](StateTape &tb) {  // current state into slot 0
      d2d(tb.pos.p, pos.p, b_pos);
      d2d(tb.rot.p, rot.p, b_pos);
      d2d(tb.vel.p, vel.p, b_vel);
      if (h.plastic) {
        d2d(tb.ep.p, ep.p, b_ep);
        d2d(tb.al.p, alpha.p, b_al);
        d2d(tb.epsc.p, epsc.p, b_ep);
      }
    };
    // tape of one segment (K + 1 slots; the whole run when full); a second
    // set when segments are recomputed
    const int n_sets = reverse ? (full || C == 1 ? 1 : 2) : 0;
    for (int b = 0; b < n_sets; ++b) {
      ensure_pool(tape[b].pos, static_cast<size_t>(K + 1) * b_pos);
      ensure_pool(tape[b].rot, static_cast<size_t>(K + 1) * b_pos);
      ensure_pool(tape[b].vel, static_cast<size_t>(K + 1) * b_vel);
      if (h.plastic) {
        ensure_pool(tape[b].ep, static_cast<size_t>(K + 1) * b_ep);
        ensure_pool(tape[b].al, static_cast<size_t>(K + 1) * b_al);
        ensure_pool(tape[b].epsc, static_cast<size_t>(K + 1) * b_ep);
      }
    }
    for (int64_t c = 0; c < C; ++c) {
      save(c);
      t_ck[c] = t;
      if (full) {
        tape_slot0(tape[0]);
        tape_on(tape[0], step);
      }
      run(std::min<int64_t>(K, nsteps - c * K));
      tape_off();
    }
    save(C);
    t_ck[C] = t;
    m.grp_flag = nullptr;
    m.grp_hist = nullptr;
    m.br = nullptr;
    m.br_mode = 0;
    fetch_last_energies();
    const dl_energies last_fwd = last;
    double Jv = last.dissipated;
    int64_t peak_step = -1;
    double peak_sign = 1.0;
    if (peak) {
      // the peak magnitude of the group force, max_k |R(k)|, reached at
      // step kbest (or the recorded step when the branches are imposed)
      std::vector<double> hist(nsteps + 1);
      DL_CUDA(cudaMemcpy(hist.data(), grp_hist_dev.p, hist.size() * sizeof(double), cudaMemcpyDeviceToHost));
      int64_t kbest = 1;
      for (int64_t k = 2; k <= nsteps; ++k)
        if (std::fabs(hist[k]) > std::fabs(hist[kbest])) kbest = k;
      peak_sign = hist[kbest] < 0.0 ? -1.0 : 1.0;
      if (branches && br_mode == 2) {
        if (br_peak_step < 1 || br_peak_step > nsteps) throw std::invalid_argument("imposed peak step out of range");
        kbest = br_peak_step;
        peak_sign = br_peak_sign;
      }
      peak_step = base + kbest;
      Jv += react_w * peak_sign * hist[kbest];
      if (branches && br_mode == 1) {
        br_peak_step = kbest;
        br_peak_sign = peak_sign;
      }
    }
    if (branches && br_mode == 1) {
      br_host.resize(br_bytes);
      DL_CUDA(cudaMemcpy(br_host.data(), br_dev.p, br_bytes, cudaMemcpyDeviceToHost));
    }
    if (!reverse) {
      every = every_saved;
      for (int k = 0; k < n_params; ++k) grad[k] = 0.0;
      if (J) *J = Jv;
      return;
    }
    // adjoint state
    auto zero = [&](DevBuf &b, size_t n) {
      if (b.bytes < n) b.alloc(n);
      DL_CUDA(cudaMemsetAsync(b.p, 0, n, stream));
    };
    zero(a_lx, 3 * N * sizeof(double));
    zero(a_lth, 3 * N * sizeof(double));
    zero(a_lv, 6 * N * sizeof(double));
    zero(a_lf, 6 * N * sizeof(double));
    zero(a_aslot, 12 * static_cast<size_t>(E) * sizeof(double));
    zero(a_lC, 6 * static_cast<size_t>(E) * sizeof(double));
    zero(a_lec, 2 * static_cast<size_t>(E) * sizeof(double));
    zero(a_lmass, N * sizeof(double));
    zero(a_lS, 6 * N * sizeof(double));
    if (h.plastic) {
      zero(a_lep, NG * 6 * sizeof(double));
      zero(a_lal, NG * nhA * sizeof(double));
      zero(a_lepsc, NG * 6 * sizeof(double));
    }
    AdjCtx<T> a;
    a.lx = a_lx.as<double>();
    a.lth = a_lth.as<double>();
    a.lv = a_lv.as<double>();
    a.lf = a_lf.as<double>();
    a.aslot = a_aslot.as<double>();
    a.lep = a_lep.as<double>();
    a.lal = a_lal.as<double>();
    a.lepsc = a_lepsc.as<double>();
    a.lC = a_lC.as<double>();
    a.lec = a_lec.as<double>();
    a.lmass = a_lmass.as<double>();
    a.lS = a_lS.as<double>();
    a.w_diss = 1.0;
    a.w_peak = peak ? react_w * peak_sign : 0.0;
    a.peak_step = peak_step;
    a.peak_dof = react_dof;
    a.peak_flag = peak ? grp_flag_dev.as<uint8_t>() : nullptr;
    const int EP = E * adj_lanes(G);  // element adjoint: one thread per (element, Gauss point)
    const int tn = threads_for(N), te = threads_for(EP);
    const int nb = std::max(1, (N + tn - 1) / tn);
    const int eb = std::max(1, (EP + te - 1) / te);
    if (!rstream) {
      int lo = 0, hi = 0;
      DL_CUDA(cudaDeviceGetStreamPriorityRange(&lo, &hi));
      DL_CUDA(cudaStreamCreateWithPriority(&rstream, cudaStreamNonBlocking, hi));
      for (cudaEvent_t *ev : {&ev_ready[0], &ev_ready[1], &ev_free[0], &ev_free[1], &ev_join})
        DL_CUDA(cudaEventCreateWithFlags(ev, cudaEventDisableTiming));
    }
    // Segment c is recomputed on `stream` into tape set c % 2 while the
    // reverse sweep over segment c + 1 runs on `rstream` from the other set.
    // The reverse kernels read only the tape, the constant model arrays and
    // the adjoint buffers, none of which the recomputation writes.
    auto recompute = [&](int64_t c) {
      StateTape &tb = tape[c % 2];
      if (c + 2 < C) DL_CUDA(cudaStreamWaitEvent(stream, ev_free[c % 2], 0));  // reverse of c + 2 done with it
      restore(c);
      tape_slot0(tb);
      step = base + c * K;
      t = t_ck[c];
      tape_on(tb, step);
      run(std::min<int64_t>(K, nsteps - c * K));
      tape_off();
      DL_CUDA(cudaEventRecord(ev_ready[c % 2], stream));
    };
    if (full) {
      DL_CUDA(cudaEventRecord(ev_ready[0], stream));
    } else {
      recompute(C - 1);
    }
    for (int64_t c = C - 1; c >= 0; --c) {
      const int64_t len = std::min<int64_t>(K, nsteps - c * K);
      StateTape &tb = tape[full ? 0 : c % 2];
      // ev_ready of the last launch also orders the zeroed adjoint buffers
      DL_CUDA(cudaStreamWaitEvent(rstream, ev_ready[full ? 0 : c % 2], 0));
      DevModel<T> mt = m;  // the adjoint kernels read the tape through a copy of the model
      tape_into(mt, tb, base + c * K);
      for (int64_t k = base + c * K + len; k > base + c * K; --k) {
        int64_t kk = k;
        void *args[] = {&mt, &a, &kk};
        DL_CUDA(cudaLaunchKernel(ak.node, dim3(nb), dim3(tn), args, 0, rstream));
        DL_CUDA(cudaLaunchKernel(ak.elem, dim3(eb), dim3(te), args, 0, rstream));
        adj_launches += 2;
      }
      if (!full) {
        DL_CUDA(cudaEventRecord(ev_free[c % 2], rstream));
        if (c > 0) recompute(c - 1);
      }
    }
    DL_CUDA(cudaEventRecord(ev_join, rstream));
    DL_CUDA(cudaStreamWaitEvent(stream, ev_join, 0));
    // back to the final state of the forward run
    if (!full) restore(C);
    step = base + nsteps;
    t = t_ck[C];
    every = every_saved;
    DL_CUDA(cudaMemcpyAsync(wext_dev.p, &wext_saved, sizeof(double), cudaMemcpyHostToDevice, stream));
    {  // the energies of the final step, as after the forward run
      const double le[5] = {last_fwd.kinetic, last_fwd.potential, last_fwd.dissipated, last_fwd.external_work,
                            last_fwd.contact};
      DL_CUDA(cudaMemcpyAsync(energy_slots.as<double>() + 5 * last_slot, le, sizeof le, cudaMemcpyHostToDevice,
                              stream));
      DL_CUDA(cudaStreamSynchronize(stream));
      last = last_fwd;
    }
    // radius derivatives (host, FP64) from the accumulated adjoints
    std::vector<double> lC(6 * static_cast<size_t>(E)), lec(2 * static_cast<size_t>(E)), lm(N), lS(6 * static_cast<size_t>(N));
    DL_CUDA(cudaMemcpyAsync(lC.data(), a_lC.p, lC.size() * sizeof(double), cudaMemcpyDeviceToHost, stream));
    DL_CUDA(cudaMemcpyAsync(lec.data(), a_lec.p, lec.size() * sizeof(double), cudaMemcpyDeviceToHost, stream));
    DL_CUDA(cudaMemcpyAsync(lm.data(), a_lmass.p, lm.size() * sizeof(double), cudaMemcpyDeviceToHost, stream));
    DL_CUDA(cudaMemcpyAsync(lS.data(), a_lS.p, lS.size() * sizeof(double), cudaMemcpyDeviceToHost, stream));
    uint32_t ew = 0;
    DL_CUDA(cudaMemcpyAsync(&ew, err.p, sizeof ew, cudaMemcpyDeviceToHost, stream));
    DL_CUDA(cudaStreamSynchronize(stream));
    if (ew & (DL_EW_TIMEOUT | DL_EW_NONFINITE | DL_EW_RETURN_MAP))
      throw std::runtime_error("the forward run reported an error (see dl_get_error_word)");
    for (int k = 0; k < n_params; ++k) grad[k] = 0.0;
    for (int ei = 0; ei < E; ++ei) {
      const double r = h.ec[ei];
      const double L0 = 1.0 / h.invL0[ei];
      const double rho = h.erho[ei], ic = h.eic[ei];
      double g = 0.0;
      // section stiffness: G k A, G k A, E A (~ r^2), E I, E I, G J (~ r^4)
      const double pw[6] = {2, 2, 2, 4, 4, 4};
      for (int q = 0; q < 6; ++q) g += lC[static_cast<size_t>(q) * E + ei] * pw[q] * h.C[static_cast<size_t>(q) * E + ei] / r;
      // yield-expression variables radius and area = pi r^2
      g += lec[ei] + lec[E + ei] * 2.0 * M_PI * r;
      // lumped mass of both ends: translational rho A L0/2; rotational
      // 1/2 Lambda_N diag(rho I ic L0 + rho A L0^3/12, same, rho J ic L0) Lambda_N^T
      const double dA = 2.0 * M_PI * r, dI = M_PI * r * r * r, dJ = 2.0 * dI;
      const double dD[3] = {rho * dI * ic * L0 + rho * dA * L0 * L0 * L0 / 12.0,
                            rho * dI * ic * L0 + rho * dA * L0 * L0 * L0 / 12.0, rho * dJ * ic * L0};
      for (int s2 = 0; s2 < 2; ++s2) {
        const int nd = h.conn[2 * ei + s2];
        g += lm[nd] * rho * dA * L0 / 2.0;
        const double *qq = &h.qN[(static_cast<size_t>(s2) * E + ei) * 4];
        double Rm[3][3];
        qmat(Q4<double>{qq[0], qq[1], qq[2], qq[3]}, Rm);
        double dS[3][3];
        for (int i = 0; i < 3; ++i)
          for (int j = 0; j < 3; ++j) {
            double acc = 0.0;
            for (int k = 0; k < 3; ++k) acc += Rm[i][k] * dD[k] * Rm[j][k];
            dS[i][j] = 0.5 * acc;
          }
        const double *l = &lS[0];
        const double lxx = l[0 * N + nd], lyy = l[1 * N + nd], lzz = l[2 * N + nd];
        const double lxy = l[3 * N + nd], lxz = l[4 * N + nd], lyz = l[5 * N + nd];
        g += lxx * dS[0][0] + lyy * dS[1][1] + lzz * dS[2][2] + 2.0 * (lxy * dS[0][1] + lxz * dS[0][2] + lyz * dS[1][2]);
      }
      const int eo = h.elem_old[ei];
      const int k = elem_param ? elem_param[eo] : eo;
      if (k < 0 || k >= n_params) throw std::invalid_argument("elem_param out of range");
      grad[k] += g;
    }
    if (J) *J = Jv;
  }

  void contact_stats(int64_t *cand, int64_t *builds) override {
    if (cand) *cand = contact_on ? m.n_pairs : 0;
    if (builds) *builds = list_builds;
  }

  void plate_reaction(double *out) override {
    DL_CUDA(cudaStreamSynchronize(stream));
    for (int k = 0; k < 6; ++k) out[k] = 0.0;
    if (m.plate_force) DL_CUDA(cudaMemcpy(out, m.plate_force, 6 * sizeof(double), cudaMemcpyDeviceToHost));
  }

  void fetch_last_energies() {
    // a pinned staging slot and an async copy on the handle's stream: a
    // pageable 40-byte copy costs several microseconds per call
    if (!pinned_energy)
      DL_CUDA(cudaMallocHost(reinterpret_cast<void **>(&pinned_energy), 5 * sizeof(double)));
    DL_CUDA(cudaMemcpyAsync(pinned_energy, energy_slots.as<double>() + 5 * last_slot, 5 * sizeof(double),
                            cudaMemcpyDeviceToHost, stream));
    DL_CUDA(cudaStreamSynchronize(stream));
    const double *le = pinned_energy;
    last.kinetic = le[0];
    last.potential = le[1];
    last.dissipated = le[2];
    last.external_work = le[3];
    last.contact = le[4];
  }

  void get_samples(int64_t *n, int64_t *steps, double *rows, dl_energies *en, int64_t max) override {
    HostLattice &h = *host;
    if (n) *n = n_samples;
    const int64_t k = std::min(n_samples, max);
    if (k <= 0) return;
    const size_t nw = watch.size();
    std::vector<double> raw(static_cast<size_t>(k) * std::max<size_t>(nw, 1) * 13);
    std::vector<double> e5(static_cast<size_t>(k) * 5);
    std::vector<int64_t> st(k);
    DL_CUDA(cudaStreamSynchronize(stream));
    DL_CUDA(cudaMemcpy(e5.data(), s_energy.p, e5.size() * sizeof(double), cudaMemcpyDeviceToHost));
    DL_CUDA(cudaMemcpy(st.data(), s_steps.p, k * sizeof(int64_t), cudaMemcpyDeviceToHost));
    if (nw) DL_CUDA(cudaMemcpy(raw.data(), s_rows.p, static_cast<size_t>(k) * nw * 13 * sizeof(double), cudaMemcpyDeviceToHost));
    for (int64_t s = 0; s < k; ++s) {
      if (steps) steps[s] = st[s];
      if (en) {
        en[s].kinetic = e5[s * 5];
        en[s].potential = e5[s * 5 + 1];
        en[s].dissipated = e5[s * 5 + 2];
        en[s].external_work = e5[s * 5 + 3];
        en[s].contact = e5[s * 5 + 4];
      }
      if (rows)
        for (size_t w = 0; w < nw; ++w) {
          const double *r = &raw[(s * nw + w) * 13];
          double *o = rows + (s * nw + w) * 12;
          const int n0 = watch[w];
          for (int q = 0; q < 3; ++q) o[q] = r[q] - h.X0[n0 * 3 + q];
          V3<double> th = qlog(Q4<double>{r[3], r[4], r[5], r[6]});
          o[3] = th.x;
          o[4] = th.y;
          o[5] = th.z;
          for (int q = 0; q < 6; ++q) o[6 + q] = r[7 + q];
        }
    }
  }

  // Caller arrays in the original numbering; copies run on the handle's stream
  // (true DMA when the caller's buffers are pinned).
  void get_state(double *u, double *th, double *v) override {
    HostLattice &h = *host;
    const size_t N = h.N;
    double *d = xfer.as<double>();
    cudaError_t e = launch_state_out(m.pos, m.rot, m.vel, X0dev.as<double>(), node_old_dev.as<int32_t>(), h.N,
                                     u ? d : nullptr, th ? d + 3 * N : nullptr, v ? d + 6 * N : nullptr, stream);
    if (e != cudaSuccess) throw CudaError(cudaGetErrorString(e));
    if (u) DL_CUDA(cudaMemcpyAsync(u, d, 3 * N * sizeof(double), cudaMemcpyDeviceToHost, stream));
    if (th) DL_CUDA(cudaMemcpyAsync(th, d + 3 * N, 3 * N * sizeof(double), cudaMemcpyDeviceToHost, stream));
    if (v) DL_CUDA(cudaMemcpyAsync(v, d + 6 * N, 6 * N * sizeof(double), cudaMemcpyDeviceToHost, stream));
    DL_CUDA(cudaStreamSynchronize(stream));
  }

  void set_state(const double *u, const double *th, const double *v) override {
    HostLattice &h = *host;
    const size_t N = h.N;
    double *d = xfer.as<double>();
    if (u) DL_CUDA(cudaMemcpyAsync(d, u, 3 * N * sizeof(double), cudaMemcpyHostToDevice, stream));
    if (th) DL_CUDA(cudaMemcpyAsync(d + 3 * N, th, 3 * N * sizeof(double), cudaMemcpyHostToDevice, stream));
    if (v) DL_CUDA(cudaMemcpyAsync(d + 6 * N, v, 6 * N * sizeof(double), cudaMemcpyHostToDevice, stream));
    cudaError_t e = launch_state_in(m.pos, m.rot, m.vel, X0dev.as<double>(), node_old_dev.as<int32_t>(), h.N,
                                    u ? d : nullptr, th ? d + 3 * N : nullptr, v ? d + 6 * N : nullptr, stream);
    if (e != cudaSuccess) throw CudaError(cudaGetErrorString(e));
    // the caller may reuse its buffers on return
    DL_CUDA(cudaStreamSynchronize(stream));
    list_budget = 0;  // positions or velocities changed: rebuild the contact list
  }

  void internal_force(const double *u, const double *th, double *fint) override {
    HostLattice &h = *host;
    const int N = h.N;
    // evaluate at the given configuration, then restore the state
    DL_CUDA(cudaStreamSynchronize(stream));
    DevBuf sp, sr, fd;
    sp.alloc(pos.bytes);
    sr.alloc(rot.bytes);
    DL_CUDA(cudaMemcpy(sp.p, pos.p, pos.bytes, cudaMemcpyDeviceToDevice));
    DL_CUDA(cudaMemcpy(sr.p, rot.p, rot.bytes, cudaMemcpyDeviceToDevice));
    set_state(u, th, nullptr);
    fd.alloc(static_cast<size_t>(N) * 6 * sizeof(double));
    cudaError_t e = launch_internal_force<T>(kernels, m, fd.as<double>(), stream);
    if (e != cudaSuccess) throw CudaError(cudaGetErrorString(e));
    std::vector<double> f(static_cast<size_t>(N) * 6);
    DL_CUDA(cudaStreamSynchronize(stream));
    DL_CUDA(cudaMemcpy(f.data(), fd.p, f.size() * sizeof(double), cudaMemcpyDeviceToHost));
    DL_CUDA(cudaMemcpy(pos.p, sp.p, pos.bytes, cudaMemcpyDeviceToDevice));
    DL_CUDA(cudaMemcpy(rot.p, sr.p, rot.bytes, cudaMemcpyDeviceToDevice));
    for (int n = 0; n < N; ++n)
      for (int k = 0; k < 6; ++k) fint[n * 6 + k] = f[static_cast<size_t>(h.node_new[n]) * 6 + k];
  }

  int internal_force_static(const double *u, const double *th, double *fint, const char **why) override {
    return dl::internal_force_static<T>(kernels, m, device, X0dev.as<double>(), node_old_dev.as<int32_t>(), u, th,
                                        fint, stream, why);
  }

  void get_history(double *epo, double *hpo, double *edo) override {
    HostLattice &h = *host;
    const int E = h.E, G = h.G, nh = h.nh;
    DL_CUDA(cudaStreamSynchronize(stream));
    const size_t NG = static_cast<size_t>(E) * G;
    std::vector<T> a, b;
    std::vector<double> d;
    if (h.plastic) {
      a.resize(NG * 6);
      b.resize(NG * std::max(1, nh));
      d.resize(NG);
      DL_CUDA(cudaMemcpy(a.data(), ep.p, a.size() * sizeof(T), cudaMemcpyDeviceToHost));
      DL_CUDA(cudaMemcpy(b.data(), alpha.p, b.size() * sizeof(T), cudaMemcpyDeviceToHost));
      DL_CUDA(cudaMemcpy(d.data(), ediss.p, d.size() * sizeof(double), cudaMemcpyDeviceToHost));
    }
    for (int e = 0; e < E; ++e) {
      const int ei = h.elem_new[e];
      for (int g = 0; g < G; ++g) {
        const size_t o = static_cast<size_t>(e) * G + g;
        for (int k = 0; k < 6; ++k)
          if (epo) epo[o * 6 + k] = h.plastic ? double(a[(static_cast<size_t>(g) * 6 + k) * E + ei]) : 0.0;
        for (int k = 0; k < 7; ++k)
          if (hpo) hpo[o * 7 + k] = (h.plastic && k < nh) ? double(b[(static_cast<size_t>(g) * nh + k) * E + ei]) : 0.0;
        if (edo) edo[o] = h.plastic ? d[static_cast<size_t>(g) * E + ei] : 0.0;
      }
    }
  }

  uint32_t error_word() override {
    uint32_t w = 0;
    DL_CUDA(cudaStreamSynchronize(stream));
    DL_CUDA(cudaMemcpy(&w, err.p, sizeof w, cudaMemcpyDeviceToHost));
    // a wait that ran out left the arrival word mid-count and the abort flag
    // set: the next launch starts from a clean barrier
    if (w & DL_EW_TIMEOUT) reset_barrier();
    return w;
  }

  void reset_barrier() {
    GridBarrier gb{};
    DL_CUDA(cudaMemcpy(&gb, barrier.p, sizeof gb, cudaMemcpyDeviceToHost));
    gb.count = 0;
    gb.abort = 0;
    DL_CUDA(cudaMemcpy(barrier.p, &gb, sizeof gb, cudaMemcpyHostToDevice));
  }

  void set_barrier_test(uint32_t limit_us, uint32_t phantom) override {
    DL_CUDA(cudaStreamSynchronize(stream));
    GridBarrier gb{};
    gb.limit_us = limit_us;
    gb.phantom = phantom;
    DL_CUDA(cudaMemcpy(barrier.p, &gb, sizeof gb, cudaMemcpyHostToDevice));
  }

  void clear_error() override {
    DL_CUDA(cudaStreamSynchronize(stream));
    DL_CUDA(cudaMemset(err.p, 0, err.bytes));
    reset_barrier();
  }

  void group_sums(int n, const int32_t *nodes, double *resp, double *load) override {
    HostLattice &h = *host;
    // internal force of the last step (fint of the state before it, plus
    // contact and the gyroscopic moment), as GroupOutputModule samples "resp"
    if (resp && !m.fint_last)
      throw std::invalid_argument("group output recording is off: call dl_set_group_output(h, 1) before dl_run");
    std::vector<double> f(static_cast<size_t>(h.N) * 6);
    DL_CUDA(cudaStreamSynchronize(stream));
    if (resp) DL_CUDA(cudaMemcpy(f.data(), fint_last.p, f.size() * sizeof(double), cudaMemcpyDeviceToHost));
    for (int i = 0; i < n; ++i)
      if (nodes[i] < 0 || nodes[i] >= h.N) throw std::invalid_argument("group node out of range");
    for (int k = 0; k < 6; ++k) {
      double s = 0.0;
      for (int i = 0; i < n; ++i) s += f[static_cast<size_t>(k) * h.N + h.node_new[nodes[i]]];
      if (resp) resp[k] = s;
      if (load) load[k] = 0.0;
    }
    // loads at the last completed step
    if (load) {
      std::vector<char> in(h.N, 0);
      for (int i = 0; i < n; ++i) in[nodes[i]] = 1;
      for (int ni = 0; ni < h.N; ++ni) {
        if (!in[h.node_old[ni]]) continue;
        for (int b = h.bc_ptr[ni]; b < h.bc_ptr[ni + 1]; ++b) {
          const BcTerm &bt = h.bc[b];
          if (bt.kind != BCD_NEUMANN) continue;
          double sc = 1.0;
          if (bt.scale >= 0) {
            const double vars[3] = {t, static_cast<double>(step), h.dt};
            sc = evalExpr(h.scales[bt.scale].expr.get(), vars);
          }
          load[bt.dof] += bt.factor * sc;
        }
      }
    }
  }
};

}  // namespace dl

// ---------------------------------------------------------------------------
// C ABI
// ---------------------------------------------------------------------------
struct dl_handle_s {
  std::unique_ptr<dl::EngineBase> eng;
};

namespace dl {
// the output modules' view of an engine handle
class HandleOutput final : public OutputHost {
 public:
  explicit HandleOutput(EngineBase &e) : e_(e) {}
  int n_nodes() override { return e_.host->N; }
  int n_elems() override { return e_.host->E; }
  int nodes_per_elem() override { return e_.host->nen; }
  void reference_coords(double *X0) override { std::copy(e_.host->X0.begin(), e_.host->X0.end(), X0); }
  void connectivity(int32_t *conn) override {
    const HostLattice &h = *e_.host;
    const int n = h.nen;
    for (int ei = 0; ei < h.E; ++ei) {
      const int eo = h.elem_old[ei];
      for (int a = 0; a < n; ++a)
        conn[static_cast<size_t>(eo) * n + a] = h.node_old[h.conn[static_cast<size_t>(ei) * n + a]];
    }
  }
  void state(double *u, double *th, double *v) override { e_.get_state(u, th, v); }
  void internal_force(const double *u, const double *th, double *f) override { e_.internal_force(u, th, f); }
  void external_force(double *f) override { e_.external_force(f); }
  void element_table(const std::string &name, double *out) override { e_.element_table(name, out); }
  void energies(dl_energies *en) override {
    e_.fetch_last_energies();
    *en = e_.last;
  }
  void time(double *t, double *dt, int64_t *step) override { e_.get_time(t, dt, step, nullptr); }
  void run(int64_t n) override {
    e_.run(n);
    const uint32_t w = e_.error_word();
    if (w) throw std::runtime_error("device error word " + std::to_string(w) + " during the run");
  }
  bool adaptive() override { return e_.adaptive(); }

 private:
  EngineBase &e_;
};
}  // namespace dl

namespace {

int set_err(int code, const std::string &msg) {
  dl::g_last_error = msg;
  return code;
}

template <class F>
int guard(F &&f) {
  try {
    f();
    return DL_OK;
  } catch (const dl::CudaError &e) {
    return set_err(DL_ERR_CUDA, e.what());
  } catch (const std::invalid_argument &e) {
    return set_err(DL_ERR_INVALID, e.what());
  } catch (const dl::UnsupportedError &e) {
    return set_err(DL_ERR_UNSUPPORTED, e.what());
  } catch (const dl::MassError &e) {
    return set_err(DL_ERR_MASS, e.what());
  } catch (const std::bad_alloc &) {
    return set_err(DL_ERR_NOMEM, "host allocation failed");
  } catch (const std::exception &e) {
    return set_err(DL_ERR_PARSE, e.what());
  }
}

int require_device() {
  int n = 0;
  if (cudaGetDeviceCount(&n) != cudaSuccess || n == 0) {
    cudaGetLastError();
    return set_err(DL_ERR_NO_DEVICE, "no CUDA device: the engine has no CPU path");
  }
  return DL_OK;
}

}  // namespace

DL_API const char *dl_last_error(void) { return dl::g_last_error.c_str(); }

DL_API const char *dl_version(void) { return "dynlattice-b200 0.1 (sm_100a)"; }

DL_API int dl_device_binary_version(int32_t *version) {
  if (!version) return set_err(DL_ERR_INVALID, "null argument");
  int rc = require_device();
  if (rc) return rc;
  cudaFuncAttributes a{};
  const cudaError_t e = cudaFuncGetAttributes(&a, dl::aot_kernels<double>(false).internal_force);
  if (e != cudaSuccess) {
    cudaGetLastError();
    return set_err(DL_ERR_CUDA, cudaGetErrorString(e));
  }
  *version = a.binaryVersion;
  return DL_OK;
}

DL_API int dl_device_count(int *count) {
  int n = 0;
  if (cudaGetDeviceCount(&n) != cudaSuccess) {
    cudaGetLastError();
    n = 0;
  }
  if (count) *count = n;
  return DL_OK;
}

DL_API int dl_create(const dl_model_desc *desc, int precision, dl_handle **out) {
  if (!desc || !out) return set_err(DL_ERR_INVALID, "null argument");
  if (precision != DL_PLAIN_FP64 && precision != DL_MIXED) return set_err(DL_ERR_INVALID, "bad precision");
  int rc = require_device();
  if (rc) return rc;
  return guard([&] {
    auto hl = dl::build_lattice(*desc, precision == DL_MIXED);
    auto h = std::make_unique<dl_handle_s>();
    if (precision == DL_MIXED)
      h->eng = std::make_unique<dl::Engine<float>>(std::move(hl), precision);
    else
      h->eng = std::make_unique<dl::Engine<double>>(std::move(hl), precision);
    *out = h.release();
  });
}

DL_API int dl_create_batch(const dl_model_desc *descs, int32_t n, int precision, dl_handle **out) {
  if (!descs || !out || n <= 0) return set_err(DL_ERR_INVALID, "null argument or empty batch");
  if (precision != DL_PLAIN_FP64 && precision != DL_MIXED) return set_err(DL_ERR_INVALID, "bad precision");
  int rc = require_device();
  if (rc) return rc;
  return guard([&] {
    auto hl = dl::build_batch(descs, n, precision == DL_MIXED);
    auto h = std::make_unique<dl_handle_s>();
    if (precision == DL_MIXED)
      h->eng = std::make_unique<dl::Engine<float>>(std::move(hl), precision);
    else
      h->eng = std::make_unique<dl::Engine<double>>(std::move(hl), precision);
    *out = h.release();
  });
}

DL_API int dl_batch_get_state(dl_handle *h, int32_t lattice, double *u, double *theta, double *v) {
  if (!h) return set_err(DL_ERR_INVALID, "null handle");
  const dl::HostLattice &hl = *h->eng->host;
  if (lattice < 0 || lattice >= hl.n_lat) return set_err(DL_ERR_INVALID, "lattice index out of range");
  return guard([&] {
    const size_t N = hl.N;
    std::vector<double> U(N * 3), TH(N * 3), V(N * 6);
    h->eng->get_state(U.data(), TH.data(), V.data());
    const size_t a = hl.n_lat > 1 ? hl.lat_node_off[lattice] : 0;
    const size_t b = hl.n_lat > 1 ? hl.lat_node_off[lattice + 1] : N;
    if (u) std::copy(U.begin() + a * 3, U.begin() + b * 3, u);
    if (theta) std::copy(TH.begin() + a * 3, TH.begin() + b * 3, theta);
    if (v) std::copy(V.begin() + a * 6, V.begin() + b * 6, v);
  });
}

DL_API int dl_batch_get_energies(dl_handle *h, int32_t lattice, dl_energies *e) {
  if (!h || !e) return set_err(DL_ERR_INVALID, "null argument");
  return guard([&] { h->eng->batch_energies(lattice, e); });
}

DL_API int dl_batch_sizes(dl_handle *h, int32_t *n_lattices, int32_t *node_offsets, int32_t *elem_offsets) {
  if (!h) return set_err(DL_ERR_INVALID, "null handle");
  const dl::HostLattice &hl = *h->eng->host;
  if (n_lattices) *n_lattices = hl.n_lat;
  for (int i = 0; i <= hl.n_lat; ++i) {
    if (node_offsets) node_offsets[i] = hl.n_lat > 1 ? hl.lat_node_off[i] : (i ? hl.N : 0);
    if (elem_offsets) elem_offsets[i] = hl.n_lat > 1 ? hl.lat_elem_off[i] : (i ? hl.E : 0);
  }
  return DL_OK;
}

DL_API int dl_contact_pairs(dl_handle *h, int64_t *n_pairs, int32_t *pairs, double *gaps, int64_t max_pairs) {
  if (!h) return set_err(DL_ERR_INVALID, "null handle");
  return guard([&] { h->eng->contact_pairs(n_pairs, pairs, gaps, max_pairs); });
}

DL_API int dl_adjoint_radius(dl_handle *h, int64_t nsteps, int32_t checkpoint_every, int32_t n_params,
                             const int32_t *elem_param, int32_t n_react_nodes, const int32_t *react_nodes,
                             int32_t react_dof, double react_weight, double *objective, double *grad) {
  if (!h || !grad || n_params <= 0 || (n_react_nodes > 0 && !react_nodes))
    return set_err(DL_ERR_INVALID, "null or inconsistent argument");
  return guard([&] {
    h->eng->adjoint_radius(nsteps, checkpoint_every, n_params, elem_param, n_react_nodes, react_nodes, react_dof,
                           react_weight, objective, grad);
  });
}

DL_API int dl_adjoint_branch_mode(dl_handle *h, int32_t mode) {
  if (!h) return set_err(DL_ERR_INVALID, "null handle");
  if (mode < 0 || mode > 2) return set_err(DL_ERR_INVALID, "branch mode must be 0, 1 or 2");
  h->eng->br_mode = mode;
  return DL_OK;
}

DL_API int dl_adjoint_branch_tape(dl_handle *h, int32_t get, uint8_t *tape, int64_t bytes, int64_t *peak_step,
                                  double *peak_sign) {
  if (!h) return set_err(DL_ERR_INVALID, "null handle");
  dl::EngineBase &e = *h->eng;
  if (get) {
    if (peak_step) *peak_step = e.br_peak_step;
    if (peak_sign) *peak_sign = e.br_peak_sign;
    if (!tape) {
      if (bytes < 0) return set_err(DL_ERR_INVALID, "negative size");
      return DL_OK;
    }
    if (bytes != static_cast<int64_t>(e.br_host.size()))
      return set_err(DL_ERR_INVALID, "tape size differs from the recorded tape");
    std::copy(e.br_host.begin(), e.br_host.end(), tape);
    return DL_OK;
  }
  if (!tape || bytes <= 0 || !peak_step || !peak_sign) return set_err(DL_ERR_INVALID, "null argument");
  e.br_host.assign(tape, tape + bytes);
  e.br_peak_step = *peak_step;
  e.br_peak_sign = *peak_sign < 0.0 ? -1.0 : 1.0;
  return DL_OK;
}

DL_API int dl_adjoint_branch_bytes(dl_handle *h, int64_t *bytes) {
  if (!h || !bytes) return set_err(DL_ERR_INVALID, "null argument");
  *bytes = static_cast<int64_t>(h->eng->br_host.size());
  return DL_OK;
}

DL_API int dl_set_threads(dl_handle *h, int32_t threads) {
  if (!h || !(threads == 0 || threads == 32 || threads == 64 || threads == 128 || threads == 256))
    return set_err(DL_ERR_INVALID, "threads per block must be 0 (automatic), 32, 64, 128 or 256");
  return guard([&] { h->eng->set_threads(threads); });
}

DL_API int dl_autotune(dl_handle *h, int64_t steps, int32_t *best_mode, int32_t *best_threads, double *best_ms) {
  if (!h || steps <= 0) return set_err(DL_ERR_INVALID, "bad argument");
  return guard([&] { h->eng->autotune(steps, best_mode, best_threads, best_ms); });
}

DL_API int dl_set_group_output(dl_handle *h, int32_t on) {
  if (!h) return DL_ERR_INVALID;
  return guard([&] { h->eng->set_group_output(on != 0); });
}

DL_API int dl_set_integrator(dl_handle *h, const dl_integrator_desc *d) {
  if (!h || !d) return set_err(DL_ERR_INVALID, "null argument");
  return guard([&] { h->eng->set_integrator(*d); });
}

DL_API int dl_get_time(dl_handle *h, double *t, double *dt, int64_t *step, int64_t *rejected) {
  if (!h) return set_err(DL_ERR_INVALID, "null handle");
  return guard([&] { h->eng->get_time(t, dt, step, rejected); });
}

DL_API int dl_get_sample_times(dl_handle *h, double *times, int64_t max_samples) {
  if (!h || !times) return set_err(DL_ERR_INVALID, "null argument");
  return guard([&] {
    const auto &v = h->eng->sample_t;
    const int64_t n = std::min<int64_t>(max_samples, static_cast<int64_t>(v.size()));
    for (int64_t i = 0; i < n; ++i) times[i] = v[i];
  });
}

DL_API int dl_element_table(dl_handle *h, const char *name, double *out) {
  if (!h || !name || !out) return set_err(DL_ERR_INVALID, "null argument");
  return guard([&] { h->eng->element_table(name, out); });
}

DL_API int dl_write_vtu(dl_handle *h, const char *path, int32_t node_data) {
  if (!h || !path) return set_err(DL_ERR_INVALID, "null argument");
  return guard([&] {
    dl::HandleOutput out(*h->eng);
    dl::write_vtu(out, path, node_data);
  });
}

DL_API int dl_write_pvd(const char *path, int32_t n, const double *times, const char *const *files) {
  if (!path || n < 0 || (n > 0 && (!times || !files))) return set_err(DL_ERR_INVALID, "null argument");
  return guard([&] {
    std::vector<double> t(times, times + n);
    std::vector<std::string> f;
    for (int i = 0; i < n; ++i) f.emplace_back(files[i]);
    dl::write_pvd(path, t, f);
  });
}

DL_API int dl_trim_retained_memory(void) {
  return guard([&] { dl::trim_retained_pool(); });
}

DL_API int dl_set_tape_budget(dl_handle *h, int64_t bytes) {
  if (!h) return set_err(DL_ERR_INVALID, "null handle");
  return guard([&] { h->eng->set_tape_budget(bytes); });
}

DL_API int dl_launch_count(dl_handle *h, int64_t *n) {
  if (!h || !n) return set_err(DL_ERR_INVALID, "null argument");
  return guard([&] { *n = h->eng->launch_count(); });
}

DL_API int dl_joint_contact_pairs(dl_handle *h, int64_t *n_pairs, int32_t *pairs, double *gaps, int64_t max_pairs) {
  if (!h) return set_err(DL_ERR_INVALID, "null handle");
  return guard([&] { h->eng->joint_contact_pairs(n_pairs, pairs, gaps, max_pairs); });
}

DL_API int dl_contact_stats(dl_handle *h, int64_t *n_candidates, int64_t *n_builds) {
  if (!h) return set_err(DL_ERR_INVALID, "null handle");
  return guard([&] { h->eng->contact_stats(n_candidates, n_builds); });
}

DL_API int dl_plate_reaction(dl_handle *h, double *out) {
  if (!h || !out) return set_err(DL_ERR_INVALID, "null argument");
  return guard([&] { h->eng->plate_reaction(out); });
}

struct dl_pro_s {
  std::unique_ptr<dl::ProModel> model;
};

DL_API int dl_pro_open(const char *pro_path, dl_pro **out) {
  if (!pro_path || !out) return set_err(DL_ERR_INVALID, "null argument");
  *out = nullptr;
  try {
    auto p = std::make_unique<dl_pro>();
    p->model = dl::load_pro(pro_path);
    *out = p.release();
    return DL_OK;
  } catch (const std::exception &e) {
    const std::string m = e.what();
    return set_err(m.rfind("cannot open", 0) == 0 ? DL_ERR_IO : DL_ERR_PARSE, m);
  }
}

DL_API int dl_pro_desc(dl_pro *p, const dl_model_desc **desc) {
  if (!p || !desc) return set_err(DL_ERR_INVALID, "null argument");
  *desc = &p->model->desc;
  return DL_OK;
}

DL_API int dl_pro_steps(dl_pro *p, int64_t *nsteps) {
  if (!p || !nsteps) return set_err(DL_ERR_INVALID, "null argument");
  *nsteps = p->model->steps;
  return DL_OK;
}

DL_API int dl_pro_group(dl_pro *p, const char *name, int32_t *n_nodes, const int32_t **nodes) {
  if (!p || !name || !n_nodes) return set_err(DL_ERR_INVALID, "null argument");
  auto it = p->model->groups.find(name);
  if (it == p->model->groups.end()) return set_err(DL_ERR_INVALID, std::string("no node group ") + name);
  *n_nodes = static_cast<int32_t>(it->second.size());
  if (nodes) *nodes = it->second.data();
  return DL_OK;
}

DL_API int dl_pro_integrator(dl_pro *p, dl_integrator_desc *out) {
  if (!p || !out) return set_err(DL_ERR_INVALID, "null argument");
  *out = p->model->integ;
  return DL_OK;
}

DL_API int dl_pro_run(dl_pro *p, dl_handle *h, const char *out_dir, int64_t max_steps, int64_t *steps_run) {
  if (!p || !h) return set_err(DL_ERR_INVALID, "null argument");
  return guard([&] {
    dl::HandleOutput out(*h->eng);
    const int64_t n = dl::run_pro(out, *p->model, out_dir ? out_dir : "", max_steps);
    if (steps_run) *steps_run = n;
  });
}

DL_API int dl_pro_end_time(dl_pro *p, double *t_end) {
  if (!p || !t_end) return set_err(DL_ERR_INVALID, "null argument");
  *t_end = p->model->t_end;
  return DL_OK;
}

DL_API int dl_pro_note(dl_pro *p, int32_t i, int32_t *n, const char **text) {
  if (!p) return set_err(DL_ERR_INVALID, "null argument");
  const auto &notes = p->model->notes;
  if (n) *n = static_cast<int32_t>(notes.size());
  if (text) {
    if (i < 0 || i >= static_cast<int32_t>(notes.size())) return set_err(DL_ERR_INVALID, "note index out of range");
    *text = notes[static_cast<size_t>(i)].c_str();
  }
  return DL_OK;
}

DL_API int dl_pro_close(dl_pro *p) {
  delete p;
  return DL_OK;
}

DL_API int dl_create_from_pro(const char *pro_path, int precision, dl_handle **out) {
  dl_pro *p = nullptr;
  int rc = dl_pro_open(pro_path, &p);
  if (rc) return rc;
  rc = dl_create(&p->model->desc, precision, out);
  if (rc == DL_OK && p->model->integ.kind != DL_INTEG_LEAPFROG) {
    rc = dl_set_integrator(*out, &p->model->integ);
    if (rc != DL_OK) {
      dl_destroy(*out);
      *out = nullptr;
    }
  }
  dl_pro_close(p);
  return rc;
}

DL_API int dl_destroy(dl_handle *h) {
  delete h;
  return DL_OK;
}

DL_API int dl_set_stream(dl_handle *h, void *stream) {
  if (!h) return set_err(DL_ERR_INVALID, "null handle");
  h->eng->stream = static_cast<cudaStream_t>(stream);
  return DL_OK;
}

DL_API int dl_set_exec_mode(dl_handle *h, int mode) {
  if (!h) return set_err(DL_ERR_INVALID, "null handle");
  if (mode != dl::EXEC_PERSISTENT && mode != dl::EXEC_STREAM && mode != dl::EXEC_GRAPH)
    return set_err(DL_ERR_INVALID, "bad mode");
  h->eng->exec_mode = mode;
  return DL_OK;
}

DL_API int dl_get_info(dl_handle *h, int32_t *jit_active, int32_t *persistent_blocks, const char **jit_log) {
  if (!h) return set_err(DL_ERR_INVALID, "null handle");
  h->eng->info(jit_active, persistent_blocks, jit_log);
  return DL_OK;
}

DL_API int dl_run(dl_handle *h, int64_t nsteps) {
  if (!h) return set_err(DL_ERR_INVALID, "null handle");
  if (nsteps < 0) return set_err(DL_ERR_INVALID, "negative step count");
  return guard([&] { h->eng->run(nsteps); });
}

DL_API int dl_set_sampling(dl_handle *h, int32_t every, int32_t n_watch, const int32_t *watch_nodes,
                           int64_t capacity) {
  if (!h) return set_err(DL_ERR_INVALID, "null handle");
  std::vector<int32_t> w;
  if (n_watch > 0) w.assign(watch_nodes, watch_nodes + n_watch);
  return guard([&] { h->eng->set_sampling(every, w, capacity); });
}

DL_API int dl_get_samples(dl_handle *h, int64_t *n_samples, int64_t *steps, double *node_rows,
                          dl_energies *energies, int64_t max_samples) {
  if (!h) return set_err(DL_ERR_INVALID, "null handle");
  return guard([&] { h->eng->get_samples(n_samples, steps, node_rows, energies, max_samples); });
}

DL_API int dl_clear_error(dl_handle *h) {
  if (!h) return set_err(DL_ERR_INVALID, "null handle");
  return guard([&] { h->eng->clear_error(); });
}

DL_API int dl_set_barrier_test(dl_handle *h, uint32_t limit_us, uint32_t phantom_blocks) {
  if (!h) return set_err(DL_ERR_INVALID, "null handle");
  if (phantom_blocks > 1) return set_err(DL_ERR_INVALID, "phantom_blocks must be 0 or 1");
  return guard([&] { h->eng->set_barrier_test(limit_us, phantom_blocks); });
}

DL_API int dl_get_error_word(dl_handle *h, uint32_t *word) {
  if (!h || !word) return set_err(DL_ERR_INVALID, "null argument");
  return guard([&] { *word = h->eng->error_word(); });
}

static int status_of_word(uint32_t w) {
  if (w & DL_EW_RETURN_MAP) return set_err(DL_ERR_RETURN_MAP, "Too many iterations in plasticity loop");
  if (w & DL_EW_TIMEOUT) return set_err(DL_ERR_TIMEOUT, "grid barrier wait timed out");
  if (w & DL_EW_NONFINITE) return set_err(DL_ERR_NONFINITE, "non-finite state");
  if (w & DL_EW_CONTACT_OVERFLOW) return set_err(DL_ERR_NOMEM, "contact pair list overflow");
  if (w & DL_EW_CONTACT_STALE)
    return set_err(DL_ERR_CONTACT, "contact candidate list went stale (a node moved beyond margin/2)");
  if (w & DL_EW_STEP_CONTROL)
    return set_err(DL_ERR_NONFINITE, "step control failed (non-finite error estimate or endless rejections)");
  return DL_OK;
}

DL_API int dl_synchronize(dl_handle *h) {
  if (!h) return set_err(DL_ERR_INVALID, "null handle");
  uint32_t w = 0;
  int rc = guard([&] { w = h->eng->error_word(); });
  if (rc) return rc;
  return status_of_word(w);
}

DL_API int dl_get_sizes(dl_handle *h, int32_t *n_nodes, int32_t *n_elems, int32_t *n_gauss, int64_t *step) {
  if (!h) return set_err(DL_ERR_INVALID, "null handle");
  if (n_nodes) *n_nodes = h->eng->host->N;
  if (n_elems) *n_elems = h->eng->host->E;
  if (n_gauss) *n_gauss = h->eng->host->G;
  if (step) *step = h->eng->step;
  return DL_OK;
}

DL_API int dl_get_state(dl_handle *h, double *u, double *theta, double *v) {
  if (!h) return set_err(DL_ERR_INVALID, "null handle");
  return guard([&] { h->eng->get_state(u, theta, v); });
}

DL_API int dl_set_state(dl_handle *h, const double *u, const double *theta, const double *v) {
  if (!h) return set_err(DL_ERR_INVALID, "null handle");
  return guard([&] { h->eng->set_state(u, theta, v); });
}

DL_API int dl_get_energies(dl_handle *h, dl_energies *e) {
  if (!h || !e) return set_err(DL_ERR_INVALID, "null argument");
  return guard([&] {
    h->eng->fetch_last_energies();
    *e = h->eng->last;
  });
}

DL_API int dl_internal_force(dl_handle *h, const double *u, const double *theta, double *fint) {
  if (!h || !u || !theta || !fint) return set_err(DL_ERR_INVALID, "null argument");
  return guard([&] { h->eng->internal_force(u, theta, fint); });
}

DL_API int dl_internal_force_static(dl_handle *h, const double *u_dev, const double *theta_dev, double *fint_dev) {
  if (!h || !u_dev || !theta_dev || !fint_dev) return set_err(DL_ERR_INVALID, "null argument");
  const char *why = "";
  const int rc = h->eng->internal_force_static(u_dev, theta_dev, fint_dev, &why);
  return rc == DL_OK ? DL_OK : set_err(rc, why);
}

DL_API int dl_get_history(dl_handle *h, double *plastic_strain, double *hard_params, double *dissipation) {
  if (!h) return set_err(DL_ERR_INVALID, "null handle");
  return guard([&] { h->eng->get_history(plastic_strain, hard_params, dissipation); });
}

DL_API int dl_group_sums(dl_handle *h, int32_t n_nodes, const int32_t *nodes, double *out_resp, double *out_load) {
  if (!h || (n_nodes > 0 && !nodes)) return set_err(DL_ERR_INVALID, "null argument");
  for (int i = 0; i < n_nodes; ++i)
    if (nodes[i] < 0 || nodes[i] >= h->eng->host->N) return set_err(DL_ERR_INVALID, "node out of range");
  return guard([&] { h->eng->group_sums(n_nodes, nodes, out_resp, out_load); });
}

DL_API int dl_inspect_setup(const dl_model_desc *desc, int precision, double *frames, double *strain0,
                            double *mass, double *rot_inertia) {
  if (!desc) return set_err(DL_ERR_INVALID, "null argument");
  return guard([&] {
    auto hl = dl::build_lattice(*desc, precision == DL_MIXED);
    const dl::HostLattice &h = *hl;
    const int E = h.E, G = h.G;
    for (int e = 0; e < E; ++e) {
      const int ei = h.elem_new[e];
      for (int s = 0; s < h.nen; ++s)
        for (int k = 0; k < 4; ++k)
          if (frames)
            frames[(static_cast<size_t>(e) * h.nen + s) * 4 + k] = h.qN[(static_cast<size_t>(s) * E + ei) * 4 + k];
      for (int g = 0; g < G; ++g)
        for (int k = 0; k < 3; ++k) {
          if (!strain0) continue;
          // Gamma0 = (Gamma0 - e3) + e3
          strain0[(static_cast<size_t>(e) * G + g) * 6 + k] =
              h.g0[(static_cast<size_t>(g) * 3 + k) * E + ei] + (k == 2 ? 1.0 : 0.0);
          strain0[(static_cast<size_t>(e) * G + g) * 6 + 3 + k] = h.k0[(static_cast<size_t>(g) * 3 + k) * E + ei];
        }
    }
    for (int n = 0; n < h.N; ++n) {
      const int ni = h.node_new[n];
      if (mass) mass[n] = h.mass[ni];
      if (rot_inertia) {
        dl::Q4<double> P{h.iframe[ni * 4], h.iframe[ni * 4 + 1], h.iframe[ni * 4 + 2], h.iframe[ni * 4 + 3]};
        double R[3][3];
        dl::qmat(P, R);
        for (int i = 0; i < 3; ++i)
          for (int j = 0; j < 3; ++j) {
            double acc = 0.0;
            for (int k = 0; k < 3; ++k) acc += R[i][k] * h.idiag[ni * 4 + k] * R[j][k];
            rot_inertia[static_cast<size_t>(n) * 9 + i * 3 + j] = acc;
          }
      }
    }
  });
}

DL_API int dl_jit_check(const dl_model_desc *desc, int precision, size_t *cubin_bytes, char *log, size_t log_size) {
  if (!desc) return set_err(DL_ERR_INVALID, "null argument");
  std::string l;
  bool ok = false;
  int rc = guard([&] {
    auto hl = dl::build_lattice(*desc, precision == DL_MIXED);
    if (!hl->plastic) throw std::invalid_argument("runtime compilation applies to elastoplastic lattices");
    const std::string code = dl::emitYieldPolicy(hl->yield_expr, hl->grad_exprs, precision == DL_MIXED);
    std::vector<char> cubin;
    std::vector<std::string> lowered;
    ok = dl::jit_compile(code, precision == DL_MIXED, &cubin, &lowered, &l);
    size_t bytes = ok ? cubin.size() : 0;
    if (ok) {  // and the adjoint kernels of the same model
      const std::string acode = dl::emitYieldAdjPolicy(hl->yield_expr, hl->grad_exprs, precision == DL_MIXED,
                                                       "__device__");
      ok = dl::jit_compile_adjoint(acode, precision == DL_MIXED, &cubin, &lowered, &l);
      bytes += ok ? cubin.size() : 0;
    }
    if (cubin_bytes) *cubin_bytes = ok ? bytes : 0;
  });
  if (log && log_size) {
    std::snprintf(log, log_size, "%s", l.c_str());
  }
  if (rc) return rc;
  return ok ? DL_OK : set_err(DL_ERR_CUDA, "runtime compilation failed: " + l);
}

DL_API int dl_yield_source(const char *yield_cond, int32_t n_deriv, const char *const *yield_deriv, int32_t n_vars,
                           const char *const *names, int32_t fp32, int32_t adjoint, int32_t host, char *buf,
                           int64_t buf_len, int64_t *needed) {
  if (!yield_cond || (n_deriv > 0 && !yield_deriv) || (n_vars > 0 && !names))
    return set_err(DL_ERR_INVALID, "null argument");
  return guard([&] {
    std::vector<std::string> nm;
    for (int i = 0; i < n_vars; ++i) nm.emplace_back(names[i]);
    dl::ExprPtr f = dl::parseExpr(yield_cond, nm);
    std::vector<dl::ExprPtr> gs;
    for (int k = 0; k < n_deriv; ++k) gs.push_back(dl::parseExpr(yield_deriv[k], nm));
    const std::string src = adjoint ? dl::emitYieldAdjPolicy(f, gs, fp32 != 0, host ? "inline" : "__device__")
                                    : dl::emitYieldPolicy(f, gs, fp32 != 0);
    if (needed) *needed = static_cast<int64_t>(src.size()) + 1;
    if (buf && buf_len > 0) {
      const size_t n = std::min<size_t>(src.size(), static_cast<size_t>(buf_len - 1));
      std::memcpy(buf, src.data(), n);
      buf[n] = 0;
    }
  });
}

DL_API int dl_eval_expression(const char *expr, int32_t n_vars, const char *const *names, const double *values,
                              double *out) {
  if (!expr || !out) return set_err(DL_ERR_INVALID, "null argument");
  return guard([&] {
    std::vector<std::string> nm;
    for (int i = 0; i < n_vars; ++i) nm.emplace_back(names[i]);
    dl::ExprPtr e = dl::parseExpr(expr, nm);
    // both the tree walker and the compiled program must agree
    double a = dl::evalExpr(e.get(), values);
    dl::ExprProgram p = dl::compileExprs({e});
    double b = 0.0;
    dl::runProgram(p, values, &b);
    const bool same = (a == b) || (std::isnan(a) && std::isnan(b)) ||
                      std::fabs(a - b) <= 1e-13 * std::max(std::fabs(a), std::fabs(b));
    if (!same) throw std::runtime_error("compiled program disagrees with the expression tree");
    *out = a;
  });
}
