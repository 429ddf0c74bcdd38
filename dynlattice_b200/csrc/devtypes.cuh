// Device data layout of one rod lattice (or a batch of lattices) and the
// kernel entry points.  All arrays live in HBM, engine-owned.
//
// Nodes (renumbered along a Morton curve so that elements gather neighbours):
//   pos   double4[N]    x, y, z, (unused)          -- FP64 state
//   rot   double4[N]    unit quaternion w,x,y,z    -- FP64 state
//   vel   double[6][N]  SoA, translational + spatial angular velocity
//   mass  double[N]     translational lumped mass
//   iframe T4[N]        principal frame P of the rotational inertia S = P D P^T
//   idiag  T4[N]        D (3 principal moments), w = unused; idinv: 1/D
//   imass  double[N]    1 / mass
//   slot_ptr int[N+1]   node n owns end-force slots [slot_ptr[n], slot_ptr[n+1]),
//                       one per incident element end, in element order
//   bc_ptr/bc           per-node boundary-condition terms
// Elements (Morton order of their midpoints):
//   conn  int2[E], invL0 double[E], L0 T[E]
//   qN    T4[2][E]      element-end frames Lambda_N (initRotation_)
//   g0    T[G*3][E]     Gamma0 - e3 ; k0 T[G*3][E]: K0  (initStrain_)
//   C     T[6][E]       diag(GkA, GkA, EA, EI1, EI2, GJ)
//   ec    T[2][E]       element variables of yield expressions: radius, area
//   ep    T[G*6][E], alpha T[G*nh][E], epsc T[G*6][E]: plastic strain,
//                       hardening parameters, committed total strain
//   ediss double[G][E]  dissipated energy per Gauss point
//   eslot int2[E]       slots of the element's two ends
//   ef    T[2E][6]      end forces in node-ordered slots: an element writes
//                       its two records, a node sums its contiguous run
// Plain-data device types of the engine, shared by the ahead-of-time build
// (nvcc) and the runtime-compiled kernels (NVRTC): no standard headers here.
#pragma once

#ifdef __CUDACC_RTC__
typedef long long int64_t;
typedef unsigned long long uint64_t;
typedef int int32_t;
typedef unsigned int uint32_t;
typedef unsigned char uint8_t;
#else
#include <cstdint>
#include <cuda_runtime.h>
#endif

namespace dl {

enum ExprOpCode : unsigned char {
  XO_CONST = 0, XO_ARG, XO_ADD, XO_SUB, XO_MUL, XO_DIV, XO_POW, XO_NEG, XO_ABS, XO_SQRT,
  XO_EXP, XO_LOG, XO_SIN, XO_COS, XO_TAN, XO_ATAN, XO_FLOOR, XO_CEIL, XO_SIGN, XO_MIN,
  XO_MAX, XO_MOD, XO_LT, XO_LE, XO_GT, XO_GE, XO_EQ, XO_NE, XO_AND, XO_OR, XO_NOT,
  XO_SELECT, XO_SQUARE, XO_COUNT
};

// One instruction: dst <- op(r[a], r[b], r[c]); XO_CONST reads consts[a | b<<8],
// XO_ARG reads args[a].
struct ExprOp {
  uint8_t op, dst, a, b, c, pad0, pad1, pad2;
};

constexpr int kMaxExprRegs = 48;
constexpr int kMaxExprOps = 1024;

enum BcKindDev : int { BCD_DIRICHLET = 0, BCD_NEUMANN = 1 };

struct BcTerm {
  int32_t kind;
  int32_t dof;
  int32_t scale;    // column of the per-step scale table, -1 = constant 1
  int32_t pad;
  double factor;
};

template <class T>
struct Vec4 {
  using type = double4;
};
template <>
struct Vec4<float> {
  using type = float4;
};

// Expression program in device memory
template <class T>
struct DevProg {
  const ExprOp *ops = nullptr;
  const T *consts = nullptr;
  int n_ops = 0;
  int out0 = 0;          // register of the first output
  const uint8_t *outs = nullptr;
};

struct SampleSpec {
  int every = 0;           // sample when step % every == 0
  int n_watch = 0;
  const int32_t *watch_slot = nullptr;  // [N] -1 or slot
  double *rows = nullptr;  // [capacity][n_watch][13]: x(3) q(4) v(6)
  double *energy = nullptr;  // [capacity][5]
  int64_t *steps = nullptr;  // [capacity]
  int64_t capacity = 0;
  int64_t *count = nullptr;  // device counter of written samples
  double *times = nullptr;   // [capacity] time of each sample (predictor-corrector runs)
};

template <class T>
struct DevModel {
  using T4 = typename Vec4<T>::type;
  int N = 0, E = 0, G = 2, nh = 0;
  int plastic = 0;
  int gyro = 1, so3 = 1;
  int lumped = 0;  // diagonal node mass (DL_MASS_LUMPED)
  // rigid tie groups: tie_nodes[tie_ptr[n] .. tie_ptr[n + 1]) are the members
  // of node n's group, master first (empty for untied nodes); every member
  // carries the group's combined mass and boundary conditions (null: no ties)
  const int32_t *tie_ptr = nullptr;
  const int32_t *tie_nodes = nullptr;
  double dt = 0.0;
  // nodes
  double4 *pos = nullptr;
  double4 *rot = nullptr;
  double *vel = nullptr;
  const double *mass = nullptr;
  const double *imass = nullptr;
  const T4 *iframe = nullptr;
  const T4 *idiag = nullptr;
  const T4 *idinv = nullptr;
  const int32_t *slot_ptr = nullptr;
  const int32_t *bc_ptr = nullptr;
  const BcTerm *bc = nullptr;
  // elements
  const int2 *conn = nullptr;
  const int2 *eslot = nullptr;
  const double *invL0 = nullptr;
  const T *L0 = nullptr;
  const T4 *qN = nullptr;
  const T *g0 = nullptr;
  const T *k0 = nullptr;
  const T *C = nullptr;
  const T *ec = nullptr;
  T *ep = nullptr;
  T *alpha = nullptr;
  T *epsc = nullptr;
  double *ediss = nullptr;
  T *ef = nullptr;
  // elements of 3 or 4 nodes (nen > 2; two-node elements use conn/eslot):
  // node and end-force slot of local node a at conn_n/eslot_n[a * E + e];
  // per Gauss point its weight and the shape gradients,
  // shp[(e * G + g) * (nen + 1) + {0, 1 + a}]; the shape values Nq[a][g];
  // qN then holds nen frames per element ([nen][E])
  int nen = 2;
  const int32_t *conn_n = nullptr;
  const int32_t *eslot_n = nullptr;
  const double *shp = nullptr;
  // their reference strains in FP64, [G*6][E] (Gamma0 - e3, K0): the strain is
  // the FP64 difference, rounded to T once (a curved rod's K0 is far larger
  // than a deformation's change of it)
  const double *s0_n = nullptr;
  double Nq[4][4];
  // plasticity law
  DevProg<T> yield;     // f(args)
  DevProg<T> grad;      // gradient, 6 + nh outputs
  T H[7][7];
  int max_iter = 20;
  T prec = T(1e-5);
  // per-step scale table of the running chunk: scales[(step - scale_step0) * n_scales + s]
  const double *scales = nullptr;
  int n_scales = 0;
  int64_t scale_step0 = 0;
  // batches of independent lattices: per-node dt and lattice index, per-element
  // lattice index, per-lattice energies of the final step of a launch [n_lat][5]
  int n_lat = 1;
  const double *dtn = nullptr;
  const int32_t *nlat = nullptr;
  const int32_t *elat = nullptr;
  double *lat_energy = nullptr;
  // rod--rod contact: candidate pairs (element indices, reference orientation),
  // contact/plate forces accumulated as internal force per node [N][3]
  int n_pairs = 0;
  const int2 *pairs = nullptr;
  double c_radius = 0.0, c_ks = 0.0, c_kn = 0.0;
  // per candidate pair: closed in this step [n_pairs], and its node forces
  // [n_pairs][4][3] when closed; the node-ordered index of the pair ends
  // (c_ptr [N + 1], c_ent: p * 4 + end), summed by each node in that order
  uint8_t *pclosed = nullptr;
  double *pforce = nullptr;
  const int4 *c_quad = nullptr;  // [n_pairs] the pair's end nodes (A0, A1, B0, B1), for its gathers
  const uint32_t *c_ptr = nullptr;
  // [N] the last step at which a rod or joint contact pair of the node was
  // closed (-1: none yet), set by the pair in the element phase: the node
  // phase walks a node's pair ends only in such a step (null: always)
  int64_t *cstamp = nullptr;
  const int32_t *c_ent = nullptr;
  double *pair_gap = nullptr;         // [n_pairs] gap of the last energy step (closed pairs, else +inf)
  const double *xbuild = nullptr;     // [N][3] positions at the last list build
  double half_margin = 0.0;
  // added point masses (MassModel): [6][N] diagonal of the node mass matrix, or null
  const double *madd = nullptr;
  // joint contact: candidate joint pairs (internal node indices, A before B
  // in the joint list), joint radius and penalty; per pair closed flag and
  // forces [n_jpairs][2][3], node-ordered index (j_ptr, j_ent: p * 2 + end)
  int n_jpairs = 0;
  const int2 *jpairs = nullptr;
  uint8_t *jclosed = nullptr;
  double *jforce = nullptr;
  const uint32_t *j_ptr = nullptr;
  const int32_t *j_ent = nullptr;
  double j_radius = 0.0, j_k = 0.0;
  double *jpair_gap = nullptr;        // [n_jpairs] gap of the last energy step (closed pairs, else +inf)
  // rigid plates (engine extension)
  int n_plates = 0;
  double plate_n[2][3], plate_p0[2][3], plate_v[2][3], plate_k[2];
  double t0 = 0.0;                    // time at step tstep0 (set per launch)
  int64_t tstep0 = 0;
  double *plate_force = nullptr;      // [2][3] plate reaction of the last energy step
  // diagnostics
  uint32_t *err = nullptr;
  double *wext = nullptr;   // accumulated external work
  double *fint_last = nullptr;  // [6][N] internal force of the last step of a launch (GroupOutput "resp")
  // state tape of the adjoint's recomputation (null in plain runs): slot
  // s = step - tp_step0 holds the state after that step; tp_pos/tp_rot [slot][N],
  // tp_vel [slot][6][N], tp_ep/tp_epsc [slot][G*6*E], tp_al [slot][G*nh*E]
  double4 *tp_pos = nullptr;
  double4 *tp_rot = nullptr;
  double *tp_vel = nullptr;
  T *tp_ep = nullptr;
  T *tp_al = nullptr;
  T *tp_epsc = nullptr;
  int64_t tp_step0 = 0;
  // per-step sum of one internal-force component over a node group (null in
  // plain runs): grp_hist[step - grp_step0] += fint[grp_dof] of flagged nodes
  const uint8_t *grp_flag = nullptr;
  double *grp_hist = nullptr;
  int grp_dof = 0;
  int64_t grp_step0 = 0;
  // return-map branch tape of a differentiated run (null in plain runs):
  // br[((step - br_step0 - 1) * G + g) * E + e] = cutting-plane iterations of
  // Gauss point g of element e in that step; br_mode 1 records them, 2
  // imposes them in place of the stop test f < precision
  uint8_t *br = nullptr;
  int br_mode = 0;
  int64_t br_step0 = 0;
};

// Time and step of a predictor-corrector run, kept on the device between
// launches (the accepted steps and the adapted dt are decided there).
struct MilneCtl {
  double t;
  double dt;
  int64_t step;
  int64_t rejected;
};

// Buffers and constants of the MilneDevice predictor-corrector
// (MilneDeviceModule.cpp:41-118, ExplicitModule::commit :291-334).
template <class T>
struct MilneDev {
  double4 *pos_pre, *rot_pre;  // predicted, then corrected node state
  double *vel_pre;             // [6][N]
  T *ep_new, *alpha_new, *epsc_new;  // history of the corrector's force evaluation
  double *ediss_new;
  double *partial;             // [gridDim][3] per-block sums of the error norms and the external work
  MilneCtl *ctl;
  double *wext;                // accumulated external work
  DevProg<double> scale_prog;  // LoadScale functions of (t, i, deltaTime), one output each
  int n_scales;
  double prec, min_dt, max_dt, safety, incr, decr, len_scale;
};
constexpr int kMilneMaxScales = 32;
constexpr int kMilneMaxAttempts = 1000;  // per step; beyond it the run stops with an error

// Lanes per element in the element adjoint kernel: one per Gauss point,
// rounded up to a divisor of the warp size so that an element's lanes share
// a warp.
__host__ __device__ inline int adj_lanes(int G) { return G <= 1 ? 1 : (G == 2 ? 2 : 4); }

// Adjoint state and objective of the reverse sweep (adjoint kernels).
template <class T>
struct AdjCtx {
  double *lx = nullptr;     // [3][N] node part of the translational adjoint
  double *lth = nullptr;    // [3][N] rotational adjoint (spatial tangent)
  double *lv = nullptr;     // [6][N] velocity adjoint
  double *lf = nullptr;     // [6][N] adjoint of the internal force of the step
  double *aslot = nullptr;  // [2E][6] element-end contributions (translation 3, rotation 3)
  double *lep = nullptr;    // [G*6][E] history adjoints (component-major, as DevModel::ep)
  double *lal = nullptr;    // [G*nh][E]
  double *lepsc = nullptr;  // [G*6][E]
  double *lC = nullptr;     // [6][E] accumulated adjoint of the section stiffness
  double *lec = nullptr;    // [2][E] of the yield-expression variables (radius, area)
  double *lmass = nullptr;  // [N] of the translational node mass
  double *lS = nullptr;     // [6][N] of the node inertia (xx yy zz xy xz yz, symmetric)
  double w_diss = 0.0;      // objective weight of the final dissipated energy
  double w_peak = 0.0;      // weight of the peak group force ...
  int64_t peak_step = -1;   // ... reached at this step
  int peak_dof = 0;
  const uint8_t *peak_flag = nullptr;
};

// Grid barrier of the persistent kernels.  count: arrival word whose bit 31
// flips when every block of the launch has arrived (block 0 adds
// 0x80000000 - (blocks - 1), the others 1), so it returns to its low bits
// after every barrier; abort: set by a block whose wait ran out, seen by all
// others; limit_us: bound of one wait (0: 2 s); phantom: blocks the arrival
// count expects beyond the launch's own (0; the failure-path test sets 1 so
// that the wait runs out without a fault).
struct GridBarrier {
  unsigned int count;
  unsigned int phantom;
  unsigned int abort;
  unsigned int limit_us;
};

struct StepCtx {
  int64_t step0;        // last completed step before this launch
  int nsteps;
  int64_t sample_base;  // samples written before this launch
  double *wstep;        // [nsteps] external work done in each step
  double *last_energy;  // [5] energies of the final step of this launch (zeroed by
                        // the previous launch)
  double *next_energy;  // [5] slot of the following launch, zeroed by this one
};


}  // namespace dl
