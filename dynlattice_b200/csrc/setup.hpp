// Host-side set-up of one lattice: everything the INIT action of the
// reference computes once (frames, reference strains, lumped masses, BC
// tables), in FP64, plus the engine's own layout decisions (Morton
// renumbering, incidence CSR).  Output is plain host arrays in the engine's
// internal numbering, ready to be uploaded.
#pragma once

#include <cstdint>
#include <memory>
#include <string>
#include <vector>

#include "../../include/dynlattice.h"
#include "engine.hpp"
#include "expr.hpp"

namespace dl {

struct ScaleFn {
  std::string src;
  ExprPtr expr;   // variables: t, i, deltaTime
};

struct HostLattice {
  int N = 0, E = 0, G = 2, nh = 0;
  bool plastic = false;
  bool so3 = true, gyro = true;
  bool lumped = false;  // DL_MASS_LUMPED: diagonal node mass, no gyroscopic term
  // rigid tie groups (internal numbering): members of node n's group are
  // tie_nodes[tie_ptr[n] .. tie_ptr[n + 1]), master first; empty when untied
  bool ties = false;
  std::vector<int32_t> tie_ptr, tie_nodes;
  double dt = 0.0;
  // numbering: node_new[old] and node_old[new], same for elements
  std::vector<int32_t> node_new, node_old, elem_new, elem_old;
  std::vector<double> X0;           // [N][3] original numbering
  // node arrays (internal numbering)
  std::vector<double> pos;          // [N][4]
  std::vector<double> rot;          // [N][4]
  std::vector<double> vel;          // [6][N]
  std::vector<double> mass;         // [N]
  std::vector<double> iframe;       // [N][4] quaternion P
  std::vector<double> idiag;        // [N][4] principal moments
  std::vector<int32_t> slot_ptr;   // [N+1]
  std::vector<int32_t> eslot;      // [E][2] (two-node elements)
  std::vector<int32_t> bc_ptr;
  std::vector<BcTerm> bc;
  std::vector<ScaleFn> scales;
  // element arrays (internal numbering)
  int nen = 2;                      // nodes per element (2, 3 or 4)
  std::vector<int32_t> conn;        // [E][nen], nodes along the line
  std::vector<double> invL0;        // [E] 1 / chord length (end to end)
  std::vector<double> qN;           // [nen][E][4] element-node frames Lambda_N
  // elements of 3 or 4 nodes: component-major node and slot lists [nen][E],
  // per Gauss point the weight and shape gradients [E][G][nen + 1], and the
  // shape values at the Gauss points Nq[a][g]
  std::vector<int32_t> conn_n, eslot_n;
  std::vector<double> shp;
  double Nq[4][4] = {};
  std::vector<double> g0, k0;       // [G*3][E]
  std::vector<double> C;            // [6][E]
  std::vector<double> ec;           // [2][E]
  std::vector<double> strut_param;  // unused here
  // section data for derivatives with respect to the radius: density,
  // rotational-inertia factor, 1 for circular sections (internal numbering)
  std::vector<double> erho, eic;
  std::vector<uint8_t> ecircle;
  // plasticity
  ExprProgram yield, grad;
  ExprPtr yield_expr;
  std::vector<ExprPtr> grad_exprs;
  std::string yield_key;            // source text of yieldCond + yieldDeriv (batch compatibility)
  // batches of independent lattices (build_batch): per-node time step and
  // lattice index, per-element lattice index, node/element offsets
  int n_lat = 1;
  std::vector<double> dtn;          // [N] (empty for a single lattice)
  std::vector<int32_t> nlat, elat;  // [N], [E]
  std::vector<int32_t> lat_node_off, lat_elem_off;  // [n_lat + 1]
  double H[7][7] = {};
  int max_iter = 20;
  double prec = 1e-5;
  // neumann / dirichlet node lists per BC (internal numbering) for group sums
  dl_contact_desc contact{};
  std::vector<int32_t> elem_rod;    // internal element order
  // joint contact: the descriptor (its joints pointer is the caller's and
  // not kept past build_lattice) and the joints in list order (internal numbering)
  dl_joint_contact_desc jcontact{};
  std::vector<int32_t> joints;
  // added point masses (MassModel): [6][N] diagonal (internal numbering), empty if none
  std::vector<double> madd;
};

// Builds the lattice; `round_frames_to_float` rounds the element-end frames to
// FP32 (mixed precision) before the reference strains are formed from them.
// Throws std::runtime_error / std::invalid_argument with a message.
std::unique_ptr<HostLattice> build_lattice(const dl_model_desc &d, bool round_frames_to_float);

// Disjoint union of n independent lattices (one engine, one launch): each
// lattice keeps its own Morton order inside its block of nodes/elements, its
// own time step (per node) and BCs.  All lattices must share the Gauss rule,
// the rotation-update options and (when elastoplastic) the yield function.
std::unique_ptr<HostLattice> build_batch(const dl_model_desc *descs, int n, bool round_frames_to_float);

// Rotation matrix (row-major) to unit quaternion with w >= 0.
void mat_to_quat(const double R[3][3], double q[4]);

}  // namespace dl
