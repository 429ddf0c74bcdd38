// Host set-up of a lattice (see setup.hpp).
#include "setup.hpp"

#include <algorithm>
#include <array>
#include <cfloat>
#include <cmath>
#include <cstring>
#include <numeric>
#include <stdexcept>
#include <string>

#include "contact_build.hpp"
#include "rodkin.cuh"

namespace dl {

namespace {

using M3 = std::array<std::array<double, 3>, 3>;

M3 skew(const double v[3]) {
  M3 r{};
  r[0][1] = -v[2];
  r[0][2] = v[1];
  r[1][0] = v[2];
  r[1][2] = -v[0];
  r[2][0] = -v[1];
  r[2][1] = v[0];
  return r;
}
M3 mul(const M3 &a, const M3 &b) {
  M3 r{};
  for (int i = 0; i < 3; ++i)
    for (int j = 0; j < 3; ++j)
      for (int k = 0; k < 3; ++k) r[i][j] += a[i][k] * b[k][j];
  return r;
}

uint64_t spread3(uint64_t v) {  // 21 bits -> every third bit
  v &= 0x1fffffULL;
  v = (v | v << 32) & 0x1f00000000ffffULL;
  v = (v | v << 16) & 0x1f0000ff0000ffULL;
  v = (v | v << 8) & 0x100f00f00f00f00fULL;
  v = (v | v << 4) & 0x10c30c30c30c30c3ULL;
  v = (v | v << 2) & 0x1249249249249249ULL;
  return v;
}

std::vector<uint64_t> morton_codes(const std::vector<double> &pts, int n) {
  double lo[3] = {1e300, 1e300, 1e300}, hi[3] = {-1e300, -1e300, -1e300};
  for (int i = 0; i < n; ++i)
    for (int k = 0; k < 3; ++k) {
      lo[k] = std::min(lo[k], pts[i * 3 + k]);
      hi[k] = std::max(hi[k], pts[i * 3 + k]);
    }
  double ext = 0.0;
  for (int k = 0; k < 3; ++k) ext = std::max(ext, hi[k] - lo[k]);
  if (ext <= 0.0) ext = 1.0;
  std::vector<uint64_t> c(n);
  for (int i = 0; i < n; ++i) {
    uint64_t q[3];
    for (int k = 0; k < 3; ++k) {
      double t = (pts[i * 3 + k] - lo[k]) / ext;
      q[k] = static_cast<uint64_t>(std::min(2097151.0, std::max(0.0, t * 2097151.0)));
    }
    c[i] = spread3(q[0]) | (spread3(q[1]) << 1) | (spread3(q[2]) << 2);
  }
  return c;
}

// symmetric 3x3 eigen-decomposition (cyclic Jacobi): A = V diag(w) V^T
void jacobi3(double A[3][3], double V[3][3], double w[3]) {
  for (int i = 0; i < 3; ++i)
    for (int j = 0; j < 3; ++j) V[i][j] = (i == j) ? 1.0 : 0.0;
  for (int sweep = 0; sweep < 50; ++sweep) {
    double off = std::fabs(A[0][1]) + std::fabs(A[0][2]) + std::fabs(A[1][2]);
    double diag = std::fabs(A[0][0]) + std::fabs(A[1][1]) + std::fabs(A[2][2]);
    if (off <= 1e-300 || off < 1e-17 * diag) break;
    for (int p = 0; p < 2; ++p)
      for (int q = p + 1; q < 3; ++q) {
        if (std::fabs(A[p][q]) < 1e-300) continue;
        const double theta = (A[q][q] - A[p][p]) / (2.0 * A[p][q]);
        const double t = (theta >= 0 ? 1.0 : -1.0) / (std::fabs(theta) + std::sqrt(theta * theta + 1.0));
        const double c = 1.0 / std::sqrt(t * t + 1.0), s = t * c;
        for (int k = 0; k < 3; ++k) {  // A <- J^T A J
          const double akp = A[k][p], akq = A[k][q];
          A[k][p] = c * akp - s * akq;
          A[k][q] = s * akp + c * akq;
        }
        for (int k = 0; k < 3; ++k) {
          const double apk = A[p][k], aqk = A[q][k];
          A[p][k] = c * apk - s * aqk;
          A[q][k] = s * apk + c * aqk;
        }
        for (int k = 0; k < 3; ++k) {
          const double vkp = V[k][p], vkq = V[k][q];
          V[k][p] = c * vkp - s * vkq;
          V[k][q] = s * vkp + c * vkq;
        }
      }
  }
  for (int i = 0; i < 3; ++i) w[i] = A[i][i];
  // proper rotation
  const double det = V[0][0] * (V[1][1] * V[2][2] - V[1][2] * V[2][1]) -
                     V[0][1] * (V[1][0] * V[2][2] - V[1][2] * V[2][0]) +
                     V[0][2] * (V[1][0] * V[2][1] - V[1][1] * V[2][0]);
  if (det < 0)
    for (int k = 0; k < 3; ++k) V[k][2] = -V[k][2];
}


// Line3D shape functions of an n-node line (nodes at xi = -1 + 2a/(n-1), in
// order along the line) at the points of the Gauss rule of G points (Line3D.cpp:
// 57-115): values N[a][q], derivatives dN[a][q] = dN_a/dxi, weights W[q].
struct LineRule {
  int n = 2, G = 1;
  double xi[4] = {}, W[4] = {}, N[4][4] = {}, dN[4][4] = {};
};
LineRule line_rule(int n, int G) {
  LineRule r;
  r.n = n;
  r.G = G;
  switch (G) {
    case 1: r.xi[0] = 0.0; r.W[0] = 2.0; break;
    case 2: r.xi[0] = -1.0 / std::sqrt(3.0); r.xi[1] = -r.xi[0]; r.W[0] = r.W[1] = 1.0; break;
    case 3:
      r.xi[0] = -std::sqrt(0.6); r.xi[1] = 0.0; r.xi[2] = std::sqrt(0.6);
      r.W[0] = r.W[2] = 5.0 / 9.0; r.W[1] = 8.0 / 9.0;
      break;
    case 4: {
      const double p = std::sqrt(3.0 / 7.0 - 2.0 / 7.0 * std::sqrt(1.2));
      const double q = std::sqrt(3.0 / 7.0 + 2.0 / 7.0 * std::sqrt(1.2));
      r.xi[0] = -q; r.xi[1] = -p; r.xi[2] = p; r.xi[3] = q;
      r.W[1] = r.W[2] = (18.0 + std::sqrt(30.0)) / 36.0;
      r.W[0] = r.W[3] = (18.0 - std::sqrt(30.0)) / 36.0;
      break;
    }
    default: throw std::invalid_argument("Gauss rules of 1 to 4 points only");
  }
  double xn[4];
  for (int a = 0; a < n; ++a) xn[a] = -1.0 + 2.0 * a / (n - 1);
  for (int q = 0; q < G; ++q)
    for (int a = 0; a < n; ++a) {
      double l = 1.0, dl = 0.0;
      for (int b = 0; b < n; ++b)
        if (b != a) l *= (r.xi[q] - xn[b]) / (xn[a] - xn[b]);
      for (int k = 0; k < n; ++k) {  // product rule over the factors of l
        if (k == a) continue;
        double t = 1.0 / (xn[a] - xn[k]);
        for (int b = 0; b < n; ++b)
          if (b != a && b != k) t *= (r.xi[q] - xn[b]) / (xn[a] - xn[b]);
        dl += t;
      }
      r.N[a][q] = l;
      r.dN[a][q] = dl;
    }
  return r;
}

// Integration weights and shape gradients of one element (Line3D::
// getIntegrationWeights/getShapeGradients, Line3D.cpp:91-115): the 1-D
// coordinates are the accumulated chord lengths of the reference nodes.
void line_weights(const LineRule &r, const double *X0, const int *nodes, double *w, double (*g)[4]) {
  double c1[4];
  c1[0] = 0.0;
  for (int a = 1; a < r.n; ++a) {
    double d2 = 0.0;
    for (int k = 0; k < 3; ++k) {
      const double d = X0[nodes[a] * 3 + k] - X0[nodes[a - 1] * 3 + k];
      d2 += d * d;
    }
    c1[a] = c1[a - 1] + std::sqrt(d2);
  }
  for (int q = 0; q < r.G; ++q) {
    double J = 0.0;
    for (int a = 0; a < r.n; ++a) J += r.dN[a][q] * c1[a];
    if (!(std::fabs(J) > 0.0)) throw std::invalid_argument("degenerate element (zero Jacobian)");
    w[q] = r.W[q] * std::fabs(J);
    if (g)
      for (int a = 0; a < r.n; ++a) g[a][q] = r.dN[a][q] / J;
  }
}

}  // namespace

void mat_to_quat(const double R[3][3], double q[4]) {
  const double tr = R[0][0] + R[1][1] + R[2][2];
  if (tr > 0.0) {
    const double s = std::sqrt(tr + 1.0) * 2.0;
    q[0] = 0.25 * s;
    q[1] = (R[2][1] - R[1][2]) / s;
    q[2] = (R[0][2] - R[2][0]) / s;
    q[3] = (R[1][0] - R[0][1]) / s;
  } else if (R[0][0] > R[1][1] && R[0][0] > R[2][2]) {
    const double s = std::sqrt(1.0 + R[0][0] - R[1][1] - R[2][2]) * 2.0;
    q[0] = (R[2][1] - R[1][2]) / s;
    q[1] = 0.25 * s;
    q[2] = (R[0][1] + R[1][0]) / s;
    q[3] = (R[0][2] + R[2][0]) / s;
  } else if (R[1][1] > R[2][2]) {
    const double s = std::sqrt(1.0 + R[1][1] - R[0][0] - R[2][2]) * 2.0;
    q[0] = (R[0][2] - R[2][0]) / s;
    q[1] = (R[0][1] + R[1][0]) / s;
    q[2] = 0.25 * s;
    q[3] = (R[1][2] + R[2][1]) / s;
  } else {
    const double s = std::sqrt(1.0 + R[2][2] - R[0][0] - R[1][1]) * 2.0;
    q[0] = (R[1][0] - R[0][1]) / s;
    q[1] = (R[0][2] + R[2][0]) / s;
    q[2] = (R[1][2] + R[2][1]) / s;
    q[3] = 0.25 * s;
  }
  if (q[0] < 0)
    for (int k = 0; k < 4; ++k) q[k] = -q[k];
  const double n = std::sqrt(q[0] * q[0] + q[1] * q[1] + q[2] * q[2] + q[3] * q[3]);
  for (int k = 0; k < 4; ++k) q[k] /= n;
}

std::unique_ptr<HostLattice> build_lattice(const dl_model_desc &d, bool round_frames_to_float) {
  auto L = std::make_unique<HostLattice>();
  HostLattice &h = *L;
  if (d.nodes_per_elem < 2 || d.nodes_per_elem > 4)
    throw std::invalid_argument("elements have 2, 3 or 4 nodes");
  const int nen = d.nodes_per_elem;
  h.nen = nen;
  h.N = d.n_nodes;
  h.E = d.n_elems;
  h.G = d.n_gauss > 0 ? d.n_gauss : nen - 1;  // Gauss(n-1) default, Line3D.cpp:72-73
  if (h.G < 1 || h.G > 3) throw std::invalid_argument("n_gauss must be 1, 2 or 3");
  if (h.N <= 0 || h.E <= 0) throw std::invalid_argument("empty model");
  if (!d.coords || !d.conn) throw std::invalid_argument("coords/conn missing");
  if (d.n_materials <= 0 || !d.materials) throw std::invalid_argument("no material");
  if (!(d.dt > 0.0)) throw std::invalid_argument("deltaTime must be positive");
  const int N = h.N, E = h.E, G = h.G;
  h.dt = d.dt;
  h.so3 = d.so3_update != 0;
  if (d.mass_mode != DL_MASS_CONSISTENT && d.mass_mode != DL_MASS_LUMPED)
    throw std::invalid_argument("mass_mode must be DL_MASS_CONSISTENT or DL_MASS_LUMPED");
  h.lumped = d.mass_mode == DL_MASS_LUMPED;
  // the rod model adds the gyroscopic moment only with the consistent matrix
  // (SpecialCosseratRodModel.cpp:351-355)
  h.gyro = d.gyroscopic != 0 && !h.lumped;
  h.contact = d.contact;
  h.jcontact = d.joint_contact;
  if (nen > 2 && (h.contact.enabled || h.jcontact.enabled))
    throw UnsupportedError("contact runs on two-node elements (segments between element end nodes)");
  if (h.jcontact.enabled) {
    if (!(h.jcontact.radius > 0.0)) throw std::invalid_argument("joint contact radius must be positive");
    if (h.jcontact.n_joints < 0 || (h.jcontact.n_joints > 0 && !h.jcontact.joints))
      throw std::invalid_argument("joint list missing");
    for (int j = 0; j < h.jcontact.n_joints; ++j)
      if (h.jcontact.joints[j] < 0 || h.jcontact.joints[j] >= N)
        throw std::invalid_argument("joint node index out of range");
  }
  h.X0.assign(d.coords, d.coords + static_cast<size_t>(N) * 3);
  for (size_t i = 0; i < static_cast<size_t>(nen) * E; ++i)
    if (d.conn[i] < 0 || d.conn[i] >= N) throw std::invalid_argument("connectivity index out of range");
  for (int e = 0; e < E; ++e)
    for (int a = 0; a < nen; ++a)
      for (int b = a + 1; b < nen; ++b)
        if (d.conn[nen * e + a] == d.conn[nen * e + b]) throw std::invalid_argument("element with repeated node");

  // ---- materials: one law for all plastic materials (same expression set)
  const dl_material_desc *plast = nullptr;
  for (int mi = 0; mi < d.n_materials; ++mi)
    if (d.materials[mi].type == DL_MAT_ELASTOPLASTIC_ROD) {
      if (plast && std::string(plast->yield_cond ? plast->yield_cond : "") !=
                       std::string(d.materials[mi].yield_cond ? d.materials[mi].yield_cond : ""))
        throw std::invalid_argument("all elastoplastic materials of one lattice must share yieldCond");
      plast = &d.materials[mi];
    }
  for (int e = 0; e < E; ++e) {
    const int mi = d.elem_mat ? d.elem_mat[e] : 0;
    if (mi < 0 || mi >= d.n_materials) throw std::invalid_argument("material index out of range");
    if (plast && d.materials[mi].type != DL_MAT_ELASTOPLASTIC_ROD)
      throw std::invalid_argument("mixing elastic and elastoplastic materials in one lattice is not supported");
  }
  h.plastic = plast != nullptr;
  std::vector<std::string> dofn = {"dx", "dy", "dz", "rx", "ry", "rz"};
  if (d.dof_names)
    for (int k = 0; k < 6; ++k) dofn[k] = d.dof_names[k];
  if (h.plastic) {
    const dl_material_desc &md = *plast;
    std::vector<std::string> names(dofn);
    int nh = 0;
    if (md.has_isotropic) {
      names.push_back("h_0");
      ++nh;
    }
    if (md.kinematic_tensor) {
      for (int k = 0; k < 6; ++k) names.push_back("h_" + dofn[k]);
      nh += 6;
    }
    names.push_back("radius");
    names.push_back("area");
    h.nh = nh;
    std::memset(h.H, 0, sizeof h.H);
    if (nh == 1 || nh == 7) h.H[0][0] = md.isotropic_coefficient;
    const int off = (nh == 7) ? 1 : 0;
    if (md.kinematic_tensor)
      for (int i = 0; i < 6; ++i)
        for (int j = 0; j < 6; ++j) h.H[off + j][off + i] = md.kinematic_tensor[i * 6 + j];
    if (!md.yield_cond) throw std::invalid_argument("elastoplastic material needs yieldCond");
    ExprPtr f = parseExpr(md.yield_cond, names);
    h.yield = compileExprs({f});
    h.yield_expr = f;
    if (!md.yield_deriv || md.n_yield_deriv <= 0)
      throw std::invalid_argument("the engine needs yieldDeriv (one derivative per argument)");
    if (md.n_yield_deriv != 6 + nh) throw std::invalid_argument("yieldDeriv needs one entry per argument");
    std::vector<ExprPtr> gs;
    for (int k = 0; k < md.n_yield_deriv; ++k) gs.push_back(parseExpr(md.yield_deriv[k], names));
    h.grad = compileExprs(gs);
    h.grad_exprs = gs;
    h.yield_key = std::string(md.yield_cond);
    for (int k = 0; k < md.n_yield_deriv; ++k) h.yield_key += std::string("|") + md.yield_deriv[k];
    h.max_iter = md.max_iter > 0 ? md.max_iter : 20;
    h.prec = md.precision > 0 ? md.precision : 1e-5;
  }

  // ---- renumbering along a Morton curve
  {
    std::vector<uint64_t> nc = morton_codes(h.X0, N);
    h.node_old.resize(N);
    std::iota(h.node_old.begin(), h.node_old.end(), 0);
    std::stable_sort(h.node_old.begin(), h.node_old.end(), [&](int a, int b) { return nc[a] < nc[b]; });
    h.node_new.resize(N);
    for (int i = 0; i < N; ++i) h.node_new[h.node_old[i]] = i;
    // joints of the joint contact, in list order (internal numbering)
    if (h.jcontact.enabled)
      for (int j = 0; j < h.jcontact.n_joints; ++j) h.joints.push_back(h.node_new[d.joint_contact.joints[j]]);
    h.jcontact.joints = nullptr;
    std::vector<double> mid(static_cast<size_t>(E) * 3);
    for (int e = 0; e < E; ++e)
      for (int k = 0; k < 3; ++k)
        mid[e * 3 + k] = 0.5 * (h.X0[d.conn[nen * e] * 3 + k] + h.X0[d.conn[nen * e + nen - 1] * 3 + k]);
    std::vector<uint64_t> ecd = morton_codes(mid, E);
    h.elem_old.resize(E);
    std::iota(h.elem_old.begin(), h.elem_old.end(), 0);
    std::stable_sort(h.elem_old.begin(), h.elem_old.end(), [&](int a, int b) { return ecd[a] < ecd[b]; });
    h.elem_new.resize(E);
    for (int i = 0; i < E; ++i) h.elem_new[h.elem_old[i]] = i;
  }

  // ---- SpecialCosseratRodModel::initRotation_ (SpecialCosseratRodModel.cpp:574-658), per rod
  // element-end frames in the ORIGINAL element numbering first
  std::vector<double> frames(static_cast<size_t>(E) * nen * 4);
  {
    const int R = d.n_rods > 0 ? d.n_rods : 1;
    std::vector<std::vector<int>> rodElems(R);
    for (int e = 0; e < E; ++e) {
      const int r = d.elem_rod ? d.elem_rod[e] : 0;
      if (r < 0 || r >= R) throw std::invalid_argument("rod index out of range");
      rodElems[r].push_back(e);
    }
    std::vector<double> dirs(static_cast<size_t>(N) * 3, 0.0);
    std::vector<int> stamp(N, -1);
    for (int r = 0; r < R; ++r) {
      auto &els = rodElems[r];
      for (int e : els)
        for (int a = 0; a < nen; ++a) {
          const int nd = d.conn[nen * e + a];
          if (stamp[nd] != r) {
            stamp[nd] = r;
            dirs[nd * 3] = dirs[nd * 3 + 1] = dirs[nd * 3 + 2] = 0.0;
          }
        }
      // node tangents: the chord to the next node at the first node, to the
      // previous one at the last, the chord between the neighbours in between
      for (int e : els) {
        const int *c = d.conn + static_cast<size_t>(nen) * e;
        for (int a = 0; a < nen; ++a) {
          const int lo = a == 0 ? 0 : a - 1, hi = a == nen - 1 ? nen - 1 : a + 1;
          for (int k = 0; k < 3; ++k) dirs[c[a] * 3 + k] += h.X0[c[hi] * 3 + k] - h.X0[c[lo] * 3 + k];
        }
      }
      for (int gdi = 0; gdi < d.n_given_dirs; ++gdi) {
        const int nd = d.given_dir_nodes[gdi];
        if (nd >= 0 && nd < N && stamp[nd] == r)
          for (int k = 0; k < 3; ++k) dirs[nd * 3 + k] = d.given_dirs[gdi * 3 + k];
      }
      for (int e : els)
        for (int a = 0; a < nen; ++a) {
          const int nd = d.conn[nen * e + a];
          double t[3] = {dirs[nd * 3], dirs[nd * 3 + 1], dirs[nd * 3 + 2]};
          const double nn = std::sqrt(t[0] * t[0] + t[1] * t[1] + t[2] * t[2]);
          if (!(nn > 0.0)) throw std::invalid_argument("zero-length rod tangent");
          for (int k = 0; k < 3; ++k) t[k] /= nn;
          double Rm[3][3];
          if (d.has_material_ey) {
            const double *ey = d.material_ey;
            const double ex[3] = {ey[1] * t[2] - ey[2] * t[1], ey[2] * t[0] - ey[0] * t[2], ey[0] * t[1] - ey[1] * t[0]};
            for (int k = 0; k < 3; ++k) {
              Rm[k][0] = ex[k];
              Rm[k][1] = ey[k];
              Rm[k][2] = t[k];
            }
          } else {
            const double v[3] = {-t[1], t[0], 0.0};  // e3 x t
            const double c = t[2];
            if (std::fabs(c + 1.0) > DBL_EPSILON) {
              M3 S = skew(v), S2 = mul(S, S);
              for (int i = 0; i < 3; ++i)
                for (int j = 0; j < 3; ++j) Rm[i][j] = (i == j ? 1.0 : 0.0) + S[i][j] + S2[i][j] / (1.0 + c);
            } else {
              // tangent exactly -e3: the reference uses -I (an improper matrix);
              // the engine uses the proper rotation by pi about e1.
              const double P[3][3] = {{1, 0, 0}, {0, -1, 0}, {0, 0, -1}};
              std::memcpy(Rm, P, sizeof P);
            }
          }
          double q[4];
          mat_to_quat(Rm, q);
          if (round_frames_to_float) {
            for (int k = 0; k < 4; ++k) q[k] = static_cast<double>(static_cast<float>(q[k]));
            const double n2 = std::sqrt(q[0] * q[0] + q[1] * q[1] + q[2] * q[2] + q[3] * q[3]);
            for (int k = 0; k < 4; ++k) q[k] = static_cast<double>(static_cast<float>(q[k] / n2));
          }
          std::memcpy(&frames[(static_cast<size_t>(e) * nen + a) * 4], q, sizeof q);
        }
    }
  }

  // ---- element arrays in internal numbering
  const double gxi[3][3] = {{0.0, 0.0, 0.0},
                            {-0.57735026918962576451, 0.57735026918962576451, 0.0},
                            {-0.77459666924148337704, 0.0, 0.77459666924148337704}};
  h.conn.resize(static_cast<size_t>(E) * nen);
  h.invL0.resize(E);
  h.qN.resize(static_cast<size_t>(nen) * E * 4);
  h.g0.assign(static_cast<size_t>(G) * 3 * E, 0.0);
  h.k0.assign(static_cast<size_t>(G) * 3 * E, 0.0);
  h.C.resize(static_cast<size_t>(6) * E);
  h.ec.resize(static_cast<size_t>(2) * E);
  h.elem_rod.resize(E);
  h.erho.resize(E);
  h.eic.resize(E);
  h.ecircle.resize(E);
  // stiffness rule (Gauss G) and mass rule (Gauss nen, the massShape of
  // SpecialCosseratRodModel.cpp:105-109) of the element's shape
  const LineRule kr = line_rule(nen, G), mr = line_rule(nen, nen);
  if (nen > 2) {
    h.conn_n.resize(static_cast<size_t>(nen) * E);
    h.shp.resize(static_cast<size_t>(E) * G * (nen + 1));
    for (int a = 0; a < nen; ++a)
      for (int g = 0; g < G; ++g) h.Nq[a][g] = kr.N[a][g];
  }
  std::vector<double> mnode(N, 0.0);
  std::vector<double> Snode(static_cast<size_t>(N) * 9, 0.0);
  for (int ei = 0; ei < E; ++ei) {
    const int e = h.elem_old[ei];
    const int *ce = d.conn + static_cast<size_t>(nen) * e;
    for (int a = 0; a < nen; ++a) h.conn[static_cast<size_t>(nen) * ei + a] = h.node_new[ce[a]];
    h.elem_rod[ei] = d.elem_rod ? d.elem_rod[e] : 0;
    for (int s = 0; s < nen; ++s)
      for (int k = 0; k < 4; ++k)
        h.qN[(static_cast<size_t>(s) * E + ei) * 4 + k] = frames[(static_cast<size_t>(e) * nen + s) * 4 + k];
    // section (ElasticRodMaterial.cpp:114-185, 265-287) with the per-element radius extension
    const int mi = d.elem_mat ? d.elem_mat[e] : 0;
    const dl_material_desc &md = d.materials[mi];
    double A = md.area, I1 = md.area_moment[0], I2 = md.area_moment[1], J = md.polar_moment, r = md.radius;
    if (d.elem_radius) {
      if (!md.circle) throw std::invalid_argument("per-element radius needs a circular section");
      r = d.elem_radius[e];
      A = M_PI * r * r;
      I1 = I2 = M_PI * std::pow(r, 4) / 4.0;
      J = I1 + I2;
    }
    const double Gm = md.shear_modulus, ks = md.shear_correction, Ey = md.young;
    const double Cd[6] = {Gm * ks * A, Gm * ks * A, Ey * A, Ey * I1, Ey * I2, Gm * J};
    for (int k = 0; k < 6; ++k) h.C[static_cast<size_t>(k) * E + ei] = Cd[k];
    h.ec[ei] = r;
    h.ec[E + ei] = A;
    const double ic = md.inertia_correct > 0 ? md.inertia_correct : 1.0;
    const double rho = md.density;
    h.erho[ei] = rho;
    h.eic[ei] = ic;
    h.ecircle[ei] = md.circle ? 1 : 0;
    // rotational node block Lambda_N D Lambda_N^T, D = diag(rho I1 ic l + rho A l^3/12,
    // rho I2 ic l + rho A l^3/12, rho J ic l) (ElasticRodMaterial::getLumpedMass,
    // ElasticRodMaterial.cpp:289-297), half of it at the element's end nodes
    auto add_rot_block = [&](int nd, const double *q, double l, double f) {
      const double Dg[3] = {rho * I1 * ic * l + rho * A * l * l * l / 12.0, rho * I2 * ic * l + rho * A * l * l * l / 12.0,
                            rho * J * ic * l};
      double Rm[3][3];
      qmat(Q4<double>{q[0], q[1], q[2], q[3]}, Rm);
      for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j) {
          double acc = 0.0;
          for (int k = 0; k < 3; ++k) acc += Rm[i][k] * Dg[k] * Rm[j][k];
          Snode[static_cast<size_t>(nd) * 9 + i * 3 + j] += f * acc;
        }
    };
    if (nen == 2) {
      const int a = ce[0], b = ce[1];
      double c[3];
      for (int k = 0; k < 3; ++k) c[k] = h.X0[b * 3 + k] - h.X0[a * 3 + k];
      const double L0 = std::sqrt(c[0] * c[0] + c[1] * c[1] + c[2] * c[2]);
      if (!(L0 > 0.0)) throw std::invalid_argument("zero-length element");
      h.invL0[ei] = 1.0 / L0;
      // initStrain_: strains of the undeformed element with the same closed form the kernel uses
      const double *fi = &frames[(static_cast<size_t>(e) * 2) * 4], *fj = &frames[(static_cast<size_t>(e) * 2 + 1) * 4];
      Q4<double> qi{fi[0], fi[1], fi[2], fi[3]};
      Q4<double> qj{fj[0], fj[1], fj[2], fj[3]};
      const Q4<double> I{1.0, 0.0, 0.0, 0.0};
      V3<double> xa{h.X0[a * 3], h.X0[a * 3 + 1], h.X0[a * 3 + 2]};
      V3<double> xb{h.X0[b * 3], h.X0[b * 3 + 1], h.X0[b * 3 + 2]};
      ElemKin<double> kin = elem_kin<double>(xa, xb, I, I, qi, qj, 1.0 / L0);
      for (int g = 0; g < G; ++g) {
        const double zero[3] = {0, 0, 0};
        double eps[6];
        Q4<double> qg;
        gp_strain(kin, gxi[G - 1][g], 1.0 / L0, zero, zero, eps, &qg);
        for (int k = 0; k < 3; ++k) {
          h.g0[(static_cast<size_t>(g) * 3 + k) * E + ei] = eps[k];
          h.k0[(static_cast<size_t>(g) * 3 + k) * E + ei] = eps[3 + k];
        }
      }
      // SpecialCosseratRodModel::assembleM_ for a 2-node element (Gauss2 mass
      // shape): translational rho A L/2 per end; rotational half blocks
      mnode[a] += rho * A * L0 / 2.0;
      add_rot_block(a, fi, L0, 0.5);
      mnode[b] += rho * A * L0 / 2.0;
      add_rot_block(b, fj, L0, 0.5);
    } else {
      for (int a = 0; a < nen; ++a) h.conn_n[static_cast<size_t>(a) * E + ei] = h.node_new[ce[a]];
      double w[4], g[4][4], wm[4];
      line_weights(kr, h.X0.data(), ce, w, g);
      line_weights(mr, h.X0.data(), ce, wm, nullptr);
      double chord = 0.0;
      for (int q = 0; q < nen; ++q) chord += wm[q];  // the line's length (the sum of the mass weights)
      h.invL0[ei] = 1.0 / chord;
      for (int q = 0; q < G; ++q) {
        double *sh = &h.shp[(static_cast<size_t>(ei) * G + q) * (nen + 1)];
        sh[0] = w[q];
        for (int a = 0; a < nen; ++a) sh[1 + a] = g[a][q];
      }
      // initStrain_ (SpecialCosseratRodModel.cpp:536-569): the strains of the
      // undeformed element, with the kernel's own kinematics
      V3<double> x[4];
      Q4<double> Lf[4];
      for (int a = 0; a < nen; ++a) {
        x[a] = V3<double>{h.X0[ce[a] * 3], h.X0[ce[a] * 3 + 1], h.X0[ce[a] * 3 + 2]};
        const double *f = &frames[(static_cast<size_t>(e) * nen + a) * 4];
        Lf[a] = Q4<double>{f[0], f[1], f[2], f[3]};
      }
      Q4<double> Lr;
      V3<double> psi[4];
      line_ref(Lf, nen, Lr, psi);
      for (int q = 0; q < G; ++q) {
        double Nn[4], dN[4];
        for (int a = 0; a < nen; ++a) {
          Nn[a] = kr.N[a][q];
          dN[a] = g[a][q];
        }
        const GpKinN k = gp_kin_n(x, Lr, psi, nen, Nn, dN);
        const double s0[6] = {k.gme3.x, k.gme3.y, k.gme3.z, k.K.x, k.K.y, k.K.z};
        for (int c = 0; c < 3; ++c) {
          h.g0[(static_cast<size_t>(q) * 3 + c) * E + ei] = s0[c];
          h.k0[(static_cast<size_t>(q) * 3 + c) * E + ei] = s0[3 + c];
        }
      }
      // SpecialCosseratRodModel::assembleM_ (SpecialCosseratRodModel.cpp:969-1031):
      // translational rho A sum_b int N_a N_b, rotational blocks with l = length / (n - 1)
      const double l = chord / (nen - 1);
      for (int a = 0; a < nen; ++a) {
        double sm = 0.0;
        for (int b = 0; b < nen; ++b)
          for (int q = 0; q < nen; ++q) sm += wm[q] * mr.N[a][q] * mr.N[b][q];
        mnode[ce[a]] += sm * rho * A;
        add_rot_block(ce[a], &frames[(static_cast<size_t>(e) * nen + a) * 4], l, (a == 0 || a == nen - 1) ? 0.5 : 1.0);
      }
    }
  }

  // ---- rigid ties (HingeModel constraints, condensed): every member of a
  // group carries the group's summed translational mass and rotational
  // inertia (the members share their rotation, so the node-frame inertias add)
  std::vector<int> master_of(N, -1);
  std::vector<std::vector<int>> slaves(N);
  if (d.n_ties > 0) {
    if (!d.ties) throw std::invalid_argument("tie list missing");
    if (h.lumped) throw UnsupportedError("rigid ties need the consistent mass (the lumped mode is not provided)");
    for (int k = 0; k < d.n_ties; ++k) {
      const int a = d.ties[2 * k], b = d.ties[2 * k + 1];
      if (a < 0 || a >= N || b < 0 || b >= N || a == b) throw std::invalid_argument("tie node out of range");
      if (master_of[b] >= 0) throw std::invalid_argument("a node is the slave of two ties");
      master_of[b] = a;
      slaves[a].push_back(b);
    }
    for (int n = 0; n < N; ++n)
      if (master_of[n] >= 0 && !slaves[n].empty()) throw std::invalid_argument("a tie's slave is another tie's master");
    for (int n = 0; n < N; ++n) {
      if (slaves[n].empty()) continue;
      std::sort(slaves[n].begin(), slaves[n].end());
      for (int sl : slaves[n]) {
        for (int k = 0; k < 3; ++k)
          if (std::fabs(h.X0[3 * sl + k] - h.X0[3 * n + k]) > 1e-12 * (1.0 + std::fabs(h.X0[3 * n + k])))
            throw std::invalid_argument("tied nodes must coincide");
        mnode[n] += mnode[sl];
        for (int k = 0; k < 9; ++k) Snode[static_cast<size_t>(n) * 9 + k] += Snode[static_cast<size_t>(sl) * 9 + k];
      }
      for (int sl : slaves[n]) {
        mnode[sl] = mnode[n];
        for (int k = 0; k < 9; ++k) Snode[static_cast<size_t>(sl) * 9 + k] = Snode[static_cast<size_t>(n) * 9 + k];
      }
    }
    h.ties = true;
  }

  // ---- node arrays in internal numbering
  h.pos.assign(static_cast<size_t>(N) * 4, 0.0);
  h.rot.assign(static_cast<size_t>(N) * 4, 0.0);
  h.vel.assign(static_cast<size_t>(N) * 6, 0.0);
  h.mass.resize(N);
  h.iframe.resize(static_cast<size_t>(N) * 4);
  h.idiag.resize(static_cast<size_t>(N) * 4);
  for (int ni = 0; ni < N; ++ni) {
    const int n = h.node_old[ni];
    for (int k = 0; k < 3; ++k) h.pos[ni * 4 + k] = h.X0[n * 3 + k];
    h.rot[ni * 4] = 1.0;
    if (!(mnode[n] > DBL_MIN))
      throw MassError("Zero (or negative) masses cannot be inversed! (node without mass)");
    h.mass[ni] = mnode[n];
    double A[3][3], V[3][3], w[3];
    for (int i = 0; i < 3; ++i)
      for (int j = 0; j < 3; ++j) A[i][j] = Snode[static_cast<size_t>(n) * 9 + i * 3 + j];
    jacobi3(A, V, w);
    for (int k = 0; k < 3; ++k)
      if (!(w[k] > 0.0)) throw std::invalid_argument("rotational inertia is not positive definite");
    double q[4];
    mat_to_quat(V, q);
    for (int k = 0; k < 4; ++k) h.iframe[ni * 4 + k] = q[k];
    for (int k = 0; k < 3; ++k) h.idiag[ni * 4 + k] = w[k];
    h.idiag[ni * 4 + 3] = 0.0;
  }
  // end-force slots: node-ordered CSR, element order within a node
  h.slot_ptr.assign(N + 1, 0);
  for (size_t i = 0; i < h.conn.size(); ++i) h.slot_ptr[h.conn[i] + 1]++;
  for (int i = 0; i < N; ++i) h.slot_ptr[i + 1] += h.slot_ptr[i];
  {
    std::vector<int32_t> fill(h.slot_ptr.begin(), h.slot_ptr.end() - 1);
    if (nen == 2) {
      h.eslot.resize(static_cast<size_t>(2) * E);
      for (int ei = 0; ei < E; ++ei)
        for (int s = 0; s < 2; ++s) h.eslot[2 * ei + s] = fill[h.conn[2 * ei + s]]++;
    } else {
      h.eslot_n.resize(static_cast<size_t>(nen) * E);
      for (int ei = 0; ei < E; ++ei)
        for (int s = 0; s < nen; ++s)
          h.eslot_n[static_cast<size_t>(s) * E + ei] = fill[h.conn[static_cast<size_t>(nen) * ei + s]]++;
    }
  }

  // ---- boundary conditions (Dirichlet on accelerations, Neumann loads, InitLoad)
  std::vector<std::vector<BcTerm>> perNode(N);
  std::vector<std::string> dofLabels = {"t", "i", "deltaTime"};
  for (int bi = 0; bi < d.n_bcs; ++bi) {
    const dl_bc_desc &b = d.bcs[bi];
    if (b.dof < 0 || b.dof > 5) throw std::invalid_argument("bc dof out of range");
    for (int k = 0; k < b.n_nodes; ++k)
      if (b.nodes[k] < 0 || b.nodes[k] >= N) throw std::invalid_argument("bc node out of range");
    if (b.kind == DL_BC_INIT_VELO) {
      for (int k = 0; k < b.n_nodes; ++k) h.vel[static_cast<size_t>(b.dof) * N + h.node_new[b.nodes[k]]] = b.factor;
      continue;
    }
    if (b.kind == DL_BC_MASS) {  // MassModel (MassModel.cpp:77-99): diagonal of the node's mass matrix
      if (!std::isfinite(b.factor)) throw std::invalid_argument("added mass must be finite");
      if (h.madd.empty()) h.madd.assign(static_cast<size_t>(6) * N, 0.0);
      for (int k = 0; k < b.n_nodes; ++k) h.madd[static_cast<size_t>(b.dof) * N + h.node_new[b.nodes[k]]] += b.factor;
      continue;
    }
    if (b.kind == DL_BC_INIT_DISP) {
      for (int k = 0; k < b.n_nodes; ++k) {
        const int ni = h.node_new[b.nodes[k]];
        if (b.dof < 3) {
          h.pos[ni * 4 + b.dof] += b.factor;
        } else {
          // rotation vector component (InitLoadModel sets the rx/ry/rz DOF)
          double th[3];
          V3<double> cur = qlog(Q4<double>{h.rot[ni * 4], h.rot[ni * 4 + 1], h.rot[ni * 4 + 2], h.rot[ni * 4 + 3]});
          th[0] = cur.x;
          th[1] = cur.y;
          th[2] = cur.z;
          th[b.dof - 3] = b.factor;
          Q4<double> q = qexp(V3<double>{th[0], th[1], th[2]});
          h.rot[ni * 4] = q.w;
          h.rot[ni * 4 + 1] = q.x;
          h.rot[ni * 4 + 2] = q.y;
          h.rot[ni * 4 + 3] = q.z;
        }
      }
      continue;
    }
    if (b.kind != DL_BC_DIRICHLET && b.kind != DL_BC_NEUMANN) throw std::invalid_argument("unknown bc kind");
    int sc = -1;
    if (b.scale && b.scale[0]) {
      for (size_t s = 0; s < h.scales.size(); ++s)
        if (h.scales[s].src == b.scale) sc = static_cast<int>(s);
      if (sc < 0) {
        ScaleFn f;
        f.src = b.scale;
        f.expr = parseExpr(b.scale, dofLabels);
        h.scales.push_back(f);
        sc = static_cast<int>(h.scales.size()) - 1;
      }
    }
    for (int k = 0; k < b.n_nodes; ++k) {
      BcTerm t{};
      t.kind = (b.kind == DL_BC_DIRICHLET) ? BCD_DIRICHLET : BCD_NEUMANN;
      t.dof = b.dof;
      t.scale = sc;
      t.factor = b.factor;
      perNode[h.node_new[b.nodes[k]]].push_back(t);
    }
  }
  if (h.ties && !h.madd.empty()) throw UnsupportedError("rigid ties with added point masses are not provided");
  if (h.ties) {
    // a group's boundary conditions act on all its members (master's terms
    // first, then the slaves' in order) and its members start from the
    // master's state; the group index lists the members, master first
    h.tie_ptr.assign(N + 1, 0);
    std::vector<std::vector<int32_t>> members(N);
    for (int n = 0; n < N; ++n) {
      if (slaves[n].empty()) continue;
      std::vector<int32_t> grp = {h.node_new[n]};
      for (int sl : slaves[n]) grp.push_back(h.node_new[sl]);
      std::vector<BcTerm> all;
      for (int32_t q : grp) all.insert(all.end(), perNode[q].begin(), perNode[q].end());
      for (int32_t q : grp) {
        perNode[q] = all;
        members[q] = grp;
        if (q == grp[0]) continue;
        for (int k = 0; k < 4; ++k) {
          h.pos[static_cast<size_t>(q) * 4 + k] = h.pos[static_cast<size_t>(grp[0]) * 4 + k];
          h.rot[static_cast<size_t>(q) * 4 + k] = h.rot[static_cast<size_t>(grp[0]) * 4 + k];
        }
        for (int k = 0; k < 6; ++k) h.vel[static_cast<size_t>(k) * N + q] = h.vel[static_cast<size_t>(k) * N + grp[0]];
      }
    }
    for (int i = 0; i < N; ++i) h.tie_ptr[i + 1] = h.tie_ptr[i] + static_cast<int32_t>(members[i].size());
    for (int i = 0; i < N; ++i) h.tie_nodes.insert(h.tie_nodes.end(), members[i].begin(), members[i].end());
  }
  h.bc_ptr.assign(N + 1, 0);
  for (int i = 0; i < N; ++i) h.bc_ptr[i + 1] = h.bc_ptr[i] + static_cast<int>(perNode[i].size());
  for (int i = 0; i < N; ++i) h.bc.insert(h.bc.end(), perNode[i].begin(), perNode[i].end());
  return L;
}

namespace {

// append the [rows][n] component-major array `src` of one lattice into the
// [rows][N] array `dst` of the union at column offset `off`
void append_soa(std::vector<double> &dst, size_t Ntot, const std::vector<double> &src, size_t n, size_t off,
                size_t rows) {
  for (size_t r = 0; r < rows; ++r)
    for (size_t i = 0; i < n; ++i) dst[r * Ntot + off + i] = src[r * n + i];
}

}  // namespace

std::unique_ptr<HostLattice> build_batch(const dl_model_desc *descs, int n, bool round_frames_to_float) {
  if (n <= 0 || !descs) throw std::invalid_argument("empty batch");
  std::vector<std::unique_ptr<HostLattice>> parts;
  for (int i = 0; i < n; ++i) {
    if (descs[i].nodes_per_elem != 2) throw UnsupportedError("batches take two-node elements");
    parts.push_back(build_lattice(descs[i], round_frames_to_float));
  }
  const HostLattice &p0 = *parts[0];
  auto U = std::make_unique<HostLattice>();
  HostLattice &u = *U;
  u.G = p0.G;
  u.nh = p0.nh;
  u.plastic = p0.plastic;
  u.so3 = p0.so3;
  u.gyro = p0.gyro;
  u.lumped = p0.lumped;
  u.dt = p0.dt;
  u.contact = p0.contact;
  u.n_lat = n;
  u.lat_node_off.assign(n + 1, 0);
  u.lat_elem_off.assign(n + 1, 0);
  for (int i = 0; i < n; ++i) {
    const HostLattice &p = *parts[i];
    if (p.G != p0.G || p.plastic != p0.plastic || p.nh != p0.nh || p.so3 != p0.so3 || p.gyro != p0.gyro ||
        p.lumped != p0.lumped)
      throw std::invalid_argument("lattices of a batch must share the Gauss rule, material law and update options");
    if (p.plastic) {
      if (p.yield_key != p0.yield_key) throw std::invalid_argument("lattices of a batch must share the yield function");
      for (int a = 0; a < 7; ++a)
        for (int b = 0; b < 7; ++b)
          if (p.H[a][b] != p0.H[a][b]) throw std::invalid_argument("lattices of a batch must share the hardening law");
      if (p.max_iter != p0.max_iter || p.prec != p0.prec)
        throw std::invalid_argument("lattices of a batch must share maxIter/precision");
    }
    if (p.contact.enabled || p.jcontact.enabled) throw std::invalid_argument("contact is not supported in batches");
    if (!p.madd.empty()) throw std::invalid_argument("added masses are not supported in batches");
    if (p.ties) throw std::invalid_argument("rigid ties are not supported in batches");
    u.lat_node_off[i + 1] = u.lat_node_off[i] + p.N;
    u.lat_elem_off[i + 1] = u.lat_elem_off[i] + p.E;
  }
  const int N = u.lat_node_off[n], E = u.lat_elem_off[n], G = u.G;
  u.N = N;
  u.E = E;
  u.yield = p0.yield;
  u.grad = p0.grad;
  u.yield_expr = p0.yield_expr;
  u.grad_exprs = p0.grad_exprs;
  u.yield_key = p0.yield_key;
  std::memcpy(u.H, p0.H, sizeof u.H);
  u.max_iter = p0.max_iter;
  u.prec = p0.prec;
  u.node_new.resize(N);
  u.node_old.resize(N);
  u.elem_new.resize(E);
  u.elem_old.resize(E);
  u.X0.resize(static_cast<size_t>(N) * 3);
  u.pos.resize(static_cast<size_t>(N) * 4);
  u.rot.resize(static_cast<size_t>(N) * 4);
  u.vel.assign(static_cast<size_t>(N) * 6, 0.0);
  u.mass.resize(N);
  u.iframe.resize(static_cast<size_t>(N) * 4);
  u.idiag.resize(static_cast<size_t>(N) * 4);
  u.slot_ptr.assign(N + 1, 0);
  u.bc_ptr.assign(N + 1, 0);
  u.eslot.resize(static_cast<size_t>(E) * 2);
  u.conn.resize(static_cast<size_t>(E) * 2);
  u.invL0.resize(E);
  u.qN.resize(static_cast<size_t>(2) * E * 4);
  u.g0.resize(static_cast<size_t>(G) * 3 * E);
  u.k0.resize(static_cast<size_t>(G) * 3 * E);
  u.C.resize(static_cast<size_t>(6) * E);
  u.ec.resize(static_cast<size_t>(2) * E);
  u.elem_rod.resize(E);
  u.dtn.resize(N);
  u.nlat.resize(N);
  u.elat.resize(E);
  int rod_off = 0, slot_off = 0, bc_off = 0;
  for (int i = 0; i < n; ++i) {
    const HostLattice &p = *parts[i];
    const int no = u.lat_node_off[i], eo = u.lat_elem_off[i];
    const int sc_off = static_cast<int>(u.scales.size());
    u.scales.insert(u.scales.end(), p.scales.begin(), p.scales.end());
    for (int k = 0; k < p.N; ++k) {
      u.node_new[no + k] = no + p.node_new[k];
      u.node_old[no + k] = no + p.node_old[k];
      u.mass[no + k] = p.mass[k];
      u.dtn[no + k] = p.dt;
      u.nlat[no + k] = i;
      u.slot_ptr[no + k + 1] = slot_off + p.slot_ptr[k + 1];
      u.bc_ptr[no + k + 1] = bc_off + p.bc_ptr[k + 1];
      for (int c = 0; c < 4; ++c) {
        u.pos[(no + k) * 4 + c] = p.pos[k * 4 + c];
        u.rot[(no + k) * 4 + c] = p.rot[k * 4 + c];
        u.iframe[(no + k) * 4 + c] = p.iframe[k * 4 + c];
        u.idiag[(no + k) * 4 + c] = p.idiag[k * 4 + c];
      }
    }
    std::copy(p.X0.begin(), p.X0.end(), u.X0.begin() + static_cast<size_t>(no) * 3);
    append_soa(u.vel, N, p.vel, p.N, no, 6);
    for (BcTerm t : p.bc) {
      if (t.scale >= 0) t.scale += sc_off;
      u.bc.push_back(t);
    }
    int max_rod = -1;
    for (int k = 0; k < p.E; ++k) {
      u.elem_new[eo + k] = eo + p.elem_new[k];
      u.elem_old[eo + k] = eo + p.elem_old[k];
      u.conn[(eo + k) * 2] = no + p.conn[k * 2];
      u.conn[(eo + k) * 2 + 1] = no + p.conn[k * 2 + 1];
      u.eslot[(eo + k) * 2] = slot_off + p.eslot[k * 2];
      u.eslot[(eo + k) * 2 + 1] = slot_off + p.eslot[k * 2 + 1];
      u.invL0[eo + k] = p.invL0[k];
      u.elem_rod[eo + k] = rod_off + p.elem_rod[k];
      max_rod = std::max(max_rod, p.elem_rod[k]);
      u.elat[eo + k] = i;
      for (int s2 = 0; s2 < 2; ++s2)
        for (int c = 0; c < 4; ++c)
          u.qN[(static_cast<size_t>(s2) * E + eo + k) * 4 + c] = p.qN[(static_cast<size_t>(s2) * p.E + k) * 4 + c];
    }
    append_soa(u.g0, E, p.g0, p.E, eo, static_cast<size_t>(G) * 3);
    append_soa(u.k0, E, p.k0, p.E, eo, static_cast<size_t>(G) * 3);
    append_soa(u.C, E, p.C, p.E, eo, 6);
    append_soa(u.ec, E, p.ec, p.E, eo, 2);
    rod_off += max_rod + 1;
    slot_off += p.slot_ptr[p.N];
    bc_off += static_cast<int>(p.bc.size());
  }
  return U;
}

}  // namespace dl
