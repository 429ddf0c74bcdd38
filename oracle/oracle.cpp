// oracle.cpp -- CPU oracle: FP64 restatement of dynLattice's explicit path.
//
// TEST INFRASTRUCTURE ONLY (see oracle.h).  Every routine names the reference
// routine it restates; the arithmetic follows the reference's matrix
// formulation (3x3 rotation matrices, logMat via acos, Rodrigues expVec,
// expVecP, Crisfield--Jelenic interpolation) including its redundant
// recomputation, so that the oracle is also a faithful CPU cost baseline.
//
// Deliberate deviations, each also applied by the engine:
//  * LeapFrogModule::solve (LeapFrogModule.cpp:44-84) never stores u_new/v_new;
//    the oracle stores them ("as intended", as MilneDeviceModule.cpp:107-108 does).
//  * The time step is fixed at deltaTime (the reference would grow it by
//    increaseFactor per step because LeapFrog reports residual 0,
//    ExplicitModule.cpp:299-313).
//  * Mass: the node-block-diagonal mass of SpecialCosseratRodModel::assembleM_
//    (SpecialCosseratRodModel.cpp:969-1031) is inverted exactly per node (the
//    reference's consistent mode hands the same matrix to a JIVE solver).

#include "oracle.h"
#include "expr.hpp"

#include <algorithm>
#include <cfloat>
#include <cmath>
#include <cstring>
#include <memory>
#include <stdexcept>
#include <string>
#include <vector>
#ifdef _OPENMP
#include <omp.h>
#endif

namespace {

thread_local std::string g_err;

// ---------------------------------------------------------------------------
// 3x3 algebra and SO(3) helpers (src/utils/helpers.cpp)
// ---------------------------------------------------------------------------
struct M3 {
  double a[3][3];
};
struct V3 {
  double v[3];
  double &operator[](int i) { return v[i]; }
  double operator[](int i) const { return v[i]; }
};

inline M3 zero3() {
  M3 r;
  std::memset(&r, 0, sizeof r);
  return r;
}
// helpers.cpp:84-93 (eye)
inline M3 eye3() {
  M3 r = zero3();
  r.a[0][0] = r.a[1][1] = r.a[2][2] = 1.0;
  return r;
}
inline M3 mul(const M3 &x, const M3 &y) {
  M3 r;
  for (int i = 0; i < 3; ++i)
    for (int j = 0; j < 3; ++j) {
      double s = 0.0;
      for (int k = 0; k < 3; ++k) s += x.a[i][k] * y.a[k][j];
      r.a[i][j] = s;
    }
  return r;
}
inline M3 tr(const M3 &x) {
  M3 r;
  for (int i = 0; i < 3; ++i)
    for (int j = 0; j < 3; ++j) r.a[i][j] = x.a[j][i];
  return r;
}
inline V3 mulv(const M3 &x, const V3 &y) {
  V3 r;
  for (int i = 0; i < 3; ++i) r[i] = x.a[i][0] * y[0] + x.a[i][1] * y[1] + x.a[i][2] * y[2];
  return r;
}
inline V3 mulTv(const M3 &x, const V3 &y) {  // x^T y
  V3 r;
  for (int i = 0; i < 3; ++i) r[i] = x.a[0][i] * y[0] + x.a[1][i] * y[1] + x.a[2][i] * y[2];
  return r;
}
inline M3 add(const M3 &x, const M3 &y) {
  M3 r;
  for (int i = 0; i < 3; ++i)
    for (int j = 0; j < 3; ++j) r.a[i][j] = x.a[i][j] + y.a[i][j];
  return r;
}
inline M3 scale(const M3 &x, double s) {
  M3 r;
  for (int i = 0; i < 3; ++i)
    for (int j = 0; j < 3; ++j) r.a[i][j] = x.a[i][j] * s;
  return r;
}
inline double norm2(const V3 &x) { return std::sqrt(x[0] * x[0] + x[1] * x[1] + x[2] * x[2]); }
inline double dot(const V3 &x, const V3 &y) { return x[0] * y[0] + x[1] * y[1] + x[2] * y[2]; }
inline V3 cross(const V3 &x, const V3 &y) {
  return V3{{x[1] * y[2] - x[2] * y[1], x[2] * y[0] - x[0] * y[2], x[0] * y[1] - x[1] * y[0]}};
}
// helpers.cpp:242-255 (skew)
inline M3 skew(const V3 &v) {
  M3 r = zero3();
  r.a[0][1] = -v[2];
  r.a[0][2] = v[1];
  r.a[1][2] = -v[0];
  r.a[1][0] = v[2];
  r.a[2][0] = -v[1];
  r.a[2][1] = v[0];
  return r;
}
// helpers.cpp:257-282 (unskew)
inline V3 unskew(const M3 &m) {
  V3 r;
  r[0] = (m.a[2][1] - m.a[1][2]) / 2.0;
  r[1] = (m.a[0][2] - m.a[2][0]) / 2.0;
  r[2] = (m.a[1][0] - m.a[0][1]) / 2.0;
  return r;
}
// jem::isTiny: true only for magnitudes at the bottom of the double range.
inline bool isTiny(double x) { return std::fabs(x) < DBL_MIN; }
const double TINY = DBL_EPSILON * 1e6;  // helpers.h:53

// helpers.cpp:139-157 (expVec)
inline M3 expVec(const V3 &psi) {
  M3 E = eye3();
  const double theta = norm2(psi);
  if (isTiny(theta)) return add(E, skew(psi));
  V3 k{{psi[0] / theta, psi[1] / theta, psi[2] / theta}};
  M3 K = skew(k);
  E = add(E, scale(K, std::sin(theta)));
  E = add(E, scale(mul(K, K), 1.0 - std::cos(theta)));
  return E;
}
// helpers.cpp:159-197 (expVecP)
inline M3 expVecP(const V3 &psi, const V3 &psiP) {
  const double theta = norm2(psi);
  if (theta < TINY) return skew(psiP);
  const double thetaP = dot(psi, psiP) / theta;
  V3 k, kP;
  for (int i = 0; i < 3; ++i) {
    k[i] = psi[i] / theta;
    kP[i] = (psiP[i] * theta - psi[i] * thetaP) / theta / theta;
  }
  M3 K = skew(k), KP = skew(kP);
  M3 r = scale(K, std::cos(theta) * thetaP);
  r = add(r, scale(KP, std::sin(theta)));
  r = add(r, scale(mul(K, K), std::sin(theta) * thetaP));
  r = add(r, scale(mul(K, KP), 1.0 - std::cos(theta)));
  r = add(r, scale(mul(KP, K), 1.0 - std::cos(theta)));
  return r;
}
// helpers.cpp:99-111 (logMat)
inline V3 logMat(const M3 &R) {
  double trR = R.a[0][0] + R.a[1][1] + R.a[2][2];
  if (trR > 3.0) trR = 3.0;
  const double theta = std::acos((trR - 1.0) / 2.0);
  M3 A;
  for (int i = 0; i < 3; ++i)
    for (int j = 0; j < 3; ++j) A.a[i][j] = R.a[i][j] - R.a[j][i];
  V3 rv = unskew(A);
  const double f = isTiny(theta) ? 0.5 : theta / (2.0 * std::sin(theta));
  for (int i = 0; i < 3; ++i) rv[i] *= f;
  return rv;
}

// ---------------------------------------------------------------------------
// Line3D (src/misc/Line3D.cpp) for 2/3/4-node lines, Gauss 1..4 points
// ---------------------------------------------------------------------------
struct Line {
  int n = 2, G = 2;
  double xi[4], W[4];
  double N[4][4];   // N[node][gp]
  double dN[4][4];  // dN/dxi [node][gp]

  static void gauss(int G, double *xi, double *W) {
    switch (G) {
      case 1: xi[0] = 0; W[0] = 2; break;
      case 2: xi[0] = -1 / std::sqrt(3.0); xi[1] = -xi[0]; W[0] = W[1] = 1; break;
      case 3:
        xi[0] = -std::sqrt(0.6); xi[1] = 0; xi[2] = std::sqrt(0.6);
        W[0] = W[2] = 5.0 / 9.0; W[1] = 8.0 / 9.0;
        break;
      case 4: {
        const double a = std::sqrt(3.0 / 7.0 - 2.0 / 7.0 * std::sqrt(1.2));
        const double b = std::sqrt(3.0 / 7.0 + 2.0 / 7.0 * std::sqrt(1.2));
        const double wa = (18.0 + std::sqrt(30.0)) / 36.0, wb = (18.0 - std::sqrt(30.0)) / 36.0;
        xi[0] = -b; xi[1] = -a; xi[2] = a; xi[3] = b;
        W[0] = wb; W[1] = wa; W[2] = wa; W[3] = wb;
        break;
      }
      default: throw std::runtime_error("unsupported Gauss scheme");
    }
  }
  void init(int nn, int ng) {
    n = nn;
    G = ng;
    gauss(G, xi, W);
    double xn[4];
    for (int i = 0; i < n; ++i) xn[i] = -1.0 + 2.0 * i / (n - 1);
    for (int g = 0; g < G; ++g)
      for (int i = 0; i < n; ++i) {
        double l = 1.0, dl = 0.0;
        for (int j = 0; j < n; ++j) {
          if (j == i) continue;
          l *= (xi[g] - xn[j]) / (xn[i] - xn[j]);
        }
        for (int k = 0; k < n; ++k) {
          if (k == i) continue;
          double p = 1.0 / (xn[i] - xn[k]);
          for (int j = 0; j < n; ++j) {
            if (j == i || j == k) continue;
            p *= (xi[g] - xn[j]) / (xn[i] - xn[j]);
          }
          dl += p;
        }
        N[i][g] = l;
        dN[i][g] = dl;
      }
  }
  // Line3D::getIntegrationWeights / getShapeGradients (Line3D.cpp:91-115):
  // 1-D coordinates are the accumulated chord lengths of the reference nodes.
  void weightsGrads(const V3 *X0, double *w, double (*g)[4]) const {
    double c1[4];
    c1[0] = 0.0;
    for (int i = 1; i < n; ++i) {
      V3 d{{X0[i][0] - X0[i - 1][0], X0[i][1] - X0[i - 1][1], X0[i][2] - X0[i - 1][2]}};
      c1[i] = norm2(d) + c1[i - 1];
    }
    for (int q = 0; q < G; ++q) {
      double J = 0.0;
      for (int i = 0; i < n; ++i) J += dN[i][q] * c1[i];
      w[q] = W[q] * std::fabs(J);
      if (g)
        for (int i = 0; i < n; ++i) g[i][q] = dN[i][q] / J;
    }
  }
  // Line3D::getRefRot_ (Line3D.cpp:249-263)
  M3 refRot(const M3 *Rn) const {
    const int I = (n - 1) / 2, J = n / 2;
    V3 phi = logMat(mul(tr(Rn[I]), Rn[J]));
    for (int k = 0; k < 3; ++k) phi[k] *= 0.5;
    return mul(Rn[I], expVec(phi));
  }
  // Line3D::getNodeRotVecs_ (Line3D.cpp:265-273)
  void nodeRotVecs(const M3 *Rn, V3 *psi, M3 &Lr) const {
    Lr = refRot(Rn);
    for (int i = 0; i < n; ++i) psi[i] = logMat(mul(tr(Lr), Rn[i]));
  }
  // Line3D::getRotations (Line3D.cpp:117-139)
  void rotations(const M3 *Rn, M3 *Ri) const {
    V3 psi[4];
    M3 Lr;
    nodeRotVecs(Rn, psi, Lr);
    for (int q = 0; q < G; ++q) {
      V3 ip{{0, 0, 0}};
      for (int i = 0; i < n; ++i)
        for (int k = 0; k < 3; ++k) ip[k] += psi[i][k] * N[i][q];
      Ri[q] = mul(Lr, expVec(ip));
    }
  }
  // Line3D::getRotationGradients (Line3D.cpp:216-244)
  void rotationGradients(const V3 *X0, const M3 *Rn, M3 *LP) const {
    V3 psi[4];
    M3 Lr;
    nodeRotVecs(Rn, psi, Lr);
    double w[4], g[4][4];
    weightsGrads(X0, w, g);
    for (int q = 0; q < G; ++q) {
      V3 ps{{0, 0, 0}}, pp{{0, 0, 0}};
      for (int i = 0; i < n; ++i)
        for (int k = 0; k < 3; ++k) {
          ps[k] += psi[i][k] * N[i][q];
          pp[k] += psi[i][k] * g[i][q];
        }
      LP[q] = mul(Lr, expVecP(ps, pp));
    }
  }
};

// ---------------------------------------------------------------------------
// materials (ElasticRodMaterial.cpp, ElastoPlasticRodMaterial.cpp)
// ---------------------------------------------------------------------------
struct ElemMat {
  int type = 0;
  double C[6];       // diag(GkA, GkA, EA, EI1, EI2, GJ)  ElasticRodMaterial.cpp:265-275
  double Mm[6];      // diag(rhoA x3, rhoI1, rhoI2, rhoJ) (x inertia_correct)  :277-287, :192-195
  double rhoA = 0;   // for the l^3/12 term of getLumpedMass (:289-297)
  double radius = 0, area = 0;
  int mat = 0;
};

struct PlasticLaw {
  orc::Expr f;
  std::vector<orc::Expr> df;
  int nh = 0;                 // hardening argument count
  double H[7][7];             // materialH_
  int maxIter = 20;
  double prec = 1e-5;
  bool hasDeriv = false;
};

struct Bc {
  int kind, dof;
  std::vector<int> nodes;
  double factor;
  orc::Expr scale;
  bool hasScale = false;
};

}  // namespace

struct orc_handle_s {
  // mesh
  int N = 0, E = 0, nen = 2, G = 2;
  std::vector<V3> X0;
  std::vector<int> conn;      // [E][nen]
  std::vector<int> rod;
  Line line;                  // stiffShape (Gauss G)
  Line mline;                 // massShape (Gauss nen), SpecialCosseratRodModel.cpp:105-108
  std::vector<ElemMat> em;
  std::vector<PlasticLaw> laws;
  std::vector<int> lawOf;     // per material index -> law index or -1
  // frames: Lambda_N per (element, local node) (per-rod initRotation_)
  std::vector<M3> LN;         // [E][nen]
  std::vector<double> strain0;  // [E][G][6]
  // state
  std::vector<V3> u, th;
  std::vector<double> v;      // [N][6]
  // material history
  std::vector<double> epsOld, epsCur, epOld, epCur, hpOld, hpCur, dflow, ediss, epot;
  int nhMax = 0;
  // BCs
  std::vector<Bc> bcs;
  double dt = 0;
  bool so3 = true, gyro = true;
  bool lumped = false;        // explicit module's LUMPED mode (diagonal MATRIX2)
  // rigid ties (HingeModel constraints): master of each slave (-1), slaves of each master
  std::vector<int> tieMaster;
  std::vector<std::vector<int>> tieSlaves;
  double t = 0;
  int64_t step = 0;
  // sampling
  int every = 0;
  std::vector<int> watch;
  std::vector<int64_t> sampSteps;
  std::vector<double> sampRows;
  std::vector<dl_energies> sampEn;
  dl_energies last{};
  uint32_t errword = 0;
  std::vector<std::string> argNames;
  // work
  std::vector<double> fint, fext;
  std::vector<double> mT;     // [N]
  std::vector<M3> mR;         // [N]
  double wext = 0;
  // contact (RodContactModel) and rigid plates
  dl_contact_desc contact{};
  std::vector<std::vector<int>> rodElems;      // elements of each rod, mesh order
  std::vector<std::vector<int>> rodNodes;      // sorted node indices of each rod
  std::vector<std::pair<int, int>> blacklist;  // (elemA, elemB) closed at INIT
  std::vector<std::pair<int, int>> closedPairs;  // pairs that produced force in the last step
  std::vector<double> closedGaps;
  double contactEnergy = 0.0;
  std::vector<double> plateReaction;           // [n_plates][3] last step
  // added point masses (MassModel): [N][6] diagonal, empty if none
  std::vector<double> madd;
  // joint contact (JointContactModel)
  dl_joint_contact_desc jc{};
  std::vector<int> joints;                     // the "points" group, in order
  std::vector<std::pair<int, int>> closedJointPairs;  // (node, node) in contact in the last step
  std::vector<double> closedJointGaps;
  // explicit module (ExplicitModule.cpp:36-47, 124-148)
  int integ = DL_INTEG_LEAPFROG;
  double prec = 0.0, minDt = 0.0, maxDt = 0.0, safety = 0.9, incrFact = 1.2, decrFact = 0.8, lenScale = 1e-3;
  int64_t rejected = 0;
  std::vector<double> sampTimes;
};

namespace {

// ---------------------------------------------------------------------------
// SpecialCosseratRodModel pieces
// ---------------------------------------------------------------------------
struct ElemCtx {
  V3 X0[4], U[4];
  M3 Rn[4];
};

// SpecialCosseratRodModel::getDisplacments_ (SpecialCosseratRodModel.cpp:773-798)
void getDisplacements(const orc_handle_s &h, int e, const V3 *u, const V3 *th, ElemCtx &c) {
  for (int a = 0; a < h.nen; ++a) {
    int nd = h.conn[e * h.nen + a];
    c.X0[a] = h.X0[nd];
    c.U[a] = u[nd];
    c.Rn[a] = mul(expVec(th[nd]), h.LN[e * h.nen + a]);
  }
}

// SpecialCosseratRodModel::getStrains_ (SpecialCosseratRodModel.cpp:694-744), material frame
void getStrains(const orc_handle_s &h, int e, const ElemCtx &c, double (*strain)[6], bool subtract0) {
  const Line &L = h.line;
  double w[4], g[4][4];
  L.weightsGrads(c.X0, w, g);
  M3 Ri[4], LP[4];
  L.rotations(c.Rn, Ri);                 // getPi(ipPI, ipLambda, nodeLambda)
  L.rotationGradients(c.X0, c.Rn, LP);   // getRotationGradients
  for (int q = 0; q < L.G; ++q) {
    V3 phiP{{0, 0, 0}};
    for (int i = 0; i < L.n; ++i)
      for (int k = 0; k < 3; ++k) phiP[k] += (c.X0[i][k] + c.U[i][k]) * g[i][q];
    V3 gam = mulTv(Ri[q], phiP);
    V3 kap = unskew(mul(tr(Ri[q]), LP[q]));
    for (int k = 0; k < 3; ++k) {
      strain[q][k] = gam[k];
      strain[q][k + 3] = kap[k];
    }
    if (subtract0)
      for (int k = 0; k < 6; ++k) strain[q][k] -= h.strain0[(e * h.G + q) * 6 + k];
  }
}

double *hp(std::vector<double> &v, const orc_handle_s &h, int e, int q) {
  return &v[(static_cast<size_t>(e) * h.G + q) * (h.nhMax > 0 ? h.nhMax : 1)];
}

// ElasticRodMaterial::getStress (ElasticRodMaterial.cpp:369-373) and
// ElastoPlasticRodMaterial::getStress (ElastoPlasticRodMaterial.cpp:198-269)
bool materialStress(orc_handle_s &h, int e, int q, const double *strain, double *stress, bool inelastic) {
  const ElemMat &m = h.em[e];
  const size_t gi = static_cast<size_t>(e) * h.G + q;
  int li = h.lawOf[m.mat];
  if (m.type == DL_MAT_ELASTIC_ROD || li < 0) {
    for (int k = 0; k < 6; ++k) {
      h.epsCur[gi * 6 + k] = strain[k];
      stress[k] = m.C[k] * strain[k];
    }
    return true;
  }
  const PlasticLaw &P = h.laws[li];
  const int nh = P.nh;
  double ep[6], hpar[7], hs[7];
  for (int k = 0; k < 6; ++k) ep[k] = h.epOld[gi * 6 + k];
  for (int k = 0; k < nh; ++k) hpar[k] = hp(h.hpOld, h, e, q)[k];
  double deltaFlow = 0.0;
  int liter = 0;
  double args[32];
  const int nbase = 6 + nh;
  args[nbase] = m.radius;      // engine-extension element variables
  args[nbase + 1] = m.area;
  bool ok = true;
  for (;;) {
    for (int k = 0; k < 6; ++k) stress[k] = m.C[k] * (strain[k] - ep[k]);
    for (int a = 0; a < nh; ++a) {  // getHardVals: -H alpha (:185-188)
      double s = 0.0;
      for (int b = 0; b < nh; ++b) s += P.H[a][b] * hpar[b];
      hs[a] = -s;
    }
    if (!inelastic) break;
    for (int k = 0; k < 6; ++k) args[k] = stress[k];
    for (int a = 0; a < nh; ++a) args[6 + a] = hs[a];
    const double fval = P.f.eval(args);
    if (!(liter < P.maxIter)) {  // JEM_PRECHECK2 precedes the convergence test (:234)
      __atomic_fetch_or(&h.errword, DL_EW_RETURN_MAP, __ATOMIC_RELAXED);
      ok = false;
      break;
    }
    if (fval < P.prec) break;
    double grad[13];
    if (P.hasDeriv) {
      for (int k = 0; k < nbase; ++k) grad[k] = P.df[k].eval(args);
    } else {
      // numerical gradient (JEM getDeriv is not available: unpinned path)
      for (int k = 0; k < nbase; ++k) {
        double save = args[k];
        double hstep = 1e-7 * std::max(1.0, std::fabs(save));
        args[k] = save + hstep;
        double fp = P.f.eval(args);
        args[k] = save - hstep;
        double fm = P.f.eval(args);
        args[k] = save;
        grad[k] = (fp - fm) / (2 * hstep);
      }
      for (int k = 0; k < 6; ++k)
        if (std::fabs(args[k]) < DBL_EPSILON) grad[k] = 0.0;
    }
    double den = 0.0;
    for (int k = 0; k < 6; ++k) den += grad[k] * m.C[k] * grad[k];
    for (int a = 0; a < nh; ++a) {
      double s = 0.0;
      for (int b = 0; b < nh; ++b) s += P.H[a][b] * grad[6 + b];
      den += grad[6 + a] * s;
    }
    const double ddf = fval / den;
    for (int k = 0; k < 6; ++k) ep[k] += ddf * grad[k];
    for (int a = 0; a < nh; ++a) hpar[a] += ddf * grad[6 + a];
    deltaFlow += ddf;
    ++liter;
  }
  for (int k = 0; k < 6; ++k) {
    h.epsCur[gi * 6 + k] = strain[k];
    h.epCur[gi * 6 + k] = ep[k];
  }
  for (int a = 0; a < nh; ++a) hp(h.hpCur, h, e, q)[a] = hpar[a];
  h.dflow[gi] = deltaFlow;
  return ok;
}

// SpecialCosseratRodModel::getStresses_ (SpecialCosseratRodModel.cpp:746-771)
void getStresses(orc_handle_s &h, int e, const ElemCtx &c, double (*stress)[6], bool spatial, bool inelastic) {
  double strain[4][6];
  getStrains(h, e, c, strain, true);
  for (int q = 0; q < h.G; ++q) materialStress(h, e, q, strain[q], stress[q], inelastic);
  if (spatial) {
    M3 Ri[4];
    h.line.rotations(c.Rn, Ri);  // getPi again (:767)
    for (int q = 0; q < h.G; ++q) {
      V3 n{{stress[q][0], stress[q][1], stress[q][2]}}, m{{stress[q][3], stress[q][4], stress[q][5]}};
      V3 sn = mulv(Ri[q], n), sm = mulv(Ri[q], m);
      for (int k = 0; k < 3; ++k) {
        stress[q][k] = sn[k];
        stress[q][k + 3] = sm[k];
      }
    }
  }
}

// SpecialCosseratRodModel::assemble_(fint, disp) (SpecialCosseratRodModel.cpp:899-949)
// with Line3D::getXi (Line3D.cpp:141-162).  contrib[e][q][a][6] is the
// contribution w_q XI_{q,a} sigma_q; it is scattered afterwards in the
// reference's (element, ip, node) order.
void elementForce(orc_handle_s &h, int e, const V3 *u, const V3 *th, double *contrib, bool inelastic) {
  ElemCtx c;
  getDisplacements(h, e, u, th, c);
  const Line &L = h.line;
  double w[4], g[4][4];
  L.weightsGrads(c.X0, w, g);
  double stress[4][6];
  getStresses(h, e, c, stress, true, inelastic);
  for (int q = 0; q < L.G; ++q) {
    V3 phiP{{0, 0, 0}};
    for (int i = 0; i < L.n; ++i)
      for (int k = 0; k < 3; ++k) phiP[k] += (c.X0[i][k] + c.U[i][k]) * g[i][q];
    V3 n{{stress[q][0], stress[q][1], stress[q][2]}};
    V3 pxn = cross(phiP, n);  // skew(phiP) n
    for (int a = 0; a < L.n; ++a) {
      double *o = contrib + ((static_cast<size_t>(q) * L.n + a) * 6);
      for (int k = 0; k < 3; ++k) {
        o[k] = w[q] * g[a][q] * stress[q][k];
        o[k + 3] = w[q] * (g[a][q] * stress[q][k + 3] - L.N[a][q] * pxn[k]);
      }
    }
  }
}

void assembleFint(orc_handle_s &h, const V3 *u, const V3 *th, std::vector<double> &fint, bool inelastic) {
  const int E = h.E, G = h.G, n = h.nen;
  const size_t per = static_cast<size_t>(G) * n * 6;
  std::vector<double> contrib(static_cast<size_t>(E) * per);
#pragma omp parallel for schedule(static)
  for (int e = 0; e < E; ++e) elementForce(h, e, u, th, &contrib[e * per], inelastic);
  std::fill(fint.begin(), fint.end(), 0.0);
  for (int e = 0; e < E; ++e)
    for (int q = 0; q < G; ++q)
      for (int a = 0; a < n; ++a) {
        const double *o = &contrib[e * per + (static_cast<size_t>(q) * n + a) * 6];
        double *f = &fint[static_cast<size_t>(h.conn[e * n + a]) * 6];
        for (int k = 0; k < 6; ++k) f[k] += o[k];
      }
}

// SpecialCosseratRodModel::assembleM_ (SpecialCosseratRodModel.cpp:969-1031) with
// ElasticRodMaterial::getLumpedMass (ElasticRodMaterial.cpp:289-297): per node a
// translational scalar and a 3x3 rotational block.
void assembleMass(orc_handle_s &h, const V3 *th, std::vector<double> &mT, std::vector<M3> &mR) {
  std::fill(mT.begin(), mT.end(), 0.0);
  std::fill(mR.begin(), mR.end(), zero3());
  const Line &L = h.mline;
  for (int e = 0; e < h.E; ++e) {
    V3 X0[4];
    M3 Rn[4];
    for (int a = 0; a < h.nen; ++a) {
      int nd = h.conn[e * h.nen + a];
      X0[a] = h.X0[nd];
      Rn[a] = mul(expVec(th[nd]), h.LN[e * h.nen + a]);
    }
    double w[4];
    L.weightsGrads(X0, w, nullptr);
    double l = 0.0;
    for (int q = 0; q < L.G; ++q) l += w[q];
    l /= (h.nen - 1);
    const ElemMat &m = h.em[e];
    double D[3];
    D[0] = m.Mm[3] * l + m.rhoA * l * l * l / 12.0;
    D[1] = m.Mm[4] * l + m.rhoA * l * l * l / 12.0;
    D[2] = m.Mm[5] * l;
    for (int a = 0; a < h.nen; ++a) {
      int nd = h.conn[e * h.nen + a];
      double s = 0.0;
      for (int b = 0; b < h.nen; ++b)
        for (int q = 0; q < L.G; ++q) s += w[q] * L.N[a][q] * L.N[b][q];
      mT[nd] += s * m.Mm[0];
      M3 blk;
      for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j) {
          double acc = 0.0;
          for (int k = 0; k < 3; ++k) acc += Rn[a].a[i][k] * D[k] * Rn[a].a[j][k];
          blk.a[i][j] = acc;
        }
      if (a == 0 || a == h.nen - 1) blk = scale(blk, 0.5);
      mR[nd] = add(mR[nd], blk);
    }
  }
  // LUMPED mode (ExplicitModule.cpp:154-172, 445-453): the model's MATRIX2
  // assembled into a diagonal matrix keeps each DOF's diagonal entry
  if (h.lumped)
    for (int nd = 0; nd < h.N; ++nd)
      for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j)
          if (i != j) mR[nd].a[i][j] = 0.0;
}

// 3x3 solve of M x = b for the unconstrained components (mask bit set = constrained, value in x)
void solveBlock(const M3 &M, const double *b, double *x, unsigned mask) {
  int fr[3], nf = 0;
  for (int i = 0; i < 3; ++i)
    if (!(mask & (1u << i))) fr[nf++] = i;
  if (nf == 0) return;
  double A[3][3], r[3];
  for (int i = 0; i < nf; ++i) {
    r[i] = b[fr[i]];
    for (int j = 0; j < 3; ++j)
      if (mask & (1u << j)) r[i] -= M.a[fr[i]][j] * x[j];
    for (int j = 0; j < nf; ++j) A[i][j] = M.a[fr[i]][fr[j]];
  }
  // Gaussian elimination with partial pivoting
  int idx[3] = {0, 1, 2};
  for (int k = 0; k < nf; ++k) {
    int p = k;
    for (int i = k + 1; i < nf; ++i)
      if (std::fabs(A[i][k]) > std::fabs(A[p][k])) p = i;
    if (p != k) {
      for (int j = 0; j < nf; ++j) std::swap(A[k][j], A[p][j]);
      std::swap(r[k], r[p]);
    }
    for (int i = k + 1; i < nf; ++i) {
      double f = A[i][k] / A[k][k];
      for (int j = k; j < nf; ++j) A[i][j] -= f * A[k][j];
      r[i] -= f * r[k];
    }
  }
  double y[3] = {0.0, 0.0, 0.0};
  for (int k = nf - 1; k >= 0; --k) {
    double s = r[k];
    for (int j = k + 1; j < nf; ++j) s -= A[k][j] * y[j];
    y[k] = s / A[k][k];
  }
  (void)idx;
  for (int i = 0; i < nf; ++i) x[fr[i]] = y[i];
}

// a = M^-1 r for the free components of one node (constrained ones preset):
// the explicit module's mass matrix is the sum of all GET_MATRIX2
// contributions, the rods' node blocks plus the Mass models' diagonal
// (MassModel.cpp:77-99)
void nodeAccel(const orc_handle_s &h, int nd, const double *r, double *a, unsigned mask) {
  const double *ma = h.madd.empty() ? nullptr : &h.madd[static_cast<size_t>(nd) * 6];
  for (int k = 0; k < 3; ++k)
    if (!(mask & (1u << k))) a[k] = r[k] / (h.mT[nd] + (ma ? ma[k] : 0.0));
  M3 Mr = h.mR[nd];
  if (ma)
    for (int i = 0; i < 3; ++i) Mr.a[i][i] += ma[3 + i];
  solveBlock(Mr, r + 3, a + 3, (mask >> 3) & 7u);
}

// Translational mass a node is solved with: its own, or its tie group's.
double groupMass(const orc_handle_s &h, int nd) {
  if (h.tieMaster.empty()) return h.mT[nd];
  const int ms = h.tieMaster[nd] >= 0 ? h.tieMaster[nd] : nd;
  double m = h.mT[ms];
  for (int sl : h.tieSlaves[ms]) m += h.mT[sl];
  return m;
}

// Accelerations of all nodes from the residual forces r = fext - fint [N][6]
// with the prescribed values of the masked DOFs preset in a.  A rigid tie
// group (HingeModel constraints, HingeModel.cpp:172-199, with the offset
// zero of an explicit run) is solved as the constrained system's condensed
// equation: summed mass and residual of its members, the members' prescribed
// DOFs, one acceleration for all of them.
void allAccel(const orc_handle_s &h, const std::vector<double> &r, std::vector<double> &a,
              const std::vector<unsigned> &mask) {
  for (int nd = 0; nd < h.N; ++nd) {
    const bool tied = !h.tieMaster.empty();
    if (tied && h.tieMaster[nd] >= 0) continue;  // a slave: solved with its master
    if (!tied || h.tieSlaves[nd].empty()) {
      nodeAccel(h, nd, &r[static_cast<size_t>(nd) * 6], &a[static_cast<size_t>(nd) * 6], mask[nd]);
      continue;
    }
    double rc[6], ac[6];
    unsigned mc = mask[nd];
    double mt = h.mT[nd];
    M3 Mr = h.mR[nd];
    for (int k = 0; k < 6; ++k) {
      rc[k] = r[static_cast<size_t>(nd) * 6 + k];
      ac[k] = a[static_cast<size_t>(nd) * 6 + k];
    }
    for (int sl : h.tieSlaves[nd]) {
      for (int k = 0; k < 6; ++k) {
        rc[k] += r[static_cast<size_t>(sl) * 6 + k];
        if ((mask[sl] & (1u << k)) && !(mc & (1u << k))) ac[k] = a[static_cast<size_t>(sl) * 6 + k];
      }
      mc |= mask[sl];
      mt += h.mT[sl];
      Mr = add(Mr, h.mR[sl]);
    }
    for (int k = 0; k < 3; ++k)
      if (!(mc & (1u << k))) ac[k] = rc[k] / mt;
    solveBlock(Mr, rc + 3, ac + 3, (mc >> 3) & 7u);
    for (int k = 0; k < 6; ++k) a[static_cast<size_t>(nd) * 6 + k] = ac[k];
    for (int sl : h.tieSlaves[nd])
      for (int k = 0; k < 6; ++k) a[static_cast<size_t>(sl) * 6 + k] = ac[k];
  }
}

double evalScale(const Bc &b, double t, double i, double dt) {
  if (!b.hasScale) return 1.0;
  double vars[3] = {t, i, dt};
  return b.scale.eval(vars);
}

// ElasticRodMaterial::applyDeform (:377-389) / ElastoPlasticRodMaterial::applyDeform (:271-307)
void applyDeform(orc_handle_s &h) {
  const int G = h.G;
#pragma omp parallel for schedule(static)
  for (int e = 0; e < h.E; ++e) {
    const ElemMat &m = h.em[e];
    const bool plastic = (m.type == DL_MAT_ELASTOPLASTIC_ROD && h.lawOf[m.mat] >= 0);
    for (int q = 0; q < G; ++q) {
      const size_t gi = static_cast<size_t>(e) * G + q;
      if (!plastic) {
        double s = 0.0;
        for (int k = 0; k < 6; ++k) s += h.epsCur[gi * 6 + k] * m.C[k] * h.epsCur[gi * 6 + k];
        h.epot[gi] = 0.5 * s;
        for (int k = 0; k < 6; ++k) h.epsOld[gi * 6 + k] = h.epsCur[gi * 6 + k];
        continue;
      }
      double oldE[6], curE[6], dEp[6], so[6], sc[6];
      for (int k = 0; k < 6; ++k) {
        oldE[k] = h.epsOld[gi * 6 + k] - h.epOld[gi * 6 + k];
        curE[k] = h.epsCur[gi * 6 + k] - h.epCur[gi * 6 + k];
        dEp[k] = h.epCur[gi * 6 + k] - h.epOld[gi * 6 + k];
        so[k] = m.C[k] * oldE[k];
        sc[k] = m.C[k] * curE[k];
      }
      double s = 0.0;
      for (int k = 0; k < 6; ++k) s += curE[k] * sc[k];
      h.epot[gi] = 0.5 * s;
      if (std::fabs(h.dflow[gi]) > DBL_EPSILON) {
        double d = 0.0;
        for (int k = 0; k < 6; ++k) d += (so[k] + sc[k]) / 2.0 * dEp[k];
        h.ediss[gi] += d;
      }
      for (int k = 0; k < 6; ++k) {
        h.epsOld[gi * 6 + k] = h.epsCur[gi * 6 + k];
        h.epOld[gi * 6 + k] = h.epCur[gi * 6 + k];
      }
      const PlasticLaw &P = h.laws[h.lawOf[m.mat]];
      for (int a = 0; a < P.nh; ++a) hp(h.hpOld, h, e, q)[a] = hp(h.hpCur, h, e, q)[a];
      h.dflow[gi] = 0.0;
    }
  }
}

// energies as summed by SpecialCosseratRodModel (:1074-1197): w * N_n * value per node
void sumEnergies(const orc_handle_s &h, double &Epot, double &Ediss) {
  Epot = 0.0;
  Ediss = 0.0;
  for (int e = 0; e < h.E; ++e) {
    V3 X0[4];
    for (int a = 0; a < h.nen; ++a) X0[a] = h.X0[h.conn[e * h.nen + a]];
    double w[4];
    h.line.weightsGrads(X0, w, nullptr);
    for (int a = 0; a < h.nen; ++a)
      for (int q = 0; q < h.G; ++q) {
        const size_t gi = static_cast<size_t>(e) * h.G + q;
        Epot += w[q] * h.line.N[a][q] * h.epot[gi];
        Ediss += w[q] * h.line.N[a][q] * h.ediss[gi];
      }
  }
}

double kinetic(const orc_handle_s &h) {
  double ek = 0.0;
  for (int nd = 0; nd < h.N; ++nd) {
    const double *v = &h.v[static_cast<size_t>(nd) * 6];
    double s = h.mT[nd] * (v[0] * v[0] + v[1] * v[1] + v[2] * v[2]);
    for (int i = 0; i < 3; ++i)
      for (int j = 0; j < 3; ++j) s += v[3 + i] * h.mR[nd].a[i][j] * v[3 + j];
    // LatticeModel's E_kin uses the global mass matrix, Mass models included
    // (M_ = mbld->getMatrix(), LatticeModel.cpp:122-129, 223-250)
    if (!h.madd.empty())
      for (int k = 0; k < 6; ++k) s += h.madd[static_cast<size_t>(nd) * 6 + k] * v[k] * v[k];
    ek += 0.5 * s;
  }
  return ek;
}

// SpecialCosseratRodModel::initRotation_ (SpecialCosseratRodModel.cpp:574-658), per rod
void initRotation(orc_handle_s &h, const dl_model_desc *d) {
  h.LN.assign(static_cast<size_t>(h.E) * h.nen, eye3());
  std::vector<std::vector<int>> rodElems(d->n_rods > 0 ? d->n_rods : 1);
  for (int e = 0; e < h.E; ++e) rodElems[h.rod[e]].push_back(e);
  std::vector<V3> dirs(h.N);
  std::vector<char> touched(h.N, 0);
  for (auto &elems : rodElems) {
    for (int e : elems)
      for (int a = 0; a < h.nen; ++a) {
        int nd = h.conn[e * h.nen + a];
        dirs[nd] = V3{{0, 0, 0}};
        touched[nd] = 0;
      }
    const int n = h.nen;
    for (int e : elems) {
      const int *c = &h.conn[e * n];
      auto diff = [&](int a, int b) {
        return V3{{h.X0[c[a]][0] - h.X0[c[b]][0], h.X0[c[a]][1] - h.X0[c[b]][1], h.X0[c[a]][2] - h.X0[c[b]][2]}};
      };
      V3 d0 = diff(1, 0);
      for (int k = 0; k < 3; ++k) dirs[c[0]][k] += d0[k];
      for (int a = 1; a < n - 1; ++a) {
        V3 dm = diff(a + 1, a - 1);
        for (int k = 0; k < 3; ++k) dirs[c[a]][k] += dm[k];
      }
      V3 d1 = diff(n - 1, n - 2);
      for (int k = 0; k < 3; ++k) dirs[c[n - 1]][k] += d1[k];
    }
    for (int gdir = 0; gdir < d->n_given_dirs; ++gdir) {
      int nd = d->given_dir_nodes[gdir];
      bool inRod = false;
      for (int e : elems)
        for (int a = 0; a < n; ++a) inRod = inRod || (h.conn[e * n + a] == nd);
      if (inRod)
        for (int k = 0; k < 3; ++k) dirs[nd][k] = d->given_dirs[gdir * 3 + k];
    }
    for (int e : elems)
      for (int a = 0; a < n; ++a) {
        int nd = h.conn[e * n + a];
        if (touched[nd]) continue;
        touched[nd] = 1;
        double nn = norm2(dirs[nd]);
        for (int k = 0; k < 3; ++k) dirs[nd][k] /= nn;
      }
    for (int e : elems)
      for (int a = 0; a < n; ++a) {
        int nd = h.conn[e * n + a];
        const V3 &t = dirs[nd];
        M3 R;
        if (d->has_material_ey) {
          V3 ey{{d->material_ey[0], d->material_ey[1], d->material_ey[2]}};
          V3 ex = mulv(skew(ey), t);
          for (int k = 0; k < 3; ++k) {
            R.a[k][0] = ex[k];
            R.a[k][1] = ey[k];
            R.a[k][2] = t[k];
          }
        } else {
          V3 e3{{0, 0, 1}};
          V3 vv = mulTv(skew(t), e3);  // matmul(e3, skew(t)): row vector times matrix
          double c = dot(t, e3);
          R = eye3();
          if (std::fabs(c + 1.0) > DBL_EPSILON) {
            M3 S = skew(vv);
            R = add(R, add(S, scale(mul(S, S), 1.0 / (1.0 + c))));
          } else {
            R = scale(R, -1.0);
          }
        }
        h.LN[e * n + a] = R;
      }
  }
}

// SpecialCosseratRodModel::initStrain_ (SpecialCosseratRodModel.cpp:536-569)
void initStrain(orc_handle_s &h) {
  h.strain0.assign(static_cast<size_t>(h.E) * h.G * 6, 0.0);
  for (int e = 0; e < h.E; ++e) {
    ElemCtx c;
    for (int a = 0; a < h.nen; ++a) {
      int nd = h.conn[e * h.nen + a];
      c.X0[a] = h.X0[nd];
      c.U[a] = V3{{0, 0, 0}};
      c.Rn[a] = h.LN[e * h.nen + a];
    }
    double s[4][6];
    getStrains(h, e, c, s, false);
    for (int q = 0; q < h.G; ++q)
      for (int k = 0; k < 6; ++k) h.strain0[(static_cast<size_t>(e) * h.G + q) * 6 + k] = s[q][k];
  }
}


// ---------------------------------------------------------------------------
// RodContactModel (src/models/RodContactModel.cpp), force path
// ---------------------------------------------------------------------------
struct V3x {
  double v[3];
};

inline void posOf(const orc_handle_s &h, const V3 *u, int nd, double out[3]) {
  for (int k = 0; k < 3; ++k) out[k] = h.X0[nd][k] + u[nd][k];
}

bool inRod(const orc_handle_s &h, int rod, int node) {
  const auto &v = h.rodNodes[rod];
  return std::binary_search(v.begin(), v.end(), node);
}

// findPossibleBeams_ (:279-356) + findPossibleElements_ (:361-446): candidate element pairs
void findContacts(const orc_handle_s &h, const V3 *u, std::vector<int> &eA, std::vector<int> &eB) {
  const double r = h.contact.radius;
  const int R = static_cast<int>(h.rodNodes.size());
  std::vector<double> box(static_cast<size_t>(R) * 6);
  for (int i = 0; i < R; ++i) {
    double lo[3] = {1e300, 1e300, 1e300}, hi[3] = {-1e300, -1e300, -1e300};
    for (int nd : h.rodNodes[i]) {
      double p[3];
      posOf(h, u, nd, p);
      for (int k = 0; k < 3; ++k) {
        lo[k] = std::min(lo[k], p[k]);
        hi[k] = std::max(hi[k], p[k]);
      }
    }
    for (int k = 0; k < 3; ++k) {
      box[i * 6 + k] = lo[k] - r;
      box[i * 6 + 3 + k] = hi[k] + r;
    }
  }
  auto overlap = [](const double *a, const double *b) {
    bool c = true;
    for (int k = 0; k < 3; ++k) c = c && a[3 + k] >= b[k] && b[3 + k] >= a[k];
    return c;
  };
  for (int i = 0; i < R; ++i)
    for (int j = R - 1; j > i; --j) {
      if (!overlap(&box[i * 6], &box[j * 6])) continue;
      // findPossibleElements_(i, j)
      for (int a : h.rodElems[i]) {
        const int a0 = h.conn[a * 2], a1 = h.conn[a * 2 + 1];
        if (inRod(h, j, a0) || inRod(h, j, a1)) continue;
        double pa0[3], pa1[3], ba[6];
        posOf(h, u, a0, pa0);
        posOf(h, u, a1, pa1);
        for (int k = 0; k < 3; ++k) {
          ba[k] = std::min(pa0[k], pa1[k]) - r;
          ba[3 + k] = std::max(pa0[k], pa1[k]) + r;
        }
        for (int b : h.rodElems[j]) {
          const int b0 = h.conn[b * 2], b1 = h.conn[b * 2 + 1];
          if (inRod(h, i, b0) || inRod(h, i, b1)) continue;
          double pb0[3], pb1[3], bb[6];
          posOf(h, u, b0, pb0);
          posOf(h, u, b1, pb1);
          for (int k = 0; k < 3; ++k) {
            bb[k] = std::min(pb0[k], pb1[k]) - r;
            bb[3 + k] = std::max(pb0[k], pb1[k]) + r;
          }
          if (overlap(ba, bb)) {
            eA.push_back(a);
            eB.push_back(b);
          }
        }
      }
    }
}

inline double dot3(const double *a, const double *b) { return a[0] * b[0] + a[1] * b[1] + a[2] * b[2]; }

// findClosestPoints_ (:953-991), Wriggers/Zavarise: local coordinates in [-1, 1]
void closestPoints(const double A[2][3], const double B[2][3], double &uA, double &uB) {
  double bA[3], bB[3], tA[3], tB[3], d[3], vA[3], vB[3];
  for (int k = 0; k < 3; ++k) {
    bA[k] = A[1][k] + A[0][k];
    bB[k] = B[1][k] + B[0][k];
    tA[k] = A[1][k] - A[0][k];
    tB[k] = B[1][k] - B[0][k];
  }
  const double tAA = dot3(tA, tA), tBB = dot3(tB, tB), tAB = dot3(tB, tA);
  for (int k = 0; k < 3; ++k) {
    d[k] = bB[k] - bA[k];
    vA[k] = tB[k] * tAB - tA[k] * tBB;
    vB[k] = tA[k] * tAB - tB[k] * tAA;
  }
  const double den = tBB * tAA - tAB * tAB;
  uA = -1.0 * dot3(d, vA) / den;
  uB = +1.0 * dot3(d, vB) / den;
}

// getClosestPoint_ (:996-1026): projection of a point on a segment
double closestPoint(const double S[3], const double M[2][3]) {
  double bM[3], tM[3];
  for (int k = 0; k < 3; ++k) {
    bM[k] = M[1][k] + M[0][k];
    tM[k] = M[1][k] - M[0][k];
  }
  return (2 * dot3(S, tM) - dot3(tM, bM)) / dot3(tM, tM);
}

inline bool containsLocal(double u) { return u >= -1.0 && u <= 1.0; }
inline void globalPoint(const double P[2][3], double u, double out[3]) {
  const double n0 = 0.5 * (1.0 - u), n1 = 0.5 * (1.0 + u);
  for (int k = 0; k < 3; ++k) out[k] = n0 * P[0][k] + n1 * P[1][k];
}

// computeSTS_ (:1031-1152), force part; f[12] = (A0, A1, B0, B1)
bool computeSTS(double k, double r, const double A[2][3], const double B[2][3], double uA, double uB, double *f,
                double &gap) {
  double pA[3], pB[3], d[3];
  globalPoint(A, uA, pA);
  globalPoint(B, uB, pB);
  for (int c = 0; c < 3; ++c) d[c] = pB[c] - pA[c];
  const double dist = std::sqrt(dot3(d, d));
  if (isTiny(dist)) return false;
  if (dist > 2.0 * r) return false;
  gap = dist - 2.0 * r;
  if (!f) return true;
  const double NA[2] = {0.5 * (1.0 - uA), 0.5 * (1.0 + uA)}, NB[2] = {0.5 * (1.0 - uB), 0.5 * (1.0 + uB)};
  for (int c = 0; c < 3; ++c) {
    const double n = d[c] / dist;
    f[0 + c] += k * gap * (-NA[0] * n);
    f[3 + c] += k * gap * (-NA[1] * n);
    f[6 + c] += k * gap * (NB[0] * n);
    f[9 + c] += k * gap * (NB[1] * n);
  }
  return true;
}

// computeNTS_ (:1157-1208), force part; f[9] = (slave, M0, M1)
bool computeNTS(double k, double r, const double S[3], const double M[2][3], double uM, double *f, double &gap) {
  double pM[3], d[3];
  globalPoint(M, uM, pM);
  for (int c = 0; c < 3; ++c) d[c] = pM[c] - S[c];
  const double dist = std::sqrt(dot3(d, d));
  if (isTiny(dist)) return false;
  if (dist > 2.0 * r) return false;
  gap = dist - 2.0 * r;
  if (!f) return true;
  for (int c = 0; c < 3; ++c) {
    const double n = (S[c] - pM[c]) / dist;
    f[c] += k * gap * n;
    f[3 + c] += k * gap * (-0.5 * (1.0 - uM) * n);
    f[6 + c] += k * gap * (-0.5 * (1.0 + uM) * n);
  }
  return true;
}

// one candidate pair: the branch structure of computeContacts_ (:451-738) /
// computeBlacklist_ (:743-936).  Returns whether the contact is closed and adds
// the force (if f != nullptr) to f[12] in the order (A0, A1, B0, B1).
bool pairContact(const orc_handle_s &h, const double A[2][3], const double B[2][3], double *f, double &gapOut,
                 double &energy) {
  const double r = h.contact.radius, ks = h.contact.penalty_sts, kn = h.contact.penalty_nts;
  double uA = 0, uB = 0;
  closestPoints(A, B, uA, uB);
  double gap = 0.0;
  bool closed = false;
  gapOut = 0.0;
  if (containsLocal(uA) && containsLocal(uB)) {
    closed = computeSTS(ks, r, A, B, uA, uB, f, gap);
    if (closed) {
      gapOut = gap;
      energy += 0.5 * ks * gap * gap;
    }
  } else if (!containsLocal(uA) && containsLocal(uB)) {
    const int iA = (uA < -1.0) ? 0 : 1;
    // the reference projects node iA of element B here (RodContactModel.cpp:575)
    uB = closestPoint(B[iA], A);
    if (!containsLocal(uB)) return false;
    double fl[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0};
    closed = computeNTS(kn, r, A[iA], B, uB, f ? fl : nullptr, gap);
    if (closed) {
      gapOut = gap;
      energy += 0.5 * kn * gap * gap;
      if (f)
        for (int c = 0; c < 3; ++c) {
          f[iA * 3 + c] += fl[c];
          f[6 + c] += fl[3 + c];
          f[9 + c] += fl[6 + c];
        }
    }
  } else if (!containsLocal(uB) && containsLocal(uA)) {
    const int iB = (uB < -1.0) ? 0 : 1;
    uA = closestPoint(B[iB], A);
    if (!containsLocal(uA)) return false;
    double fl[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0};
    closed = computeNTS(kn, r, B[iB], A, uA, f ? fl : nullptr, gap);
    if (closed) {
      gapOut = gap;
      energy += 0.5 * kn * gap * gap;
      if (f)
        for (int c = 0; c < 3; ++c) {
          f[6 + iB * 3 + c] += fl[c];
          f[0 + c] += fl[3 + c];
          f[3 + c] += fl[6 + c];
        }
    }
  } else {
    // speculative NTS: both ends of A against B, then both ends of B against A
    bool first = true;
    for (int iA = 0; iA < 2; ++iA) {
      const double u = closestPoint(A[iA], B);
      if (!containsLocal(u)) continue;
      double fl[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0};
      if (computeNTS(kn, r, A[iA], B, u, f ? fl : nullptr, gap)) {
        closed = true;
        energy += 0.5 * kn * gap * gap;
        if (first || gap < gapOut) gapOut = gap;
        first = false;
        if (f)
          for (int c = 0; c < 3; ++c) {
            f[iA * 3 + c] += fl[c];
            f[6 + c] += fl[3 + c];
            f[9 + c] += fl[6 + c];
          }
      }
    }
    for (int iB = 0; iB < 2; ++iB) {
      const double u = closestPoint(B[iB], A);
      if (!containsLocal(u)) continue;
      double fl[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0};
      if (computeNTS(kn, r, B[iB], A, u, f ? fl : nullptr, gap)) {
        closed = true;
        energy += 0.5 * kn * gap * gap;
        if (first || gap < gapOut) gapOut = gap;
        first = false;
        if (f)
          for (int c = 0; c < 3; ++c) {
            f[6 + iB * 3 + c] += fl[c];
            f[0 + c] += fl[3 + c];
            f[3 + c] += fl[6 + c];
          }
      }
    }
  }
  return closed;
}

void pairPositions(const orc_handle_s &h, const V3 *u, int a, int b, double A[2][3], double B[2][3]) {
  posOf(h, u, h.conn[a * 2], A[0]);
  posOf(h, u, h.conn[a * 2 + 1], A[1]);
  posOf(h, u, h.conn[b * 2], B[0]);
  posOf(h, u, h.conn[b * 2 + 1], B[1]);
}

bool sameNodes(const orc_handle_s &h, int a, int b) {
  const int a0 = h.conn[a * 2], a1 = h.conn[a * 2 + 1], b0 = h.conn[b * 2], b1 = h.conn[b * 2 + 1];
  return a0 == b0 || a0 == b1 || a1 == b0 || a1 == b1;
}

// computeBlacklist_ (:743-936): pairs already in contact at INIT are ignored for good
void computeBlacklist(orc_handle_s &h) {
  std::vector<int> eA, eB;
  findContacts(h, h.u.data(), eA, eB);
  h.blacklist.clear();
  for (size_t i = 0; i < eA.size(); ++i) {
    if (sameNodes(h, eA[i], eB[i])) continue;
    double A[2][3], B[2][3], gap, en = 0.0;
    pairPositions(h, h.u.data(), eA[i], eB[i], A, B);
    if (pairContact(h, A, B, nullptr, gap, en)) h.blacklist.emplace_back(eA[i], eB[i]);
  }
  std::sort(h.blacklist.begin(), h.blacklist.end());
}

bool blacklisted(const orc_handle_s &h, int a, int b) {
  return std::binary_search(h.blacklist.begin(), h.blacklist.end(), std::make_pair(a, b)) ||
         std::binary_search(h.blacklist.begin(), h.blacklist.end(), std::make_pair(b, a));
}

// GET_INT_VECTOR of RodContactModel: contact forces on translational DOFs
void contactForces(orc_handle_s &h, std::vector<double> &fint) {
  std::vector<int> eA, eB;
  findContacts(h, h.u.data(), eA, eB);
  h.closedPairs.clear();
  h.closedGaps.clear();
  h.contactEnergy = 0.0;
  for (size_t i = 0; i < eA.size(); ++i) {
    const int a = eA[i], b = eB[i];
    if (sameNodes(h, a, b)) continue;
    if (blacklisted(h, a, b)) continue;
    double A[2][3], B[2][3], gap;
    pairPositions(h, h.u.data(), a, b, A, B);
    double f[12] = {0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0};
    if (!pairContact(h, A, B, f, gap, h.contactEnergy)) continue;
    const int nodes[4] = {h.conn[a * 2], h.conn[a * 2 + 1], h.conn[b * 2], h.conn[b * 2 + 1]};
    for (int q = 0; q < 4; ++q)
      for (int c = 0; c < 3; ++c) fint[static_cast<size_t>(nodes[q]) * 6 + c] += f[q * 3 + c];
    h.closedPairs.emplace_back(std::min(a, b), std::max(a, b));
    h.closedGaps.push_back(gap);
  }
}

// JointContactModel::takeAction(GET_INT_VECTOR) (JointContactModel.cpp:
// 122-149): findContacts_ (:236-275) over all joint pairs A < B in list order
// (in contact: current distance <= 2r, reference distance > 2r), then
// computeContact_ (:318-340) for each: n = (x_B - x_A)/d, f = k (2r - d) n,
// f_int(A) -= f, f_int(B) += f.  The contact energy is the potential of this
// force, -k (2r - d)^2 / 2 (not in the reference's energy tables).  A pair at
// d = 0 gets no force (the reference divides by d).
void jointForces(orc_handle_s &h, std::vector<double> &fint) {
  h.closedJointPairs.clear();
  h.closedJointGaps.clear();
  const double r2 = 2.0 * h.jc.radius, k = h.jc.penalty;
  const int J = static_cast<int>(h.joints.size());
  for (int ia = 0; ia + 1 < J; ++ia) {
    const int a = h.joints[ia];
    double xa[3];
    posOf(h, h.u.data(), a, xa);
    for (int ib = ia + 1; ib < J; ++ib) {
      const int b = h.joints[ib];
      double xb[3];
      posOf(h, h.u.data(), b, xb);
      const double dx = xb[0] - xa[0], dy = xb[1] - xa[1], dz = xb[2] - xa[2];
      const double d = std::sqrt(dx * dx + dy * dy + dz * dz);
      if (!(d <= r2)) continue;
      const V3 &Xa = h.X0[a], &Xb = h.X0[b];
      const double ex = Xa[0] - Xb[0], ey = Xa[1] - Xb[1], ez = Xa[2] - Xb[2];
      if (!(std::sqrt(ex * ex + ey * ey + ez * ez) > r2)) continue;
      h.closedJointPairs.emplace_back(std::min(a, b), std::max(a, b));
      h.closedJointGaps.push_back(d - r2);
      h.contactEnergy -= 0.5 * k * (r2 - d) * (r2 - d);
      if (!(d > 0.0)) continue;
      const double s = k * (r2 - d) / d;
      const double f[3] = {s * dx, s * dy, s * dz};
      for (int c = 0; c < 3; ++c) {
        fint[static_cast<size_t>(a) * 6 + c] -= f[c];
        fint[static_cast<size_t>(b) * 6 + c] += f[c];
      }
    }
  }
}

// rigid plates (engine extension): node--plane penalty with the node radius
void plateForces(orc_handle_s &h, std::vector<double> &fint, double t) {
  const int np = h.contact.n_plates;
  h.plateReaction.assign(static_cast<size_t>(np) * 3, 0.0);
  for (int p = 0; p < np; ++p) {
    const dl_plate_desc &pl = h.contact.plates[p];
    double pt[3];
    for (int k = 0; k < 3; ++k) pt[k] = pl.point0[k] + pl.velocity[k] * t;
    for (int nd = 0; nd < h.N; ++nd) {
      double x[3];
      posOf(h, h.u.data(), nd, x);
      const double g = (x[0] - pt[0]) * pl.normal[0] + (x[1] - pt[1]) * pl.normal[1] + (x[2] - pt[2]) * pl.normal[2] -
                       h.contact.radius;
      if (g >= 0.0) continue;
      for (int k = 0; k < 3; ++k) {
        fint[static_cast<size_t>(nd) * 6 + k] += pl.penalty * g * pl.normal[k];
        h.plateReaction[p * 3 + k] += pl.penalty * g * pl.normal[k];
      }
      h.contactEnergy += 0.5 * pl.penalty * g * g;
    }
  }
}

void record(orc_handle_s &h) {
  h.sampSteps.push_back(h.step);
  h.sampTimes.push_back(h.t);
  for (int nd : h.watch) {
    for (int k = 0; k < 3; ++k) h.sampRows.push_back(h.u[nd][k]);
    for (int k = 0; k < 3; ++k) h.sampRows.push_back(h.th[nd][k]);
    for (int k = 0; k < 6; ++k) h.sampRows.push_back(h.v[static_cast<size_t>(nd) * 6 + k]);
  }
  h.sampEn.push_back(h.last);
}

// One explicit step: ExplicitModule::advance (:259-272) + LeapFrogModule::solve
// (LeapFrogModule.cpp:44-84, storing the result) + ExplicitModule::commit (:291-334).
void oneStep(orc_handle_s &h) {
  const int N = h.N;
  // advance: mass update with the current state, then time/step
  assembleMass(h, h.th.data(), h.mT, h.mR);
  for (int nd = 0; nd < N; ++nd)
    if (!(groupMass(h, nd) > DBL_MIN)) h.errword |= DL_EW_MASS;
  h.t += h.dt;
  h.step += 1;
  const double tt = h.t, ii = static_cast<double>(h.step);
  // getForce: GET_EXT_VECTOR, GET_INT_VECTOR (+ gyroscopic term)
  std::fill(h.fext.begin(), h.fext.end(), 0.0);
  for (const Bc &b : h.bcs)
    if (b.kind == DL_BC_NEUMANN) {
      double val = b.factor * evalScale(b, tt, ii, h.dt);
      for (int nd : b.nodes) h.fext[static_cast<size_t>(nd) * 6 + b.dof] += val;
    }
  assembleFint(h, h.u.data(), h.th.data(), h.fint, true);
  h.contactEnergy = 0.0;
  if (h.contact.enabled) contactForces(h, h.fint);
  if (h.jc.enabled) jointForces(h, h.fint);
  if (h.contact.n_plates > 0) plateForces(h, h.fint, tt);
  if (h.gyro)
    for (int nd = 0; nd < N; ++nd) {
      V3 w{{h.v[nd * 6 + 3], h.v[nd * 6 + 4], h.v[nd * 6 + 5]}};
      V3 Mw = mulv(h.mR[nd], w);
      if (!h.madd.empty())  // assembleGyro_ multiplies by the explicit module's matrix, Mass models included
        for (int k = 0; k < 3; ++k) Mw[k] += h.madd[static_cast<size_t>(nd) * 6 + 3 + k] * w[k];
      V3 g = cross(w, Mw);
      for (int k = 0; k < 3; ++k) h.fint[static_cast<size_t>(nd) * 6 + 3 + k] += g[k];
    }
  // getAcce with Dirichlet (acceleration) constraints
  std::vector<double> a(static_cast<size_t>(N) * 6, 0.0);
  std::vector<unsigned> mask(N, 0u);
  for (const Bc &b : h.bcs)
    if (b.kind == DL_BC_DIRICHLET) {
      double val = b.factor * evalScale(b, tt, ii, h.dt);
      for (int nd : b.nodes) {
        a[static_cast<size_t>(nd) * 6 + b.dof] = val;
        mask[nd] |= 1u << b.dof;
      }
    }
  double dwext = 0.0;
  {
    std::vector<double> r(static_cast<size_t>(N) * 6);
    for (size_t k = 0; k < r.size(); ++k) r[k] = h.fext[k] - h.fint[k];
    allAccel(h, r, a, mask);
  }
  // v_new = v + dt a ; u_new = u + dt v_new ; SO(3) update (ExplicitModule::updateVec :362-392)
  for (int nd = 0; nd < N; ++nd) {
    double *v = &h.v[static_cast<size_t>(nd) * 6];
    for (int k = 0; k < 6; ++k) v[k] += h.dt * a[nd * 6 + k];
    for (int k = 0; k < 3; ++k) {
      h.u[nd][k] += h.dt * v[k];
      dwext += h.fext[nd * 6 + k] * h.dt * v[k];
    }
    V3 dr{{h.dt * v[3], h.dt * v[4], h.dt * v[5]}};
    for (int k = 0; k < 3; ++k) dwext += h.fext[nd * 6 + 3 + k] * dr[k];
    if (h.so3) {
      h.th[nd] = logMat(mul(expVec(dr), expVec(h.th[nd])));
    } else {
      for (int k = 0; k < 3; ++k) h.th[nd][k] += dr[k];
    }
    for (int k = 0; k < 6; ++k)
      if (!std::isfinite(v[k])) h.errword |= DL_EW_NONFINITE;
  }
  h.wext += dwext;
  // commit
  applyDeform(h);
  double ep, ed;
  sumEnergies(h, ep, ed);
  h.last.kinetic = kinetic(h);
  h.last.potential = ep;
  h.last.dissipated = ed;
  h.last.external_work = h.wext;
  h.last.contact = h.contactEnergy;
  if (h.every > 0 && h.step % h.every == 0) record(h);
}

// External loads and prescribed accelerations at (t, i) (GET_EXT_VECTOR,
// GET_CONSTRAINTS of the BC models).
void loadsAt(orc_handle_s &h, double tt, double ii, std::vector<double> &a, std::vector<unsigned> &mask) {
  const int N = h.N;
  std::fill(h.fext.begin(), h.fext.end(), 0.0);
  a.assign(static_cast<size_t>(N) * 6, 0.0);
  mask.assign(N, 0u);
  for (const Bc &b : h.bcs) {
    if (b.kind != DL_BC_NEUMANN && b.kind != DL_BC_DIRICHLET) continue;  // initial values act at INIT only
    const double val = b.factor * evalScale(b, tt, ii, h.dt);
    if (b.kind == DL_BC_NEUMANN) {
      for (int nd : b.nodes) h.fext[static_cast<size_t>(nd) * 6 + b.dof] += val;
    } else {
      for (int nd : b.nodes) {
        a[static_cast<size_t>(nd) * 6 + b.dof] = val;
        mask[nd] |= 1u << b.dof;
      }
    }
  }
}

// getForce / updForce at the state (u, th, v) followed by getAcce
// (ExplicitModule.cpp:339-357, 395-419; MilneDeviceModule.cpp:124-140):
// a = M^-1 (fext - fint - w x (M w)) with the prescribed accelerations of the
// constrained DOFs; M is the mass assembled at the step's start.
void accelerations(orc_handle_s &h, const std::vector<V3> &u, const std::vector<V3> &th, const std::vector<double> &v,
                   const std::vector<double> &aPre, const std::vector<unsigned> &mask, std::vector<double> &a) {
  const int N = h.N;
  assembleFint(h, u.data(), th.data(), h.fint, true);
  if (h.gyro)
    for (int nd = 0; nd < N; ++nd) {
      V3 w{{v[nd * 6 + 3], v[nd * 6 + 4], v[nd * 6 + 5]}};
      V3 Mw = mulv(h.mR[nd], w);
      if (!h.madd.empty())  // assembleGyro_ multiplies by the explicit module's matrix, Mass models included
        for (int k = 0; k < 3; ++k) Mw[k] += h.madd[static_cast<size_t>(nd) * 6 + 3 + k] * w[k];
      V3 g = cross(w, Mw);
      for (int k = 0; k < 3; ++k) h.fint[static_cast<size_t>(nd) * 6 + 3 + k] += g[k];
    }
  a = aPre;
  for (int nd = 0; nd < N; ++nd) {
    double r[6];
    for (int k = 0; k < 6; ++k) r[k] = h.fext[nd * 6 + k] - h.fint[nd * 6 + k];
    nodeAccel(h, nd, r, &a[static_cast<size_t>(nd) * 6], mask[nd]);
  }
}

// ExplicitModule::updateVec (:362-392): y = y0 + dy, rotations composed on SO(3)
void updateState(const orc_handle_s &h, const std::vector<V3> &u0, const std::vector<V3> &th0,
                 const std::vector<double> &d, std::vector<V3> &u, std::vector<V3> &th) {
  for (int nd = 0; nd < h.N; ++nd) {
    for (int k = 0; k < 3; ++k) u[nd][k] = u0[nd][k] + h.dt * d[nd * 6 + k];
    V3 dr{{h.dt * d[nd * 6 + 3], h.dt * d[nd * 6 + 4], h.dt * d[nd * 6 + 5]}};
    if (h.so3) {
      th[nd] = logMat(mul(expVec(dr), expVec(th0[nd])));
    } else {
      for (int k = 0; k < 3; ++k) th[nd][k] = th0[nd][k] + dr[k];
    }
  }
}

// ExplicitModule::getQuality (:494-501): RMS over all DOFs of the difference,
// translations (all DOFs without SO(3) rotation DOFs) divided by lengthScale
double quality(const orc_handle_s &h, const double *a, const double *b) {
  double s = 0.0;
  for (int nd = 0; nd < h.N; ++nd)
    for (int k = 0; k < 6; ++k) {
      double d = a[nd * 6 + k] - b[nd * 6 + k];
      if (k < 3 || !h.so3) d /= h.lenScale;
      s += d * d;
    }
  return std::sqrt(s) / std::sqrt(6.0 * h.N);
}

// One attempt of a MilneDevice step: ExplicitModule::advance (:259-272),
// MilneDeviceModule::solve (MilneDeviceModule.cpp:41-118) and
// ExplicitModule::commit (:291-334), or ExplicitModule::cancel (:277-286)
// when the step is rejected.  Returns whether it was accepted.
bool milneAttempt(orc_handle_s &h) {
  const int N = h.N;
  const std::vector<V3> u0 = h.u, th0 = h.th;
  const std::vector<double> v0 = h.v;
  assembleMass(h, h.th.data(), h.mT, h.mR);
  for (int nd = 0; nd < N; ++nd)
    if (!(groupMass(h, nd) > DBL_MIN)) h.errword |= DL_EW_MASS;
  const double t0 = h.t;
  const int64_t step0 = h.step;
  h.t += h.dt;
  h.step += 1;
  std::vector<double> aPre, aCur, aP;
  std::vector<unsigned> mask;
  loadsAt(h, h.t, static_cast<double>(h.step), aPre, mask);
  // predictor: v_pre = v + dt a(u), u_pre = u (+) dt v
  accelerations(h, u0, th0, v0, aPre, mask, aCur);
  std::vector<double> vPre(static_cast<size_t>(N) * 6), vNew(static_cast<size_t>(N) * 6);
  for (size_t i = 0; i < vPre.size(); ++i) vPre[i] = v0[i] + h.dt * aCur[i];
  std::vector<V3> uPre(N), thPre(N), uNew(N), thNew(N);
  updateState(h, u0, th0, v0, uPre, thPre);
  // force at the predicted state (the model sees the stored predictions)
  h.u = uPre;
  h.th = thPre;
  h.v = vPre;
  accelerations(h, uPre, thPre, vPre, aPre, mask, aP);
  // corrector: v_new = v + dt a(u_pre), u_new = u (+) dt v_pre
  for (size_t i = 0; i < vNew.size(); ++i) vNew[i] = v0[i] + h.dt * aP[i];
  updateState(h, u0, th0, vPre, uNew, thNew);
  std::vector<double> yPre(static_cast<size_t>(N) * 6), yNew(static_cast<size_t>(N) * 6);
  for (int nd = 0; nd < N; ++nd)
    for (int k = 0; k < 3; ++k) {
      yPre[nd * 6 + k] = uPre[nd][k];
      yPre[nd * 6 + 3 + k] = thPre[nd][k];
      yNew[nd * 6 + k] = uNew[nd][k];
      yNew[nd * 6 + 3 + k] = thNew[nd][k];
    }
  const double error = 0.5 * (quality(h, yPre.data(), yNew.data()) + quality(h, vPre.data(), vNew.data()) * h.dt);
  const double dtOpt = h.dt * std::pow(h.prec / error, 0.5);  // order 1: exponent 1/(1+1)
  const bool accept = error <= h.prec || h.dt <= h.minDt;
  const double dtUsed = h.dt;
  if (accept) {
    h.dt = std::max(std::max(std::min(std::min(h.safety * dtOpt, h.incrFact * h.dt), h.maxDt), h.decrFact * h.dt),
                    h.minDt);
    h.u = uNew;
    h.th = thNew;
    h.v = vNew;
    for (int nd = 0; nd < N; ++nd) {
      for (int k = 0; k < 6; ++k)
        if (!std::isfinite(vNew[nd * 6 + k])) h.errword |= DL_EW_NONFINITE;
      for (int k = 0; k < 6; ++k) h.wext += h.fext[nd * 6 + k] * dtUsed * vPre[nd * 6 + k];
    }
    applyDeform(h);
    double ep, ed;
    sumEnergies(h, ep, ed);
    h.last.kinetic = kinetic(h);
    h.last.potential = ep;
    h.last.dissipated = ed;
    h.last.external_work = h.wext;
    h.last.contact = 0.0;
    if (h.every > 0 && h.step % h.every == 0) record(h);
  } else {
    h.dt = std::max(std::max(h.safety * dtOpt, h.decrFact * h.dt), h.minDt);
    h.u = u0;
    h.th = th0;
    h.v = v0;
    h.t = t0;
    h.step = step0;
    h.rejected += 1;
  }
  return accept;
}

int fail(const std::string &m, int code = DL_ERR_INVALID) {
  g_err = m;
  return code;
}

}  // namespace

// ---------------------------------------------------------------------------
// C ABI
// ---------------------------------------------------------------------------
ORC_API const char *orc_last_error(void) { return g_err.c_str(); }

ORC_API int orc_set_threads(int n) {
#ifdef _OPENMP
  omp_set_num_threads(n > 0 ? n : 1);
#else
  (void)n;
#endif
  return DL_OK;
}

ORC_API int orc_create(const dl_model_desc *d, orc_handle **out) {
  if (!d || !out) return fail("null argument");
  try {
    auto h = std::make_unique<orc_handle_s>();
    h->N = d->n_nodes;
    h->E = d->n_elems;
    h->nen = d->nodes_per_elem;
    h->G = d->n_gauss > 0 ? d->n_gauss : h->nen - 1;
    if (h->nen < 2 || h->nen > 4) return fail("nodes_per_elem must be 2..4");
    if (h->G < 1 || h->G > 4) return fail("n_gauss must be 1..4");
    h->line.init(h->nen, h->G);
    h->mline.init(h->nen, h->nen);
    h->X0.resize(h->N);
    for (int i = 0; i < h->N; ++i)
      for (int k = 0; k < 3; ++k) h->X0[i][k] = d->coords[i * 3 + k];
    h->conn.assign(d->conn, d->conn + static_cast<size_t>(h->E) * h->nen);
    for (int c : h->conn)
      if (c < 0 || c >= h->N) return fail("connectivity out of range");
    h->rod.resize(h->E);
    for (int e = 0; e < h->E; ++e) h->rod[e] = d->elem_rod ? d->elem_rod[e] : 0;
    // argument names: dof names, h_0 / h_<dof>, then radius/area (extension)
    std::vector<std::string> dofn = {"dx", "dy", "dz", "rx", "ry", "rz"};
    if (d->dof_names)
      for (int k = 0; k < 6; ++k) dofn[k] = d->dof_names[k];
    // materials and plastic laws
    h->lawOf.assign(d->n_materials, -1);
    h->nhMax = 0;
    for (int mi = 0; mi < d->n_materials; ++mi) {
      const dl_material_desc &md = d->materials[mi];
      if (md.type != DL_MAT_ELASTOPLASTIC_ROD) continue;
      PlasticLaw P;
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
      P.nh = nh;
      std::memset(P.H, 0, sizeof P.H);
      if (nh == 1) P.H[0][0] = md.isotropic_coefficient;
      int off = (nh == 7) ? 1 : 0;
      if (nh == 7) P.H[0][0] = md.isotropic_coefficient;
      if (md.kinematic_tensor)
        for (int i = 0; i < 6; ++i)
          for (int j = 0; j < 6; ++j) P.H[off + j][off + i] = md.kinematic_tensor[i * 6 + j];
      if (!md.yield_cond) return fail("elastoplastic material needs yieldCond");
      P.f.parse(md.yield_cond, names);
      if (md.yield_deriv && md.n_yield_deriv > 0) {
        if (md.n_yield_deriv != 6 + nh) return fail("yieldDeriv needs one entry per argument");
        for (int k = 0; k < md.n_yield_deriv; ++k) P.df.emplace_back(md.yield_deriv[k], names);
        P.hasDeriv = true;
      }
      P.maxIter = md.max_iter > 0 ? md.max_iter : 20;
      P.prec = md.precision > 0 ? md.precision : 1e-5;
      h->lawOf[mi] = static_cast<int>(h->laws.size());
      h->laws.push_back(std::move(P));
      h->nhMax = std::max(h->nhMax, nh);
    }
    h->em.resize(h->E);
    for (int e = 0; e < h->E; ++e) {
      int mi = d->elem_mat ? d->elem_mat[e] : 0;
      if (mi < 0 || mi >= d->n_materials) return fail("material index out of range");
      const dl_material_desc &md = d->materials[mi];
      ElemMat &m = h->em[e];
      m.type = md.type;
      m.mat = mi;
      double A = md.area, I1 = md.area_moment[0], I2 = md.area_moment[1], J = md.polar_moment;
      double r = md.radius;
      if (d->elem_radius) {
        if (!md.circle) return fail("per-element radius needs a circular section");
        r = d->elem_radius[e];
        A = M_PI * r * r;
        I1 = I2 = M_PI * std::pow(r, 4) / 4.0;
        J = I1 + I2;
      }
      m.radius = r;
      m.area = A;
      const double G = md.shear_modulus, k = md.shear_correction, Ey = md.young;
      m.C[0] = G * k * A;
      m.C[1] = G * k * A;
      m.C[2] = Ey * A;
      m.C[3] = Ey * I1;
      m.C[4] = Ey * I2;
      m.C[5] = G * J;
      const double ic = md.inertia_correct > 0 ? md.inertia_correct : 1.0;
      m.Mm[0] = m.Mm[1] = m.Mm[2] = md.density * A;
      m.Mm[3] = md.density * I1 * ic;
      m.Mm[4] = md.density * I2 * ic;
      m.Mm[5] = md.density * J * ic;
      m.rhoA = md.density * A;
    }
    // BCs
    for (int b = 0; b < d->n_bcs; ++b) {
      const dl_bc_desc &bd = d->bcs[b];
      if (bd.kind == DL_BC_MASS) {  // MassModel::takeAction(GET_MATRIX2) (MassModel.cpp:77-99)
        if (h->madd.empty()) h->madd.assign(static_cast<size_t>(h->N) * 6, 0.0);
        for (int k = 0; k < bd.n_nodes; ++k) h->madd[static_cast<size_t>(bd.nodes[k]) * 6 + bd.dof] += bd.factor;
        continue;
      }
      Bc bc;
      bc.kind = bd.kind;
      bc.dof = bd.dof;
      bc.factor = bd.factor;
      bc.nodes.assign(bd.nodes, bd.nodes + bd.n_nodes);
      if (bd.scale && bd.scale[0]) {
        bc.scale.parse(bd.scale, {"t", "i", "deltaTime"});
        bc.hasScale = true;
      }
      h->bcs.push_back(std::move(bc));
    }
    h->dt = d->dt;
    h->so3 = d->so3_update != 0;
    h->lumped = d->mass_mode == DL_MASS_LUMPED;
    if (d->n_ties > 0) {
      if (h->lumped) throw std::runtime_error("rigid ties need the consistent mass");
      h->tieMaster.assign(d->n_nodes, -1);
      h->tieSlaves.assign(d->n_nodes, {});
      for (int k = 0; k < d->n_ties; ++k) {
        const int a = d->ties[2 * k], b = d->ties[2 * k + 1];
        if (a < 0 || a >= d->n_nodes || b < 0 || b >= d->n_nodes || a == b || h->tieMaster[b] >= 0)
          throw std::runtime_error("bad tie");
        h->tieMaster[b] = a;
        h->tieSlaves[a].push_back(b);
      }
      for (int n = 0; n < d->n_nodes; ++n)
        if (h->tieMaster[n] >= 0 && !h->tieSlaves[n].empty()) throw std::runtime_error("bad tie chain");
    }
    // the rod model adds the gyroscopic moment only with the consistent
    // matrix (SpecialCosseratRodModel.cpp:351-355)
    h->gyro = d->gyroscopic != 0 && !h->lumped;
    h->contact = d->contact;
    h->jc = d->joint_contact;
    if (h->jc.enabled) {
      if (!(h->jc.radius > 0.0)) return fail("joint contact radius must be positive");
      if (h->jc.n_joints < 0 || (h->jc.n_joints > 0 && !h->jc.joints)) return fail("joint list missing");
      h->joints.assign(h->jc.joints, h->jc.joints + h->jc.n_joints);
      for (int j : h->joints)
        if (j < 0 || j >= h->N) return fail("joint node index out of range");
      h->jc.joints = nullptr;
    }
    // state
    h->u.assign(h->N, V3{{0, 0, 0}});
    h->th.assign(h->N, V3{{0, 0, 0}});
    h->v.assign(static_cast<size_t>(h->N) * 6, 0.0);
    const size_t NG = static_cast<size_t>(h->E) * h->G;
    const int nhs = h->nhMax > 0 ? h->nhMax : 1;
    h->epsOld.assign(NG * 6, 0.0);
    h->epsCur.assign(NG * 6, 0.0);
    h->epOld.assign(NG * 6, 0.0);
    h->epCur.assign(NG * 6, 0.0);
    h->hpOld.assign(NG * nhs, 0.0);
    h->hpCur.assign(NG * nhs, 0.0);
    h->dflow.assign(NG, 0.0);
    h->ediss.assign(NG, 0.0);
    h->epot.assign(NG, 0.0);
    h->fint.assign(static_cast<size_t>(h->N) * 6, 0.0);
    h->fext.assign(static_cast<size_t>(h->N) * 6, 0.0);
    h->mT.assign(h->N, 0.0);
    h->mR.assign(h->N, zero3());
    initRotation(*h, d);
    initStrain(*h);
    // InitLoadModel::init_ (InitLoadModel.cpp:95-137)
    for (const Bc &b : h->bcs) {
      if (b.kind == DL_BC_INIT_DISP)
        for (int nd : b.nodes) {
          if (b.dof < 3) h->u[nd][b.dof] = b.factor;
          else h->th[nd][b.dof - 3] = b.factor;
        }
      if (b.kind == DL_BC_INIT_VELO)
        for (int nd : b.nodes) h->v[static_cast<size_t>(nd) * 6 + b.dof] = b.factor;
    }
    if (!h->tieMaster.empty()) {
      if (!h->madd.empty()) return fail("rigid ties with added point masses are not provided", DL_ERR_UNSUPPORTED);
      // a tie group starts from its master's state
      for (int nd = 0; nd < h->N; ++nd) {
        const int ms = h->tieMaster[nd];
        if (ms < 0) continue;
        h->u[nd] = h->u[ms];
        h->th[nd] = h->th[ms];
        for (int k = 0; k < 6; ++k) h->v[static_cast<size_t>(nd) * 6 + k] = h->v[static_cast<size_t>(ms) * 6 + k];
      }
    }
    assembleMass(*h, h->th.data(), h->mT, h->mR);
    if (h->contact.enabled || h->contact.n_plates > 0) {
      if (h->nen != 2 && h->contact.enabled) return fail("contact needs two-node elements");
      const int R = d->n_rods > 0 ? d->n_rods : 1;
      h->rodElems.assign(R, {});
      h->rodNodes.assign(R, {});
      for (int e = 0; e < h->E; ++e) {
        h->rodElems[h->rod[e]].push_back(e);
        for (int a = 0; a < h->nen; ++a) h->rodNodes[h->rod[e]].push_back(h->conn[e * h->nen + a]);
      }
      for (auto &v : h->rodNodes) {
        std::sort(v.begin(), v.end());
        v.erase(std::unique(v.begin(), v.end()), v.end());
      }
      if (h->contact.enabled) computeBlacklist(*h);
    }
    *out = h.release();
    return DL_OK;
  } catch (const std::exception &ex) {
    return fail(ex.what(), DL_ERR_PARSE);
  }
}

ORC_API int orc_destroy(orc_handle *h) {
  delete h;
  return DL_OK;
}

ORC_API int orc_run(orc_handle *h, int64_t nsteps) {
  if (!h) return fail("null handle");
  try {
    for (int64_t s = 0; s < nsteps; ++s) {
      if (h->integ == DL_INTEG_MILNE) {
        while (!milneAttempt(*h)) {
        }
      } else {
        oneStep(*h);
      }
      if (h->errword & (DL_EW_RETURN_MAP | DL_EW_MASS)) {
        g_err = (h->errword & DL_EW_RETURN_MAP) ? "Too many iterations in plasticity loop"
                                                : "Zero (or negative) masses cannot be inversed!";
        return (h->errword & DL_EW_RETURN_MAP) ? DL_ERR_RETURN_MAP : DL_ERR_MASS;
      }
    }
  } catch (const std::exception &ex) {
    return fail(ex.what());
  }
  return DL_OK;
}

ORC_API int orc_set_integrator(orc_handle *h, const dl_integrator_desc *d) {
  if (!h || !d) return fail("null argument");
  if (d->kind != DL_INTEG_LEAPFROG && d->kind != DL_INTEG_MILNE) return fail("unknown integrator");
  if (d->kind == DL_INTEG_MILNE) {
    if (!(d->precision > 0.0)) return fail("MilneDevice needs precision > 0");
    if (h->contact.enabled || h->contact.n_plates > 0 || h->jc.enabled)
      return fail("MilneDevice runs without contact", DL_ERR_UNSUPPORTED);
    if (!h->madd.empty()) return fail("MilneDevice runs without added masses", DL_ERR_UNSUPPORTED);
    if (!h->tieMaster.empty()) return fail("MilneDevice runs without rigid ties", DL_ERR_UNSUPPORTED);
  }
  h->integ = d->kind;
  h->prec = d->precision;
  h->minDt = d->min_dt > 0.0 ? d->min_dt : h->dt / 100.0;
  h->maxDt = d->max_dt > 0.0 ? d->max_dt : h->dt * 100.0;
  h->safety = d->safety > 0.0 ? d->safety : 0.9;
  h->incrFact = d->increase > 0.0 ? d->increase : 1.2;
  h->decrFact = d->decrease > 0.0 ? d->decrease : 0.8;
  h->lenScale = d->length_scale > 0.0 ? d->length_scale : 1e-3;
  return DL_OK;
}

ORC_API int orc_get_time(orc_handle *h, double *t, double *dt, int64_t *step, int64_t *rejected) {
  if (!h) return fail("null handle");
  if (t) *t = h->t;
  if (dt) *dt = h->dt;
  if (step) *step = h->step;
  if (rejected) *rejected = h->rejected;
  return DL_OK;
}

ORC_API int orc_get_sample_times(orc_handle *h, double *times, int64_t max_samples) {
  if (!h || !times) return fail("null argument");
  const int64_t n = std::min<int64_t>(max_samples, static_cast<int64_t>(h->sampTimes.size()));
  for (int64_t i = 0; i < n; ++i) times[i] = h->sampTimes[i];
  return DL_OK;
}

ORC_API int orc_set_sampling(orc_handle *h, int32_t every, int32_t n_watch, const int32_t *watch_nodes) {
  if (!h) return fail("null handle");
  h->every = every;
  h->watch.assign(watch_nodes, watch_nodes + n_watch);
  h->sampSteps.clear();
  h->sampTimes.clear();
  h->sampRows.clear();
  h->sampEn.clear();
  return DL_OK;
}

ORC_API int orc_get_samples(orc_handle *h, int64_t *n_samples, int64_t *steps, double *node_rows,
                            dl_energies *energies, int64_t max_samples) {
  if (!h) return fail("null handle");
  const int64_t n = static_cast<int64_t>(h->sampSteps.size());
  if (n_samples) *n_samples = n;
  const int64_t m = std::min(n, max_samples);
  const size_t per = h->watch.size() * 12;
  for (int64_t s = 0; s < m; ++s) {
    if (steps) steps[s] = h->sampSteps[s];
    if (node_rows) std::memcpy(node_rows + s * per, &h->sampRows[s * per], per * sizeof(double));
    if (energies) energies[s] = h->sampEn[s];
  }
  return DL_OK;
}

ORC_API int orc_get_state(orc_handle *h, double *u, double *theta, double *v) {
  if (!h) return fail("null handle");
  for (int i = 0; i < h->N; ++i)
    for (int k = 0; k < 3; ++k) {
      if (u) u[i * 3 + k] = h->u[i][k];
      if (theta) theta[i * 3 + k] = h->th[i][k];
    }
  if (v) std::memcpy(v, h->v.data(), h->v.size() * sizeof(double));
  return DL_OK;
}

ORC_API int orc_set_state(orc_handle *h, const double *u, const double *theta, const double *v) {
  if (!h) return fail("null handle");
  for (int i = 0; i < h->N; ++i)
    for (int k = 0; k < 3; ++k) {
      if (u) h->u[i][k] = u[i * 3 + k];
      if (theta) h->th[i][k] = theta[i * 3 + k];
    }
  if (v) std::memcpy(h->v.data(), v, h->v.size() * sizeof(double));
  return DL_OK;
}

ORC_API int orc_get_energies(orc_handle *h, dl_energies *e) {
  if (!h || !e) return fail("null argument");
  *e = h->last;
  return DL_OK;
}

ORC_API int orc_internal_force(orc_handle *h, const double *u, const double *theta, double *fint) {
  if (!h || !u || !theta || !fint) return fail("null argument");
  std::vector<V3> uu(h->N), tt(h->N);
  for (int i = 0; i < h->N; ++i)
    for (int k = 0; k < 3; ++k) {
      uu[i][k] = u[i * 3 + k];
      tt[i][k] = theta[i * 3 + k];
    }
  std::vector<double> f(static_cast<size_t>(h->N) * 6);
  // "output"-style evaluation: no return-map iteration, history untouched
  auto saveCur = h->epsCur;
  auto saveEp = h->epCur;
  auto saveHp = h->hpCur;
  auto saveDf = h->dflow;
  assembleFint(*h, uu.data(), tt.data(), f, false);
  h->epsCur = saveCur;
  h->epCur = saveEp;
  h->hpCur = saveHp;
  h->dflow = saveDf;
  std::memcpy(fint, f.data(), f.size() * sizeof(double));
  return DL_OK;
}

// Internal force of a static load step's Newton iteration at (u, theta):
// GET_INT_VECTOR with the return map run from the committed history
// (ElastoPlasticRodMaterial::getStress, ElastoPlasticRodMaterial.cpp:198-269,
// inelastic = true) and the rod-rod contact forces of that configuration
// (RodContactModel GET_INT_VECTOR, RodContactModel.cpp:699-738); the history
// and the committed state are left as they were.  Used by the tests' static
// equilibrium driver (the reference runs its plastic and contact benchmarks
// with JIVE's Nonlin solver).
ORC_API int orc_static_force(orc_handle *h, const double *u, const double *theta, double *fint) {
  if (!h || !u || !theta || !fint) return fail("null argument");
  std::vector<V3> uu(h->N), tt(h->N);
  for (int i = 0; i < h->N; ++i)
    for (int k = 0; k < 3; ++k) {
      uu[i][k] = u[i * 3 + k];
      tt[i][k] = theta[i * 3 + k];
    }
  std::vector<double> f(static_cast<size_t>(h->N) * 6);
  auto saveCur = h->epsCur;
  auto saveEp = h->epCur;
  auto saveHp = h->hpCur;
  auto saveDf = h->dflow;
  const uint32_t saveErr = h->errword;
  assembleFint(*h, uu.data(), tt.data(), f, true);
  if (h->contact.enabled || h->jc.enabled) {
    std::swap(h->u, uu);
    std::swap(h->th, tt);
    const double saveEc = h->contactEnergy;
    if (h->contact.enabled) contactForces(*h, f);
    if (h->jc.enabled) jointForces(*h, f);
    h->contactEnergy = saveEc;
    std::swap(h->u, uu);
    std::swap(h->th, tt);
  }
  const bool iterFail = (h->errword & DL_EW_RETURN_MAP) && !(saveErr & DL_EW_RETURN_MAP);
  h->epsCur = saveCur;
  h->epCur = saveEp;
  h->hpCur = saveHp;
  h->dflow = saveDf;
  h->errword = saveErr;
  std::memcpy(fint, f.data(), f.size() * sizeof(double));
  return iterFail ? fail("return map did not converge (maxIter)") : DL_OK;
}

// Commit of a converged static load step at (u, theta): the state becomes
// (u, theta) with zero velocity, the return map runs from the committed
// history and its result is committed (ElastoPlasticRodMaterial::applyDeform,
// ElastoPlasticRodMaterial.cpp:271-307); energies are summed as at a COMMIT.
ORC_API int orc_static_commit(orc_handle *h, const double *u, const double *theta) {
  if (!h || !u || !theta) return fail("null argument");
  for (int i = 0; i < h->N; ++i)
    for (int k = 0; k < 3; ++k) {
      h->u[i][k] = u[i * 3 + k];
      h->th[i][k] = theta[i * 3 + k];
    }
  std::fill(h->v.begin(), h->v.end(), 0.0);
  assembleFint(*h, h->u.data(), h->th.data(), h->fint, true);
  h->contactEnergy = 0.0;
  if (h->contact.enabled) contactForces(*h, h->fint);
  if (h->jc.enabled) jointForces(*h, h->fint);
  applyDeform(*h);
  double ep, ed;
  sumEnergies(*h, ep, ed);
  h->step += 1;
  h->last.kinetic = 0.0;
  h->last.potential = ep;
  h->last.dissipated = ed;
  h->last.contact = h->contactEnergy;
  return (h->errword & DL_EW_RETURN_MAP) ? fail("return map did not converge (maxIter)") : DL_OK;
}

ORC_API int orc_elastic_energy(orc_handle *h, const double *u, const double *theta, double *energy) {
  if (!h || !u || !theta || !energy) return fail("null argument");
  std::vector<V3> uu(h->N), tt(h->N);
  for (int i = 0; i < h->N; ++i)
    for (int k = 0; k < 3; ++k) {
      uu[i][k] = u[i * 3 + k];
      tt[i][k] = theta[i * 3 + k];
    }
  double E = 0.0;
  for (int e = 0; e < h->E; ++e) {
    ElemCtx c;
    getDisplacements(*h, e, uu.data(), tt.data(), c);
    double s[4][6];
    getStrains(*h, e, c, s, true);
    double w[4];
    h->line.weightsGrads(c.X0, w, nullptr);
    for (int q = 0; q < h->G; ++q) {
      const size_t gi = static_cast<size_t>(e) * h->G + q;
      double acc = 0.0;
      for (int k = 0; k < 6; ++k) {
        double el = s[q][k] - h->epOld[gi * 6 + k];
        acc += el * h->em[e].C[k] * el;
      }
      E += w[q] * 0.5 * acc;
    }
  }
  *energy = E;
  return DL_OK;
}

ORC_API int orc_get_history(orc_handle *h, double *plastic_strain, double *hard_params, double *dissipation) {
  if (!h) return fail("null handle");
  const size_t NG = static_cast<size_t>(h->E) * h->G;
  if (plastic_strain) std::memcpy(plastic_strain, h->epOld.data(), NG * 6 * sizeof(double));
  if (hard_params) {
    const int nhs = h->nhMax > 0 ? h->nhMax : 1;
    for (size_t g = 0; g < NG; ++g)
      for (int k = 0; k < 7; ++k) hard_params[g * 7 + k] = (k < h->nhMax) ? h->hpOld[g * nhs + k] : 0.0;
  }
  if (dissipation) std::memcpy(dissipation, h->ediss.data(), NG * sizeof(double));
  return DL_OK;
}

ORC_API int orc_get_frames(orc_handle *h, double *lambda_n, double *strain0) {
  if (!h) return fail("null handle");
  if (lambda_n)
    for (size_t i = 0; i < h->LN.size(); ++i)
      for (int a = 0; a < 3; ++a)
        for (int b = 0; b < 3; ++b) lambda_n[i * 9 + a * 3 + b] = h->LN[i].a[a][b];
  if (strain0) std::memcpy(strain0, h->strain0.data(), h->strain0.size() * sizeof(double));
  return DL_OK;
}

ORC_API int orc_mass(orc_handle *h, const double *theta, double *m_trans, double *m_rot) {
  if (!h) return fail("null handle");
  std::vector<V3> tt(h->N);
  for (int i = 0; i < h->N; ++i)
    for (int k = 0; k < 3; ++k) tt[i][k] = theta ? theta[i * 3 + k] : h->th[i][k];
  std::vector<double> mT(h->N);
  std::vector<M3> mR(h->N);
  assembleMass(*h, tt.data(), mT, mR);
  for (int i = 0; i < h->N; ++i) {
    if (m_trans) m_trans[i] = mT[i];
    if (m_rot)
      for (int a = 0; a < 3; ++a)
        for (int b = 0; b < 3; ++b) m_rot[i * 9 + a * 3 + b] = mR[i].a[a][b];
  }
  return DL_OK;
}

ORC_API int orc_error_word(orc_handle *h, uint32_t *word) {
  if (!h || !word) return fail("null argument");
  *word = h->errword;
  return DL_OK;
}

ORC_API int orc_contact_pairs(orc_handle *h, int64_t *n_pairs, int32_t *pairs, double *gaps, int64_t max_pairs) {
  if (!h) return fail("null handle");
  const int64_t n = static_cast<int64_t>(h->closedPairs.size());
  if (n_pairs) *n_pairs = n;
  for (int64_t i = 0; i < std::min(n, max_pairs); ++i) {
    if (pairs) {
      pairs[2 * i] = h->closedPairs[i].first;
      pairs[2 * i + 1] = h->closedPairs[i].second;
    }
    if (gaps) gaps[i] = h->closedGaps[i];
  }
  return DL_OK;
}

ORC_API int orc_joint_contact_pairs(orc_handle *h, int64_t *n_pairs, int32_t *pairs, double *gaps,
                                    int64_t max_pairs) {
  if (!h) return fail("null handle");
  std::vector<size_t> ord(h->closedJointPairs.size());
  for (size_t i = 0; i < ord.size(); ++i) ord[i] = i;
  std::sort(ord.begin(), ord.end(),
            [&](size_t a, size_t b) { return h->closedJointPairs[a] < h->closedJointPairs[b]; });
  const int64_t n = static_cast<int64_t>(ord.size());
  if (n_pairs) *n_pairs = n;
  for (int64_t i = 0; i < std::min(n, max_pairs); ++i) {
    if (pairs) {
      pairs[2 * i] = h->closedJointPairs[ord[i]].first;
      pairs[2 * i + 1] = h->closedJointPairs[ord[i]].second;
    }
    if (gaps) gaps[i] = h->closedJointGaps[ord[i]];
  }
  return DL_OK;
}

// Element tables of GET_TABLE as ParaViewModule writes them (SpecialCosseratRodModel
// getStrainTable_/getStressTable_ :426-532 with getStrains_/getStresses_ :694-771;
// ElastoPlasticRodMaterial::getTable "plast_strain" :318-340; ParaViewModule.cpp:
// 585-616): per element the sum over its Gauss points, scaled by the point
// count (the accumulated weights, applied by scaleRows without inversion).
// The stress is the output load case's: C (eps - eps_p) with the committed
// plastic strain, no return map (ElastoPlasticRodMaterial.cpp:217-224).
ORC_API int orc_element_table(orc_handle *h, const char *name, double *out) {
  if (!h || !name || !out) return fail("null argument");
  const std::string nm(name);
  int kind = 0;
  bool spatial = false;
  if (nm == "strain") spatial = true;
  else if (nm == "mat_strain") kind = 0;
  else if (nm == "stress") kind = 1, spatial = true;
  else if (nm == "mat_stress") kind = 1;
  else if (nm == "plast_strain") kind = 2;
  else return fail("unknown element table " + nm);
  for (int e = 0; e < h->E; ++e) {
    ElemCtx c;
    getDisplacements(*h, e, h->u.data(), h->th.data(), c);
    double strain[4][6];
    getStrains(*h, e, c, strain, true);
    M3 Ri[4];
    h->line.rotations(c.Rn, Ri);
    const ElemMat &em = h->em[e];
    const bool plastic = em.type == DL_MAT_ELASTOPLASTIC_ROD && h->lawOf[em.mat] >= 0;
    double acc[6] = {0, 0, 0, 0, 0, 0};
    for (int q = 0; q < h->G; ++q) {
      const size_t gi = static_cast<size_t>(e) * h->G + q;
      double val[6];
      for (int k = 0; k < 6; ++k) {
        const double ep = plastic ? h->epOld[gi * 6 + k] : 0.0;
        val[k] = kind == 0 ? strain[q][k] : (kind == 1 ? em.C[k] * (strain[q][k] - ep) : ep);
      }
      if (spatial) {
        const V3 a = mulv(Ri[q], V3{{val[0], val[1], val[2]}}), b = mulv(Ri[q], V3{{val[3], val[4], val[5]}});
        for (int k = 0; k < 3; ++k) {
          val[k] = a[k];
          val[k + 3] = b[k];
        }
      }
      for (int k = 0; k < 6; ++k) acc[k] += val[k];
    }
    for (int k = 0; k < 6; ++k) out[static_cast<size_t>(e) * 6 + k] = acc[k] * h->G;
  }
  return DL_OK;
}

ORC_API int orc_blacklist_size(orc_handle *h, int64_t *n) {
  if (!h || !n) return fail("null argument");
  *n = static_cast<int64_t>(h->blacklist.size());
  return DL_OK;
}

ORC_API int orc_plate_reaction(orc_handle *h, double *out) {
  if (!h || !out) return fail("null argument");
  for (size_t i = 0; i < h->plateReaction.size(); ++i) out[i] = h->plateReaction[i];
  return DL_OK;
}

ORC_API int orc_group_sums(orc_handle *h, int32_t n_nodes, const int32_t *nodes, double *out_resp,
                           double *out_load) {
  if (!h) return fail("null handle");
  for (int k = 0; k < 6; ++k) {
    double r = 0.0, l = 0.0;
    for (int i = 0; i < n_nodes; ++i) {
      r += h->fint[static_cast<size_t>(nodes[i]) * 6 + k];
      l += h->fext[static_cast<size_t>(nodes[i]) * 6 + k];
    }
    if (out_resp) out_resp[k] = r;
    if (out_load) out_load[k] = l;
  }
  return DL_OK;
}
