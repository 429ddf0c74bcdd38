// Expression compiler of the engine.
//
// dynLattice passes user expression strings to JEM's FuncUtils: yield
// functions and their derivatives (ElastoPlasticRodMaterial.cpp:132-143,
// helpers.cpp:11-35), LoadScale "scaleFunc", conditions such as
// control.runWhile.  The engine parses the same language, evaluates it on the
// host in double (time functions, tabulated per step), and compiles yield
// functions into a straight-line register program that the element kernel
// interprets on the device.  Programs are in SSA form with common
// subexpressions shared, then register-allocated by liveness.
#pragma once
#include <cstdint>
#include <map>
#include <memory>
#include <string>
#include <vector>

#include "devtypes.cuh"

namespace dl {

struct ExprProgram {
  std::vector<ExprOp> ops;
  std::vector<double> consts;
  std::vector<uint8_t> outputs;  // register holding each output
  int n_regs = 0;
};

struct ExprNode;
using ExprPtr = std::shared_ptr<const ExprNode>;
struct ExprNode {
  enum Kind { NUM, VAR, UN, BIN, CALL } kind;
  double num = 0.0;
  int var = -1;
  std::string op;
  std::vector<ExprPtr> kids;
};

// Parse `src` with variables `names`; throws std::runtime_error on error.
ExprPtr parseExpr(const std::string &src, const std::vector<std::string> &names);
double evalExpr(const ExprNode *n, const double *vars);

// Compile several expressions over the same argument vector into one program.
ExprProgram compileExprs(const std::vector<ExprPtr> &exprs);
// Host interpreter of a compiled program (reference for the device one).
void runProgram(const ExprProgram &p, const double *args, double *out);

// CUDA source of the yield-function policy `YieldJit` for the step kernels:
// straight-line code (common subexpressions shared) for f(args) and for the
// gradient list, in float (fp32) or double.
std::string emitYieldPolicy(const ExprPtr &f, const std::vector<ExprPtr> &grads, bool fp32);

// Source of the policy `YieldAdj` of the adjoint kernels: f and the gradient
// list as above plus vjp(a, lf, lg, la), the reverse-mode product
// la += (df/da)^T lf + sum_k (dg_k/da)^T lg[k], generated instruction by
// instruction from the same SSA code.  `qual` qualifies the member functions
// ("__device__" for the runtime compiler, "" or "inline" for host builds).
std::string emitYieldAdjPolicy(const ExprPtr &f, const std::vector<ExprPtr> &grads, bool fp32,
                               const std::string &qual);

}  // namespace dl
