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

namespace dl {

enum ExprOpCode : uint8_t {
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

}  // namespace dl
