// Expression parser / compiler of the engine (see expr.hpp).
#include "expr.hpp"

#include <cctype>
#include <cstdio>
#include <cmath>
#include <functional>
#include <stdexcept>
#include <unordered_map>

namespace dl {

namespace {

class Parser {
 public:
  Parser(const std::string &s, const std::vector<std::string> &names) : s_(s), names_(names) {}
  ExprPtr parse() {
    ExprPtr e = orExpr();
    ws();
    if (p_ != s_.size()) throw std::runtime_error("unexpected '" + s_.substr(p_) + "' in expression: " + s_);
    return e;
  }

 private:
  const std::string &s_;
  const std::vector<std::string> &names_;
  size_t p_ = 0;

  void ws() {
    while (p_ < s_.size() && std::isspace(static_cast<unsigned char>(s_[p_]))) ++p_;
  }
  bool eat(const char *t) {
    ws();
    const size_t n = std::char_traits<char>::length(t);
    if (s_.compare(p_, n, t) == 0) {
      p_ += n;
      return true;
    }
    return false;
  }
  static ExprPtr mk(ExprNode::Kind k, const std::string &op, std::vector<ExprPtr> kids) {
    auto n = std::make_shared<ExprNode>();
    n->kind = k;
    n->op = op;
    n->kids = std::move(kids);
    return n;
  }
  ExprPtr orExpr() {
    ExprPtr a = andExpr();
    while (eat("||")) a = mk(ExprNode::BIN, "||", {a, andExpr()});
    return a;
  }
  ExprPtr andExpr() {
    ExprPtr a = cmpExpr();
    while (eat("&&")) a = mk(ExprNode::BIN, "&&", {a, cmpExpr()});
    return a;
  }
  ExprPtr cmpExpr() {
    ExprPtr a = addExpr();
    for (;;) {
      const char *ops[] = {"<=", ">=", "==", "!=", "<", ">"};
      bool hit = false;
      for (const char *o : ops)
        if (eat(o)) {
          a = mk(ExprNode::BIN, o, {a, addExpr()});
          hit = true;
          break;
        }
      if (!hit) return a;
    }
  }
  ExprPtr addExpr() {
    ExprPtr a = mulExpr();
    for (;;) {
      if (eat("+")) a = mk(ExprNode::BIN, "+", {a, mulExpr()});
      else if (eat("-")) a = mk(ExprNode::BIN, "-", {a, mulExpr()});
      else return a;
    }
  }
  ExprPtr mulExpr() {
    ExprPtr a = unary();
    for (;;) {
      if (eat("*")) a = mk(ExprNode::BIN, "*", {a, unary()});
      else if (eat("/")) a = mk(ExprNode::BIN, "/", {a, unary()});
      else if (eat("%")) a = mk(ExprNode::BIN, "%", {a, unary()});
      else return a;
    }
  }
  ExprPtr unary() {
    if (eat("-")) return mk(ExprNode::UN, "-", {unary()});
    if (eat("+")) return unary();
    ws();
    if (p_ < s_.size() && s_[p_] == '!' && (p_ + 1 >= s_.size() || s_[p_ + 1] != '=')) {
      ++p_;
      return mk(ExprNode::UN, "!", {unary()});
    }
    ExprPtr a = atom();
    if (eat("^")) return mk(ExprNode::BIN, "^", {a, unary()});
    return a;
  }
  ExprPtr atom() {
    ws();
    if (p_ >= s_.size()) throw std::runtime_error("unexpected end of expression: " + s_);
    const char c = s_[p_];
    if (c == '(') {
      ++p_;
      ExprPtr a = orExpr();
      if (!eat(")")) throw std::runtime_error("missing ')' in expression: " + s_);
      return a;
    }
    if (std::isdigit(static_cast<unsigned char>(c)) || c == '.') {
      size_t q = p_;
      while (q < s_.size() && (std::isdigit(static_cast<unsigned char>(s_[q])) || s_[q] == '.')) ++q;
      if (q < s_.size() && (s_[q] == 'e' || s_[q] == 'E')) {
        size_t r = q + 1;
        if (r < s_.size() && (s_[r] == '+' || s_[r] == '-')) ++r;
        if (r < s_.size() && std::isdigit(static_cast<unsigned char>(s_[r]))) {
          q = r;
          while (q < s_.size() && std::isdigit(static_cast<unsigned char>(s_[q]))) ++q;
        }
      }
      auto n = std::make_shared<ExprNode>();
      n->kind = ExprNode::NUM;
      n->num = std::stod(s_.substr(p_, q - p_));
      p_ = q;
      return n;
    }
    if (std::isalpha(static_cast<unsigned char>(c)) || c == '_') {
      size_t q = p_;
      while (q < s_.size() &&
             (std::isalnum(static_cast<unsigned char>(s_[q])) || s_[q] == '_' || s_[q] == '.'))
        ++q;
      const std::string id = s_.substr(p_, q - p_);
      p_ = q;
      ws();
      if (p_ < s_.size() && s_[p_] == '(') {
        ++p_;
        std::vector<ExprPtr> args;
        if (!eat(")")) {
          for (;;) {
            args.push_back(orExpr());
            if (eat(")")) break;
            if (!eat(",")) throw std::runtime_error("expected ',' in call of " + id + ": " + s_);
          }
        }
        return mk(ExprNode::CALL, id, args);
      }
      auto n = std::make_shared<ExprNode>();
      if (id == "PI") {
        n->kind = ExprNode::NUM;
        n->num = M_PI;
        return n;
      }
      for (size_t i = 0; i < names_.size(); ++i)
        if (names_[i] == id) {
          n->kind = ExprNode::VAR;
          n->var = static_cast<int>(i);
          return n;
        }
      throw std::runtime_error("unknown variable '" + id + "' in expression: " + s_);
    }
    throw std::runtime_error(std::string("unexpected character '") + c + "' in expression: " + s_);
  }
};

const std::unordered_map<std::string, ExprOpCode> &binOps() {
  static const std::unordered_map<std::string, ExprOpCode> m = {
      {"+", XO_ADD}, {"-", XO_SUB}, {"*", XO_MUL}, {"/", XO_DIV}, {"^", XO_POW}, {"%", XO_MOD},
      {"<", XO_LT}, {"<=", XO_LE}, {">", XO_GT}, {">=", XO_GE}, {"==", XO_EQ}, {"!=", XO_NE},
      {"&&", XO_AND}, {"||", XO_OR}};
  return m;
}
const std::unordered_map<std::string, ExprOpCode> &unFuncs() {
  static const std::unordered_map<std::string, ExprOpCode> m = {
      {"abs", XO_ABS}, {"sqrt", XO_SQRT}, {"exp", XO_EXP}, {"log", XO_LOG}, {"sin", XO_SIN},
      {"cos", XO_COS}, {"tan", XO_TAN}, {"atan", XO_ATAN}, {"floor", XO_FLOOR},
      {"ceil", XO_CEIL}, {"sign", XO_SIGN}};
  return m;
}

double applyOp(int op, double a, double b, double c) {
  switch (op) {
    case XO_ADD: return a + b;
    case XO_SUB: return a - b;
    case XO_MUL: return a * b;
    case XO_DIV: return a / b;
    case XO_POW: return std::pow(a, b);
    case XO_SQUARE: return a * a;
    case XO_NEG: return -a;
    case XO_ABS: return std::fabs(a);
    case XO_SQRT: return std::sqrt(a);
    case XO_EXP: return std::exp(a);
    case XO_LOG: return std::log(a);
    case XO_SIN: return std::sin(a);
    case XO_COS: return std::cos(a);
    case XO_TAN: return std::tan(a);
    case XO_ATAN: return std::atan(a);
    case XO_FLOOR: return std::floor(a);
    case XO_CEIL: return std::ceil(a);
    case XO_SIGN: return static_cast<double>((a > 0.0) - (a < 0.0));
    case XO_MIN: return a < b ? a : b;
    case XO_MAX: return a > b ? a : b;
    case XO_MOD: return std::fmod(a, b);
    case XO_LT: return a < b;
    case XO_LE: return a <= b;
    case XO_GT: return a > b;
    case XO_GE: return a >= b;
    case XO_EQ: return a == b;
    case XO_NE: return a != b;
    case XO_AND: return (a != 0.0 && b != 0.0) ? 1.0 : 0.0;
    case XO_OR: return (a != 0.0 || b != 0.0) ? 1.0 : 0.0;
    case XO_NOT: return a == 0.0 ? 1.0 : 0.0;
    case XO_SELECT: return a != 0.0 ? b : c;
    default: throw std::runtime_error("bad opcode");
  }
}

// SSA builder with structural hashing (common subexpressions shared)
struct SsaInst {
  int op;
  int a = -1, b = -1, c = -1;
  double k = 0.0;
};

struct Builder {
  std::vector<SsaInst> code;
  std::map<std::tuple<int, int, int, int, double>, int> memo;

  int emit(int op, int a = -1, int b = -1, int c = -1, double k = 0.0) {
    auto key = std::make_tuple(op, a, b, c, k);
    auto it = memo.find(key);
    if (it != memo.end()) return it->second;
    // constant folding
    auto isConst = [&](int r) { return r >= 0 && code[r].op == XO_CONST; };
    if (op != XO_CONST && op != XO_ARG && (a < 0 || isConst(a)) && (b < 0 || isConst(b)) &&
        (c < 0 || isConst(c))) {
      double va = a >= 0 ? code[a].k : 0.0, vb = b >= 0 ? code[b].k : 0.0, vc = c >= 0 ? code[c].k : 0.0;
      return emit(XO_CONST, -1, -1, -1, applyOp(op, va, vb, vc));
    }
    SsaInst in;
    in.op = op;
    in.a = a;
    in.b = b;
    in.c = c;
    in.k = k;
    code.push_back(in);
    int id = static_cast<int>(code.size()) - 1;
    memo[key] = id;
    return id;
  }

  int build(const ExprNode *n) {
    switch (n->kind) {
      case ExprNode::NUM: return emit(XO_CONST, -1, -1, -1, n->num);
      case ExprNode::VAR: return emit(XO_ARG, n->var);
      case ExprNode::UN: {
        int a = build(n->kids[0].get());
        return emit(n->op == "-" ? XO_NEG : XO_NOT, a);
      }
      case ExprNode::BIN: {
        int a = build(n->kids[0].get());
        int b = build(n->kids[1].get());
        int op = binOps().at(n->op);
        if (op == XO_POW && code[b].op == XO_CONST && code[b].k == 2.0) return emit(XO_SQUARE, a);
        return emit(op, a, b);
      }
      case ExprNode::CALL: {
        const std::string &f = n->op;
        if (f == "if") {
          if (n->kids.size() != 3) throw std::runtime_error("if() takes three arguments");
          int c = build(n->kids[0].get()), x = build(n->kids[1].get()), y = build(n->kids[2].get());
          return emit(XO_SELECT, c, x, y);
        }
        auto u = unFuncs().find(f);
        if (u != unFuncs().end()) {
          if (n->kids.size() != 1) throw std::runtime_error(f + "() takes one argument");
          return emit(u->second, build(n->kids[0].get()));
        }
        if (f == "pow") {
          if (n->kids.size() != 2) throw std::runtime_error("pow() takes two arguments");
          return emit(XO_POW, build(n->kids[0].get()), build(n->kids[1].get()));
        }
        if (f == "min" || f == "max") {
          if (n->kids.empty()) throw std::runtime_error(f + "() needs arguments");
          int r = build(n->kids[0].get());
          for (size_t i = 1; i < n->kids.size(); ++i)
            r = emit(f == "min" ? XO_MIN : XO_MAX, r, build(n->kids[i].get()));
          return r;
        }
        throw std::runtime_error("unknown function " + f + "()");
      }
    }
    throw std::runtime_error("bad expression node");
  }
};

}  // namespace

ExprPtr parseExpr(const std::string &src, const std::vector<std::string> &names) {
  Parser p(src, names);
  return p.parse();
}

double evalExpr(const ExprNode *n, const double *v) {
  switch (n->kind) {
    case ExprNode::NUM: return n->num;
    case ExprNode::VAR: return v[n->var];
    case ExprNode::UN: {
      double a = evalExpr(n->kids[0].get(), v);
      return n->op == "-" ? -a : (a == 0.0 ? 1.0 : 0.0);
    }
    case ExprNode::BIN: {
      double a = evalExpr(n->kids[0].get(), v);
      if (n->op == "&&") return (a != 0.0 && evalExpr(n->kids[1].get(), v) != 0.0) ? 1.0 : 0.0;
      if (n->op == "||") return (a != 0.0 || evalExpr(n->kids[1].get(), v) != 0.0) ? 1.0 : 0.0;
      double b = evalExpr(n->kids[1].get(), v);
      return applyOp(binOps().at(n->op), a, b, 0.0);
    }
    case ExprNode::CALL: {
      const std::string &f = n->op;
      if (f == "if") {
        if (n->kids.size() != 3) throw std::runtime_error("if() takes three arguments");
        return evalExpr(n->kids[0].get(), v) != 0.0 ? evalExpr(n->kids[1].get(), v)
                                                    : evalExpr(n->kids[2].get(), v);
      }
      std::vector<double> a;
      for (auto &k : n->kids) a.push_back(evalExpr(k.get(), v));
      auto u = unFuncs().find(f);
      if (u != unFuncs().end()) {
        if (a.size() != 1) throw std::runtime_error(f + "() takes one argument");
        return applyOp(u->second, a[0], 0.0, 0.0);
      }
      if (f == "pow") {
        if (a.size() != 2) throw std::runtime_error("pow() takes two arguments");
        return std::pow(a[0], a[1]);
      }
      if (f == "min" || f == "max") {
        if (a.empty()) throw std::runtime_error(f + "() needs arguments");
        double r = a[0];
        for (double x : a) r = (f == "min") ? (x < r ? x : r) : (x > r ? x : r);
        return r;
      }
      throw std::runtime_error("unknown function " + f + "()");
    }
  }
  throw std::runtime_error("bad expression node");
}

ExprProgram compileExprs(const std::vector<ExprPtr> &exprs) {
  Builder b;
  std::vector<int> outs;
  for (auto &e : exprs) outs.push_back(b.build(e.get()));
  // liveness: last use of every SSA value
  const int n = static_cast<int>(b.code.size());
  std::vector<int> lastUse(n, -1);
  for (int i = 0; i < n; ++i) {
    const SsaInst &in = b.code[i];
    for (int r : {in.a, in.b, in.c})
      if (r >= 0 && in.op != XO_ARG) lastUse[r] = i;
  }
  for (int o : outs) lastUse[o] = n;  // outputs live to the end
  // linear-scan register allocation
  ExprProgram p;
  std::vector<int> regOf(n, -1);
  std::vector<int> freeRegs;
  int nregs = 0;
  for (int i = 0; i < n; ++i) {
    const SsaInst &in = b.code[i];
    if (lastUse[i] < 0) continue;  // dead value
    ExprOp op{};
    op.op = static_cast<uint8_t>(in.op);
    if (in.op == XO_CONST) {
      int ci = static_cast<int>(p.consts.size());
      p.consts.push_back(in.k);
      op.a = static_cast<uint8_t>(ci & 0xff);
      op.b = static_cast<uint8_t>((ci >> 8) & 0xff);
    } else if (in.op == XO_ARG) {
      op.a = static_cast<uint8_t>(in.a);
    } else {
      op.a = static_cast<uint8_t>(in.a >= 0 ? regOf[in.a] : 0);
      op.b = static_cast<uint8_t>(in.b >= 0 ? regOf[in.b] : 0);
      op.c = static_cast<uint8_t>(in.c >= 0 ? regOf[in.c] : 0);
    }
    // free operands whose last use is this instruction (before choosing dst)
    if (in.op != XO_CONST && in.op != XO_ARG)
      for (int r : {in.a, in.b, in.c})
        if (r >= 0 && lastUse[r] == i) {
          bool dup = false;
          for (int f : freeRegs) dup = dup || (f == regOf[r]);
          if (!dup) freeRegs.push_back(regOf[r]);
        }
    int dst;
    if (!freeRegs.empty()) {
      dst = freeRegs.back();
      freeRegs.pop_back();
    } else {
      dst = nregs++;
    }
    regOf[i] = dst;
    op.dst = static_cast<uint8_t>(dst);
    p.ops.push_back(op);
  }
  if (nregs > kMaxExprRegs) throw std::runtime_error("expression needs too many registers");
  if (static_cast<int>(p.ops.size()) > kMaxExprOps) throw std::runtime_error("expression too long");
  if (p.consts.size() > 65535) throw std::runtime_error("too many constants");
  for (int o : outs) p.outputs.push_back(static_cast<uint8_t>(regOf[o]));
  p.n_regs = nregs;
  return p;
}

namespace {

std::string emitSsa(const Builder &b, const std::vector<int> &live, bool fp32, std::vector<std::string> &names) {
  const char *T = fp32 ? "float" : "double";
  auto fn = [&](const char *d) { return fp32 ? std::string(d) + "f" : std::string(d); };
  std::string out;
  char buf[128];
  names.assign(b.code.size(), "");
  for (size_t i = 0; i < b.code.size(); ++i) {
    if (!live[i]) continue;
    const SsaInst &in = b.code[i];
    std::string nm = "r" + std::to_string(i);
    names[i] = nm;
    auto A = [&](int r) { return names[r]; };
    std::string e;
    switch (in.op) {
      case XO_CONST:
        std::snprintf(buf, sizeof buf, "%s(%.17g)", T, in.k);
        e = buf;
        break;
      case XO_ARG: e = "a[" + std::to_string(in.a) + "]"; break;
      case XO_ADD: e = A(in.a) + " + " + A(in.b); break;
      case XO_SUB: e = A(in.a) + " - " + A(in.b); break;
      case XO_MUL: e = A(in.a) + " * " + A(in.b); break;
      case XO_DIV: e = A(in.a) + " / " + A(in.b); break;
      case XO_SQUARE: e = A(in.a) + " * " + A(in.a); break;
      case XO_POW: e = fn("pow") + "(" + A(in.a) + ", " + A(in.b) + ")"; break;
      case XO_NEG: e = "-" + A(in.a); break;
      case XO_ABS: e = fn("fabs") + "(" + A(in.a) + ")"; break;
      case XO_SQRT: e = fn("sqrt") + "(" + A(in.a) + ")"; break;
      case XO_EXP: e = fn("exp") + "(" + A(in.a) + ")"; break;
      case XO_LOG: e = fn("log") + "(" + A(in.a) + ")"; break;
      case XO_SIN: e = fn("sin") + "(" + A(in.a) + ")"; break;
      case XO_COS: e = fn("cos") + "(" + A(in.a) + ")"; break;
      case XO_TAN: e = fn("tan") + "(" + A(in.a) + ")"; break;
      case XO_ATAN: e = fn("atan") + "(" + A(in.a) + ")"; break;
      case XO_FLOOR: e = fn("floor") + "(" + A(in.a) + ")"; break;
      case XO_CEIL: e = fn("ceil") + "(" + A(in.a) + ")"; break;
      case XO_MOD: e = fn("fmod") + "(" + A(in.a) + ", " + A(in.b) + ")"; break;
      case XO_SIGN: e = std::string(T) + "((" + A(in.a) + " > 0) - (" + A(in.a) + " < 0))"; break;
      case XO_MIN: e = "(" + A(in.a) + " < " + A(in.b) + " ? " + A(in.a) + " : " + A(in.b) + ")"; break;
      case XO_MAX: e = "(" + A(in.a) + " > " + A(in.b) + " ? " + A(in.a) + " : " + A(in.b) + ")"; break;
      case XO_LT: e = std::string(T) + "(" + A(in.a) + " < " + A(in.b) + ")"; break;
      case XO_LE: e = std::string(T) + "(" + A(in.a) + " <= " + A(in.b) + ")"; break;
      case XO_GT: e = std::string(T) + "(" + A(in.a) + " > " + A(in.b) + ")"; break;
      case XO_GE: e = std::string(T) + "(" + A(in.a) + " >= " + A(in.b) + ")"; break;
      case XO_EQ: e = std::string(T) + "(" + A(in.a) + " == " + A(in.b) + ")"; break;
      case XO_NE: e = std::string(T) + "(" + A(in.a) + " != " + A(in.b) + ")"; break;
      case XO_AND: e = std::string(T) + "(" + A(in.a) + " != 0 && " + A(in.b) + " != 0)"; break;
      case XO_OR: e = std::string(T) + "(" + A(in.a) + " != 0 || " + A(in.b) + " != 0)"; break;
      case XO_NOT: e = std::string(T) + "(" + A(in.a) + " == 0)"; break;
      case XO_SELECT: e = "(" + A(in.a) + " != 0 ? " + A(in.b) + " : " + A(in.c) + ")"; break;
      default: throw std::runtime_error("bad opcode in code emission");
    }
    out += "    const " + std::string(T) + " " + nm + " = " + e + ";\n";
  }
  return out;
}

std::vector<int> liveSet(const Builder &b, const std::vector<int> &outs) {
  std::vector<int> live(b.code.size(), 0);
  std::vector<int> stack(outs.begin(), outs.end());
  while (!stack.empty()) {
    int r = stack.back();
    stack.pop_back();
    if (r < 0 || live[r]) continue;
    live[r] = 1;
    const SsaInst &in = b.code[r];
    if (in.op == XO_CONST || in.op == XO_ARG) continue;
    stack.push_back(in.a);
    stack.push_back(in.b);
    stack.push_back(in.c);
  }
  return live;
}

}  // namespace

std::string emitYieldPolicy(const ExprPtr &f, const std::vector<ExprPtr> &grads, bool fp32) {
  const char *T = fp32 ? "float" : "double";
  std::string src = "struct YieldJit {\n  static constexpr bool kPlastic = true;\n  static constexpr int kNh = " +
                    std::to_string(static_cast<int>(grads.size()) - 6) + ";\n  static constexpr int kMinBlocks = 2;\n";
  {
    Builder b;
    int o = b.build(f.get());
    std::vector<std::string> names;
    std::string body = emitSsa(b, liveSet(b, {o}), fp32, names);
    src += "  __device__ static __forceinline__ " + std::string(T) + " f(const DevModel<" + T + "> &, const " + T +
           " *__restrict__ a, " + T + " *) {\n" + body + "    return " + names[o] + ";\n  }\n";
  }
  {
    Builder b;
    std::vector<int> outs;
    for (auto &g : grads) outs.push_back(b.build(g.get()));
    std::vector<std::string> names;
    std::string body = emitSsa(b, liveSet(b, outs), fp32, names);
    src += "  __device__ static __forceinline__ void grad(const DevModel<" + std::string(T) + "> &, const " + T +
           " *__restrict__ a, " + T + " *g, " + T + " *) {\n" + body;
    for (size_t k = 0; k < outs.size(); ++k) src += "    g[" + std::to_string(k) + "] = " + names[outs[k]] + ";\n";
    src += "  }\n";
  }
  src += "};\n";
  return src;
}

namespace {

// Reverse-mode rule of one SSA instruction as C++ statements: adds the
// contributions of the result's adjoint `d` to the adjoints of its operands.
// Piecewise-constant operations (comparisons, floor, sign, ...) contribute
// nothing; min/max/select pass the adjoint to the operand they selected.
std::string adjRule(const SsaInst &in, const std::string &d, const std::vector<std::string> &nm,
                    const std::vector<std::string> &adj, bool fp32, const std::vector<int> &isArgOrConst) {
  auto fn = [&](const char *f) { return fp32 ? std::string(f) + "f" : std::string(f); };
  const char *T = fp32 ? "float" : "double";
  auto A = [&](int r) { return nm[r]; };
  // a target that is a constant has no adjoint
  auto add = [&](int r, const std::string &e) -> std::string {
    if (r < 0 || adj[r].empty()) return "";
    return "    " + adj[r] + " += " + e + ";\n";
  };
  (void)isArgOrConst;
  switch (in.op) {
    case XO_ADD: return add(in.a, d) + add(in.b, d);
    case XO_SUB: return add(in.a, d) + add(in.b, "-" + d);
    case XO_MUL: return add(in.a, d + " * " + A(in.b)) + add(in.b, d + " * " + A(in.a));
    case XO_DIV:
      return add(in.a, d + " / " + A(in.b)) + add(in.b, "-" + d + " * " + A(in.a) + " / (" + A(in.b) + " * " + A(in.b) + ")");
    case XO_SQUARE: return add(in.a, std::string(T) + "(2) * " + A(in.a) + " * " + d);
    case XO_POW:
      return add(in.a, d + " * " + A(in.b) + " * " + fn("pow") + "(" + A(in.a) + ", " + A(in.b) + " - " + T + "(1))") +
             add(in.b, "(" + A(in.a) + " > " + T + "(0) ? " + d + " * " + fn("pow") + "(" + A(in.a) + ", " + A(in.b) +
                           ") * " + fn("log") + "(" + A(in.a) + ") : " + T + "(0))");
    case XO_NEG: return add(in.a, "-" + d);
    case XO_ABS: return add(in.a, "(" + A(in.a) + " > " + T + "(0) ? " + d + " : (" + A(in.a) + " < " + T + "(0) ? -" + d + " : " + T + "(0)))");
    case XO_SQRT: return add(in.a, d + " * " + T + "(0.5) / " + fn("sqrt") + "(" + A(in.a) + ")");
    case XO_EXP: return add(in.a, d + " * " + fn("exp") + "(" + A(in.a) + ")");
    case XO_LOG: return add(in.a, d + " / " + A(in.a));
    case XO_SIN: return add(in.a, d + " * " + fn("cos") + "(" + A(in.a) + ")");
    case XO_COS: return add(in.a, "-" + d + " * " + fn("sin") + "(" + A(in.a) + ")");
    case XO_TAN: {
      std::string t = fn("tan") + "(" + A(in.a) + ")";
      return add(in.a, d + " * (" + T + "(1) + " + t + " * " + t + ")");
    }
    case XO_ATAN: return add(in.a, d + " / (" + T + "(1) + " + A(in.a) + " * " + A(in.a) + ")");
    case XO_MOD:
      return add(in.a, d) + add(in.b, "-" + d + " * " + fn("trunc") + "(" + A(in.a) + " / " + A(in.b) + ")");
    case XO_MIN:
      return "    if (" + A(in.a) + " < " + A(in.b) + ") {\n" + add(in.a, d) + "    } else {\n" + add(in.b, d) + "    }\n";
    case XO_MAX:
      return "    if (" + A(in.a) + " > " + A(in.b) + ") {\n" + add(in.a, d) + "    } else {\n" + add(in.b, d) + "    }\n";
    case XO_SELECT:
      return "    if (" + A(in.a) + " != " + T + "(0)) {\n" + add(in.b, d) + "    } else {\n" + add(in.c, d) + "    }\n";
    default: return "";  // constants, arguments (handled by the caller), piecewise-constant ops
  }
}

}  // namespace

std::string emitYieldAdjPolicy(const ExprPtr &f, const std::vector<ExprPtr> &grads, bool fp32,
                               const std::string &qual) {
  const std::string T = fp32 ? "float" : "double";
  const int nh = static_cast<int>(grads.size()) - 6;
  std::string src = "struct YieldAdj {\n  static constexpr bool kPlastic = true;\n  static constexpr int kNh = " +
                    std::to_string(nh) + ";\n";
  {
    Builder b;
    int o = b.build(f.get());
    std::vector<std::string> names;
    std::string body = emitSsa(b, liveSet(b, {o}), fp32, names);
    src += "  template <class M> " + qual + " static " + T + " f(const M &, const " + T + " *__restrict__ a) {\n" + body +
           "    return " + names[o] + ";\n  }\n";
  }
  {
    Builder b;
    std::vector<int> outs;
    for (auto &g : grads) outs.push_back(b.build(g.get()));
    std::vector<std::string> names;
    std::string body = emitSsa(b, liveSet(b, outs), fp32, names);
    src += "  template <class M> " + qual + " static void grad(const M &, const " + T + " *__restrict__ a, " + T +
           " *g) {\n" + body;
    for (size_t k = 0; k < outs.size(); ++k) src += "    g[" + std::to_string(k) + "] = " + names[outs[k]] + ";\n";
    src += "  }\n";
  }
  {
    // vjp: la[arg] += d(lf f + sum_k lg[k] g_k)/d arg
    Builder b;
    std::vector<int> outs;
    outs.push_back(b.build(f.get()));
    for (auto &g : grads) outs.push_back(b.build(g.get()));
    std::vector<int> live = liveSet(b, outs);
    std::vector<std::string> names;
    std::string body = emitSsa(b, live, fp32, names);
    const size_t n = b.code.size();
    std::vector<std::string> adj(n);
    std::vector<int> dummy;
    std::string decl;
    for (size_t i = 0; i < n; ++i) {
      if (!live[i] || b.code[i].op == XO_CONST) continue;
      adj[i] = "d" + std::to_string(i);
      decl += "    " + T + " " + adj[i] + " = " + T + "(0);\n";
    }
    std::string seeds = "    " + adj[outs[0]] + " += lf;\n";
    for (size_t k = 1; k < outs.size(); ++k)
      if (!adj[outs[k]].empty()) seeds += "    " + adj[outs[k]] + " += lg[" + std::to_string(k - 1) + "];\n";
    std::string rev;
    for (size_t j = n; j-- > 0;) {
      if (!live[j] || adj[j].empty()) continue;
      const SsaInst &in = b.code[j];
      if (in.op == XO_ARG) {
        rev += "    la[" + std::to_string(in.a) + "] += " + adj[j] + ";\n";
        continue;
      }
      rev += adjRule(in, adj[j], names, adj, fp32, dummy);
    }
    src += "  template <class M> " + qual + " static void vjp(const M &, const " + T + " *__restrict__ a, " + T +
           " lf, const " + T + " *__restrict__ lg, " + T + " *__restrict__ la) {\n" + body + decl + seeds + rev +
           "  }\n";
  }
  src += "};\n";
  return src;
}

void runProgram(const ExprProgram &p, const double *args, double *out) {
  double r[kMaxExprRegs];
  for (const ExprOp &o : p.ops) {
    double v;
    if (o.op == XO_CONST) v = p.consts[o.a | (o.b << 8)];
    else if (o.op == XO_ARG) v = args[o.a];
    else v = applyOp(o.op, r[o.a], r[o.b], r[o.c]);
    r[o.dst] = v;
  }
  for (size_t i = 0; i < p.outputs.size(); ++i) out[i] = r[p.outputs[i]];
}

}  // namespace dl
