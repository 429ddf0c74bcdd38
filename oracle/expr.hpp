// Oracle (test infrastructure only): a small evaluator for the expression
// strings of dynLattice .pro files.  The reference hands these strings to
// JEM's FuncUtils (src/utils/helpers.cpp:11-35,
// src/materials/ElastoPlasticRodMaterial.cpp:132-143, JIVE LoadScale
// "scaleFunc" in tests/transient/test1.pro:28); JEM is not available, so the
// grammar is restated from the expressions the reference's tests use:
//   numbers (1, 1.5, .5, 2e-3), variables, PI,
//   + - * / % ^ (right-assoc power), unary -, !,
//   < <= > >= == != && ||, parentheses,
//   abs sqrt exp log sin cos tan atan floor ceil sign min max pow if(c,a,b).
// This evaluator walks an AST in double precision; it is the checker's own
// implementation and shares no code with the engine's expression compiler.
#pragma once
#include <cmath>
#include <memory>
#include <stdexcept>
#include <string>
#include <vector>

namespace orc {

struct ExprNode {
  enum Kind { NUM, VAR, UN, BIN, CALL } kind;
  double num = 0.0;
  int var = -1;
  std::string op;                            // operator or function name
  std::vector<std::unique_ptr<ExprNode>> kids;
};

class Expr {
 public:
  Expr() = default;
  Expr(const std::string &src, const std::vector<std::string> &names) { parse(src, names); }

  void parse(const std::string &src, const std::vector<std::string> &names) {
    s_ = src;
    p_ = 0;
    names_ = names;
    root_ = parseOr();
    skip();
    if (p_ != s_.size()) throw std::runtime_error("trailing characters in expression: " + src);
  }
  bool empty() const { return !root_; }
  double eval(const double *vars) const { return ev(root_.get(), vars); }

 private:
  std::string s_;
  size_t p_ = 0;
  std::vector<std::string> names_;
  std::unique_ptr<ExprNode> root_;

  void skip() {
    while (p_ < s_.size() && std::isspace(static_cast<unsigned char>(s_[p_]))) ++p_;
  }
  bool accept(const char *tok) {
    skip();
    size_t n = std::char_traits<char>::length(tok);
    if (s_.compare(p_, n, tok) == 0) {
      // do not take "<" when "<=" is there, etc. (callers try longer first)
      p_ += n;
      return true;
    }
    return false;
  }
  static std::unique_ptr<ExprNode> bin(const std::string &op, std::unique_ptr<ExprNode> a,
                                       std::unique_ptr<ExprNode> b) {
    auto n = std::make_unique<ExprNode>();
    n->kind = ExprNode::BIN;
    n->op = op;
    n->kids.push_back(std::move(a));
    n->kids.push_back(std::move(b));
    return n;
  }
  std::unique_ptr<ExprNode> parseOr() {
    auto a = parseAnd();
    while (accept("||")) a = bin("||", std::move(a), parseAnd());
    return a;
  }
  std::unique_ptr<ExprNode> parseAnd() {
    auto a = parseCmp();
    while (accept("&&")) a = bin("&&", std::move(a), parseCmp());
    return a;
  }
  std::unique_ptr<ExprNode> parseCmp() {
    auto a = parseAdd();
    for (;;) {
      if (accept("<=")) a = bin("<=", std::move(a), parseAdd());
      else if (accept(">=")) a = bin(">=", std::move(a), parseAdd());
      else if (accept("==")) a = bin("==", std::move(a), parseAdd());
      else if (accept("!=")) a = bin("!=", std::move(a), parseAdd());
      else if (accept("<")) a = bin("<", std::move(a), parseAdd());
      else if (accept(">")) a = bin(">", std::move(a), parseAdd());
      else return a;
    }
  }
  std::unique_ptr<ExprNode> parseAdd() {
    auto a = parseMul();
    for (;;) {
      if (accept("+")) a = bin("+", std::move(a), parseMul());
      else if (accept("-")) a = bin("-", std::move(a), parseMul());
      else return a;
    }
  }
  std::unique_ptr<ExprNode> parseMul() {
    auto a = parseUnary();
    for (;;) {
      if (accept("*")) a = bin("*", std::move(a), parseUnary());
      else if (accept("/")) a = bin("/", std::move(a), parseUnary());
      else if (accept("%")) a = bin("%", std::move(a), parseUnary());
      else return a;
    }
  }
  std::unique_ptr<ExprNode> parseUnary() {
    if (accept("-")) {
      auto n = std::make_unique<ExprNode>();
      n->kind = ExprNode::UN;
      n->op = "-";
      n->kids.push_back(parseUnary());
      return n;
    }
    if (accept("+")) return parseUnary();
    if (accept("!")) {
      auto n = std::make_unique<ExprNode>();
      n->kind = ExprNode::UN;
      n->op = "!";
      n->kids.push_back(parseUnary());
      return n;
    }
    return parsePow();
  }
  std::unique_ptr<ExprNode> parsePow() {
    auto a = parseAtom();
    if (accept("^")) return bin("^", std::move(a), parseUnary());
    return a;
  }
  std::unique_ptr<ExprNode> parseAtom() {
    skip();
    if (p_ >= s_.size()) throw std::runtime_error("unexpected end of expression: " + s_);
    char c = s_[p_];
    if (c == '(') {
      ++p_;
      auto a = parseOr();
      if (!accept(")")) throw std::runtime_error("missing ) in " + s_);
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
      auto n = std::make_unique<ExprNode>();
      n->kind = ExprNode::NUM;
      n->num = std::stod(s_.substr(p_, q - p_));
      p_ = q;
      return n;
    }
    if (std::isalpha(static_cast<unsigned char>(c)) || c == '_') {
      size_t q = p_;
      while (q < s_.size() && (std::isalnum(static_cast<unsigned char>(s_[q])) || s_[q] == '_' || s_[q] == '.')) ++q;
      std::string id = s_.substr(p_, q - p_);
      p_ = q;
      skip();
      if (p_ < s_.size() && s_[p_] == '(') {
        ++p_;
        auto n = std::make_unique<ExprNode>();
        n->kind = ExprNode::CALL;
        n->op = id;
        skip();
        if (!accept(")")) {
          for (;;) {
            n->kids.push_back(parseOr());
            if (accept(")")) break;
            if (!accept(",")) throw std::runtime_error("expected , in call of " + id);
          }
        }
        return n;
      }
      auto n = std::make_unique<ExprNode>();
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
      throw std::runtime_error("unknown variable '" + id + "' in " + s_);
    }
    throw std::runtime_error(std::string("unexpected character '") + c + "' in " + s_);
  }

  static double ev(const ExprNode *n, const double *v) {
    switch (n->kind) {
      case ExprNode::NUM: return n->num;
      case ExprNode::VAR: return v[n->var];
      case ExprNode::UN: {
        double a = ev(n->kids[0].get(), v);
        return n->op == "-" ? -a : (a == 0.0 ? 1.0 : 0.0);
      }
      case ExprNode::BIN: {
        const std::string &o = n->op;
        double a = ev(n->kids[0].get(), v);
        if (o == "&&") return (a != 0.0 && ev(n->kids[1].get(), v) != 0.0) ? 1.0 : 0.0;
        if (o == "||") return (a != 0.0 || ev(n->kids[1].get(), v) != 0.0) ? 1.0 : 0.0;
        double b = ev(n->kids[1].get(), v);
        if (o == "+") return a + b;
        if (o == "-") return a - b;
        if (o == "*") return a * b;
        if (o == "/") return a / b;
        if (o == "%") return std::fmod(a, b);
        if (o == "^") return std::pow(a, b);
        if (o == "<") return a < b;
        if (o == "<=") return a <= b;
        if (o == ">") return a > b;
        if (o == ">=") return a >= b;
        if (o == "==") return a == b;
        if (o == "!=") return a != b;
        break;
      }
      case ExprNode::CALL: {
        const std::string &f = n->op;
        if (f == "if") {
          if (n->kids.size() != 3) throw std::runtime_error("if() takes 3 arguments");
          return ev(n->kids[0].get(), v) != 0.0 ? ev(n->kids[1].get(), v) : ev(n->kids[2].get(), v);
        }
        std::vector<double> a;
        for (auto &k : n->kids) a.push_back(ev(k.get(), v));
        auto need = [&](size_t k) {
          if (a.size() != k) throw std::runtime_error("wrong argument count for " + f);
        };
        if (f == "abs") { need(1); return std::fabs(a[0]); }
        if (f == "sqrt") { need(1); return std::sqrt(a[0]); }
        if (f == "exp") { need(1); return std::exp(a[0]); }
        if (f == "log") { need(1); return std::log(a[0]); }
        if (f == "sin") { need(1); return std::sin(a[0]); }
        if (f == "cos") { need(1); return std::cos(a[0]); }
        if (f == "tan") { need(1); return std::tan(a[0]); }
        if (f == "atan") { need(1); return std::atan(a[0]); }
        if (f == "floor") { need(1); return std::floor(a[0]); }
        if (f == "ceil") { need(1); return std::ceil(a[0]); }
        if (f == "sign") { need(1); return (a[0] > 0.0) - (a[0] < 0.0); }
        if (f == "pow") { need(2); return std::pow(a[0], a[1]); }
        if (f == "min") {
          if (a.empty()) throw std::runtime_error("min()");
          double m = a[0];
          for (double x : a) m = x < m ? x : m;
          return m;
        }
        if (f == "max") {
          if (a.empty()) throw std::runtime_error("max()");
          double m = a[0];
          for (double x : a) m = x > m ? x : m;
          return m;
        }
        throw std::runtime_error("unknown function " + f);
      }
    }
    throw std::runtime_error("bad expression node");
  }
};

}  // namespace orc
