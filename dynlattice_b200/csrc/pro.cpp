// dynLattice .pro input surface (see pro.hpp).
#include "pro.hpp"

#include <algorithm>
#include <cctype>
#include <cmath>
#include <cstring>
#include <fstream>
#include <functional>
#include <set>
#include <sstream>
#include <stdexcept>

#include "expr.hpp"

namespace dl {

namespace {

// ---------------------------------------------------------------------------
// property store
// ---------------------------------------------------------------------------
struct Val {
  enum Kind { NUM, STR, BOOL, ARR } kind = NUM;
  double num = 0.0;
  std::string str;
  bool b = false;
  std::vector<Val> arr;
};

struct Store {
  std::map<std::string, Val> kv;  // full dotted key -> leaf

  bool has(const std::string &k) const { return kv.count(k) > 0; }
  bool has_tree(const std::string &k) const {
    auto it = kv.lower_bound(k + ".");
    return it != kv.end() && it->first.compare(0, k.size() + 1, k + ".") == 0;
  }
  const Val *get(const std::string &k) const {
    auto it = kv.find(k);
    return it == kv.end() ? nullptr : &it->second;
  }
  // keys of the subtree (relative names, first component)
  std::vector<std::string> children(const std::string &k) const {
    std::vector<std::string> out;
    std::set<std::string> seen;
    const std::string p = k + ".";
    for (auto it = kv.lower_bound(p); it != kv.end() && it->first.compare(0, p.size(), p) == 0; ++it) {
      std::string rest = it->first.substr(p.size());
      std::string first = rest.substr(0, rest.find('.'));
      if (seen.insert(first).second) out.push_back(first);
    }
    return out;
  }
  void copy_tree(const std::string &from, const std::string &to) {
    std::vector<std::pair<std::string, Val>> add;
    if (const Val *v = get(from)) add.push_back({to, *v});
    const std::string p = from + ".";
    for (auto it = kv.lower_bound(p); it != kv.end() && it->first.compare(0, p.size(), p) == 0; ++it)
      add.push_back({to + it->first.substr(from.size()), it->second});
    for (auto &a : add) kv[a.first] = a.second;
  }
};

// ---------------------------------------------------------------------------
// lexer / parser of JEM property files
// ---------------------------------------------------------------------------
struct Tok {
  enum Kind { END, IDENT, NUM, STR, PUNCT } kind = END;
  std::string s;
  double num = 0.0;
  int line = 0;
};

std::string read_text(const std::string &path) {
  std::ifstream f(path);
  if (!f) throw std::runtime_error("cannot open " + path);
  std::stringstream ss;
  ss << f.rdbuf();
  return ss.str();
}

std::string dir_of(const std::string &path) {
  const size_t p = path.find_last_of('/');
  return p == std::string::npos ? std::string(".") : path.substr(0, p);
}

std::vector<Tok> lex(const std::string &src, const std::string &file) {
  std::vector<Tok> out;
  size_t i = 0;
  int line = 1;
  const size_t n = src.size();
  while (i < n) {
    const char c = src[i];
    if (c == '\n') {
      ++line;
      ++i;
      continue;
    }
    if (std::isspace(static_cast<unsigned char>(c))) {
      ++i;
      continue;
    }
    if (c == '/' && i + 1 < n && src[i + 1] == '/') {
      while (i < n && src[i] != '\n') ++i;
      continue;
    }
    if (c == '/' && i + 1 < n && src[i + 1] == '*') {
      i += 2;
      while (i + 1 < n && !(src[i] == '*' && src[i + 1] == '/')) {
        if (src[i] == '\n') ++line;
        ++i;
      }
      i += 2;
      continue;
    }
    Tok t;
    t.line = line;
    if (c == '"') {
      ++i;
      std::string s;
      while (i < n && src[i] != '"') {
        if (src[i] == '\\' && i + 1 < n) {
          s += src[i + 1];
          i += 2;
          continue;
        }
        if (src[i] == '\n') ++line;
        s += src[i++];
      }
      if (i >= n) throw std::runtime_error(file + ":" + std::to_string(t.line) + ": unterminated string");
      ++i;
      t.kind = Tok::STR;
      t.s = s;
      out.push_back(t);
      continue;
    }
    if (std::isdigit(static_cast<unsigned char>(c)) ||
        (c == '.' && i + 1 < n && std::isdigit(static_cast<unsigned char>(src[i + 1])))) {
      size_t j = i;
      while (j < n && (std::isdigit(static_cast<unsigned char>(src[j])) || src[j] == '.')) ++j;
      if (j < n && (src[j] == 'e' || src[j] == 'E')) {
        size_t k = j + 1;
        if (k < n && (src[k] == '+' || src[k] == '-')) ++k;
        if (k < n && std::isdigit(static_cast<unsigned char>(src[k]))) {
          j = k;
          while (j < n && std::isdigit(static_cast<unsigned char>(src[j]))) ++j;
        }
      }
      t.kind = Tok::NUM;
      t.num = std::strtod(src.substr(i, j - i).c_str(), nullptr);
      out.push_back(t);
      i = j;
      continue;
    }
    if (std::isalpha(static_cast<unsigned char>(c)) || c == '_') {
      size_t j = i;
      while (j < n && (std::isalnum(static_cast<unsigned char>(src[j])) || src[j] == '_' || src[j] == '.')) ++j;
      t.kind = Tok::IDENT;
      t.s = src.substr(i, j - i);
      out.push_back(t);
      i = j;
      continue;
    }
    if (c == '+' && i + 1 < n && src[i + 1] == '=') {
      t.kind = Tok::PUNCT;
      t.s = "+=";
      out.push_back(t);
      i += 2;
      continue;
    }
    if (std::strchr("=;[]{},-", c)) {
      t.kind = Tok::PUNCT;
      t.s = std::string(1, c);
      out.push_back(t);
      ++i;
      continue;
    }
    throw std::runtime_error(file + ":" + std::to_string(line) + ": unexpected character '" + std::string(1, c) +
                             "'");
  }
  Tok e;
  e.line = line;
  out.push_back(e);
  return out;
}

struct Parser {
  Store &st;
  std::string case_name;
  int depth = 0;

  explicit Parser(Store &s, std::string cn) : st(s), case_name(std::move(cn)) {}

  std::string subst(const std::string &s) const {
    std::string out;
    size_t i = 0;
    while (i < s.size()) {
      if (s[i] == '$' && i + 1 < s.size() && s[i + 1] == '(') {
        const size_t e = s.find(')', i);
        if (e == std::string::npos) break;
        const std::string key = s.substr(i + 2, e - i - 2);
        if (key == "CASE_NAME") {
          out += case_name;
        } else if (const Val *v = st.get(key)) {
          if (v->kind == Val::NUM) {
            std::ostringstream os;
            os.precision(17);
            os << v->num;
            out += os.str();
          } else if (v->kind == Val::STR) {
            out += v->str;
          } else {
            out += s.substr(i, e - i + 1);
          }
        } else {
          out += s.substr(i, e - i + 1);
        }
        i = e + 1;
        continue;
      }
      out += s[i++];
    }
    return out;
  }

  void file(const std::string &path, const std::string &prefix) {
    if (++depth > 32) throw std::runtime_error("include nesting too deep at " + path);
    const std::vector<Tok> t = lex(read_text(path), path);
    size_t i = 0;
    block(t, i, prefix, path, false);
    --depth;
  }

  [[noreturn]] void fail(const std::string &path, const Tok &t, const std::string &msg) {
    throw std::runtime_error(path + ":" + std::to_string(t.line) + ": " + msg);
  }

  // statements until END (or '}' when nested)
  void block(const std::vector<Tok> &t, size_t &i, const std::string &prefix, const std::string &path, bool nested) {
    for (;;) {
      const Tok &a = t[i];
      if (a.kind == Tok::END) {
        if (nested) fail(path, a, "missing '}'");
        return;
      }
      if (nested && a.kind == Tok::PUNCT && a.s == "}") {
        ++i;
        return;
      }
      if (a.kind == Tok::PUNCT && a.s == ";") {
        ++i;
        continue;
      }
      if (a.kind != Tok::IDENT) fail(path, a, "expected a property name");
      if (a.s == "include" && t[i + 1].kind == Tok::STR) {
        std::string inc = subst(t[i + 1].s);
        std::string p = inc;
        if (!p.empty() && p[0] != '/') {
          std::ifstream probe(dir_of(path) + "/" + inc);
          p = probe ? dir_of(path) + "/" + inc : inc;
        }
        i += 2;
        if (t[i].kind == Tok::PUNCT && t[i].s == ";") ++i;
        file(p, prefix);
        continue;
      }
      const std::string key = prefix.empty() ? a.s : prefix + "." + a.s;
      ++i;
      if (t[i].kind != Tok::PUNCT || (t[i].s != "=" && t[i].s != "+=")) fail(path, t[i], "expected '=' or '+='");
      const bool append = t[i].s == "+=";
      ++i;
      assign(t, i, key, append, path);
      if (t[i].kind == Tok::PUNCT && t[i].s == ";") ++i;
    }
  }

  Val scalar(const std::vector<Tok> &t, size_t &i, const std::string &path) {
    Val v;
    const Tok &a = t[i];
    if (a.kind == Tok::PUNCT && a.s == "-" && t[i + 1].kind == Tok::NUM) {
      v.kind = Val::NUM;
      v.num = -t[i + 1].num;
      i += 2;
      return v;
    }
    if (a.kind == Tok::NUM) {
      v.kind = Val::NUM;
      v.num = a.num;
      ++i;
      return v;
    }
    if (a.kind == Tok::STR) {
      v.kind = Val::STR;
      v.str = subst(a.s);
      ++i;
      return v;
    }
    if (a.kind == Tok::IDENT && (a.s == "true" || a.s == "false")) {
      v.kind = Val::BOOL;
      v.b = a.s == "true";
      ++i;
      return v;
    }
    if (a.kind == Tok::IDENT) {  // reference to a leaf
      const Val *r = st.get(a.s);
      if (!r) fail(path, a, "unknown property " + a.s);
      ++i;
      return *r;
    }
    fail(path, a, "expected a value");
  }

  void assign(const std::vector<Tok> &t, size_t &i, const std::string &key, bool append, const std::string &path) {
    const Tok &a = t[i];
    if (a.kind == Tok::PUNCT && a.s == "{") {  // property block
      ++i;
      if (!append) {
        // a new block replaces the subtree
        for (auto it = st.kv.lower_bound(key + "."); it != st.kv.end() && it->first.rfind(key + ".", 0) == 0;)
          it = st.kv.erase(it);
      }
      block(t, i, key, path, true);
      return;
    }
    if (a.kind == Tok::IDENT && a.s != "true" && a.s != "false" && st.has_tree(a.s) && !st.has(a.s)) {
      // reference to a subtree: copy (or merge with +=)
      ++i;
      if (!append)
        for (auto it = st.kv.lower_bound(key + "."); it != st.kv.end() && it->first.rfind(key + ".", 0) == 0;)
          it = st.kv.erase(it);
      st.copy_tree(a.s, key);
      return;
    }
    Val v;
    if (a.kind == Tok::PUNCT && a.s == "[") {
      ++i;
      v.kind = Val::ARR;
      while (!(t[i].kind == Tok::PUNCT && t[i].s == "]")) {
        if (t[i].kind == Tok::END) fail(path, t[i], "missing ']'");
        Val e = scalar(t, i, path);
        if (e.kind == Val::ARR)
          v.arr.insert(v.arr.end(), e.arr.begin(), e.arr.end());
        else
          v.arr.push_back(e);
        if (t[i].kind == Tok::PUNCT && t[i].s == ",") ++i;
      }
      ++i;
    } else {
      v = scalar(t, i, path);
    }
    if (!append || !st.has(key)) {
      if (append && v.kind != Val::ARR) {
        Val arr;
        arr.kind = Val::ARR;
        arr.arr.push_back(v);
        st.kv[key] = arr;
      } else {
        st.kv[key] = v;
      }
      return;
    }
    Val &cur = st.kv[key];
    if (cur.kind != Val::ARR) {
      Val arr;
      arr.kind = Val::ARR;
      arr.arr.push_back(cur);
      cur = arr;
    }
    if (v.kind == Val::ARR)
      cur.arr.insert(cur.arr.end(), v.arr.begin(), v.arr.end());
    else
      cur.arr.push_back(v);
  }
};

// ---------------------------------------------------------------------------
// typed access
// ---------------------------------------------------------------------------
double num_of(const Val &v, const std::string &key) {
  if (v.kind == Val::NUM) return v.num;
  if (v.kind == Val::BOOL) return v.b ? 1.0 : 0.0;
  if (v.kind == Val::STR) {
    ExprPtr e = parseExpr(v.str, {});
    return evalExpr(e.get(), nullptr);
  }
  throw std::runtime_error("property " + key + " is not a number");
}

struct View {
  const Store &st;
  double num(const std::string &k) const {
    const Val *v = st.get(k);
    if (!v) throw std::runtime_error("missing property " + k);
    return num_of(*v, k);
  }
  double num(const std::string &k, double dflt) const {
    const Val *v = st.get(k);
    return v ? num_of(*v, k) : dflt;
  }
  bool has(const std::string &k) const { return st.has(k); }
  std::string str(const std::string &k, const std::string &dflt = "") const {
    const Val *v = st.get(k);
    if (!v) return dflt;
    if (v->kind == Val::STR) return v->str;
    if (v->kind == Val::NUM) {
      std::ostringstream os;
      os.precision(17);
      os << v->num;
      return os.str();
    }
    if (v->kind == Val::BOOL) return v->b ? "true" : "false";
    throw std::runtime_error("property " + k + " is not a string");
  }
  std::vector<std::string> strs(const std::string &k) const {
    std::vector<std::string> out;
    const Val *v = st.get(k);
    if (!v) return out;
    if (v->kind == Val::ARR) {
      for (auto &e : v->arr) out.push_back(e.kind == Val::STR ? e.str : std::to_string(e.num));
    } else {
      out.push_back(str(k));
    }
    return out;
  }
  std::vector<double> nums(const std::string &k) const {
    std::vector<double> out;
    const Val *v = st.get(k);
    if (!v) return out;
    if (v->kind == Val::ARR) {
      for (auto &e : v->arr) out.push_back(num_of(e, k));
    } else {
      out.push_back(num_of(*v, k));
    }
    return out;
  }
};

// ---------------------------------------------------------------------------
// .geo subset
// ---------------------------------------------------------------------------
struct GeoPoint {
  double x[3];
  double lc;
};

// gmsh 1D meshing of a straight curve with a characteristic length varying
// linearly from lc0 to lc1: a = integral ds / lc(s); segments = max(1,
// floor(a + 0.99)); nodes equidistributed in that metric.
std::vector<double> line_params(double L, double lc0, double lc1) {
  auto prim = [&](double s) {  // integral_0^s ds / lc
    const double d = lc1 - lc0;
    if (std::fabs(d) < 1e-14 * std::max(lc0, lc1)) return s / lc0;
    return L / d * std::log((lc0 + d * s / L) / lc0);
  };
  const double a = prim(L);
  const int nseg = std::max(1, static_cast<int>(std::floor(a + 0.99)));
  std::vector<double> u(nseg + 1);
  for (int j = 0; j <= nseg; ++j) {
    const double target = a * j / nseg;
    double lo = 0.0, hi = L;
    for (int it = 0; it < 200; ++it) {
      const double mid = 0.5 * (lo + hi);
      if (prim(mid) < target) lo = mid;
      else hi = mid;
    }
    u[j] = (j == 0) ? 0.0 : (j == nseg ? 1.0 : 0.5 * (lo + hi) / L);
  }
  return u;
}

}  // namespace

void mesh_geo(const std::string &path, int order, const std::map<std::string, double> &onelab,
              std::vector<double> &coords, std::vector<std::vector<int32_t>> &line_elems, int &nen,
              std::vector<int32_t> &point_nodes) {
  if (order != 1 && order != 2) throw std::runtime_error("GMSHInput order must be 1 or 2");
  std::string src = read_text(path);
  // strip comments
  std::string s;
  for (size_t i = 0; i < src.size(); ++i) {
    if (src[i] == '/' && i + 1 < src.size() && src[i + 1] == '/') {
      while (i < src.size() && src[i] != '\n') ++i;
      s += '\n';
      continue;
    }
    if (src[i] == '/' && i + 1 < src.size() && src[i + 1] == '*') {
      i += 2;
      while (i + 1 < src.size() && !(src[i] == '*' && src[i + 1] == '/')) ++i;
      ++i;
      continue;
    }
    s += src[i];
  }
  std::map<std::string, double> vars;
  std::map<int, GeoPoint> points;
  std::map<int, std::pair<int, int>> lines;
  std::vector<std::string> varNames;
  auto evalnum = [&](const std::string &e) {
    std::vector<std::string> names;
    std::vector<double> vals;
    for (auto &kv : vars) {
      names.push_back(kv.first);
      vals.push_back(kv.second);
    }
    ExprPtr x = parseExpr(e, names);
    return evalExpr(x.get(), vals.data());
  };
  auto split_top = [](const std::string &body) {  // split on commas outside braces/parens
    std::vector<std::string> out;
    int dep = 0;
    std::string cur;
    for (char c : body) {
      if (c == '{' || c == '(' || c == '[') ++dep;
      if (c == '}' || c == ')' || c == ']') --dep;
      if (c == ',' && dep == 0) {
        out.push_back(cur);
        cur.clear();
      } else {
        cur += c;
      }
    }
    if (!cur.empty()) out.push_back(cur);
    return out;
  };
  auto trim = [](std::string x) {
    size_t a = x.find_first_not_of(" \t\r\n"), b = x.find_last_not_of(" \t\r\n");
    return a == std::string::npos ? std::string() : x.substr(a, b - a + 1);
  };
  // statements end with ';' (DefineConstant blocks contain ';' only inside [])
  size_t i = 0;
  while (i < s.size()) {
    size_t semi = std::string::npos;
    int dep = 0;
    for (size_t j = i; j < s.size(); ++j) {
      if (s[j] == '[' || s[j] == '{' || s[j] == '(') ++dep;
      if (s[j] == ']' || s[j] == '}' || s[j] == ')') --dep;
      if (s[j] == ';' && dep == 0) {
        semi = j;
        break;
      }
    }
    if (semi == std::string::npos) break;
    const std::string st = trim(s.substr(i, semi - i));
    i = semi + 1;
    if (st.empty()) continue;
    if (st.rfind("DefineConstant", 0) == 0) {
      const size_t a = st.find('['), b = st.rfind(']');
      for (std::string item : split_top(st.substr(a + 1, b - a - 1))) {
        item = trim(item);
        if (item.empty()) continue;
        const size_t eq = item.find('=');
        const std::string name = trim(item.substr(0, eq));
        std::string rhs = trim(item.substr(eq + 1));
        std::string valtxt = rhs, oname;
        if (!rhs.empty() && rhs[0] == '{') {
          std::vector<std::string> parts = split_top(rhs.substr(1, rhs.rfind('}') - 1));
          valtxt = parts.empty() ? "0" : parts[0];
          for (size_t p = 1; p < parts.size(); ++p) {
            std::string q = trim(parts[p]);
            if (q.rfind("Name", 0) == 0) {
              const size_t qa = q.find('"'), qb = q.rfind('"');
              if (qa != std::string::npos && qb > qa) oname = q.substr(qa + 1, qb - qa - 1);
            }
          }
        }
        double v = evalnum(trim(valtxt));
        // onelab overrides by parameter name (last path component) or constant name
        std::string shortName = oname.substr(oname.find_last_of('/') + 1);
        if (!oname.empty() && onelab.count(shortName)) v = onelab.at(shortName);
        else if (onelab.count(name)) v = onelab.at(name);
        vars[name] = v;
      }
      continue;
    }
    auto entity = [&](const char *kw, int &id, std::vector<std::string> &vals) {
      if (st.rfind(kw, 0) != 0) return false;
      const size_t a = st.find('('), b = st.find(')');
      const size_t c = st.find('{'), d = st.rfind('}');
      if (a == std::string::npos || c == std::string::npos) return false;
      id = static_cast<int>(std::lround(evalnum(st.substr(a + 1, b - a - 1))));
      vals = split_top(st.substr(c + 1, d - c - 1));
      return true;
    };
    int id = 0;
    std::vector<std::string> vals;
    if (entity("Point", id, vals)) {
      if (vals.size() < 3) throw std::runtime_error(path + ": Point needs x, y, z");
      GeoPoint p;
      for (int k = 0; k < 3; ++k) p.x[k] = evalnum(trim(vals[k]));
      p.lc = vals.size() > 3 ? evalnum(trim(vals[3])) : 1e22;
      points[id] = p;
      continue;
    }
    if (entity("Line", id, vals)) {
      if (vals.size() != 2) throw std::runtime_error(path + ": Line needs two points");
      lines[id] = {static_cast<int>(std::lround(evalnum(trim(vals[0])))),
                   static_cast<int>(std::lround(evalnum(trim(vals[1]))))};
      continue;
    }
    const size_t eq = st.find('=');
    if (eq != std::string::npos && st.find('(') > eq) {  // variable assignment
      vars[trim(st.substr(0, eq))] = evalnum(trim(st.substr(eq + 1)));
      continue;
    }
    throw std::runtime_error(path + ": unsupported .geo statement: " + st);
  }
  // nodes: points in tag order, then per line (tag order) its interior nodes
  coords.clear();
  line_elems.clear();
  std::map<int, int> pnode;
  point_nodes.clear();
  for (auto &kv : points) {
    pnode[kv.first] = static_cast<int>(coords.size() / 3);
    point_nodes.push_back(pnode[kv.first]);
    for (int k = 0; k < 3; ++k) coords.push_back(kv.second.x[k]);
  }
  nen = order + 1;
  for (auto &kv : lines) {
    const GeoPoint &A = points.at(kv.second.first), &B = points.at(kv.second.second);
    double d[3], L2 = 0.0;
    for (int k = 0; k < 3; ++k) {
      d[k] = B.x[k] - A.x[k];
      L2 += d[k] * d[k];
    }
    const double L = std::sqrt(L2);
    const std::vector<double> u = line_params(L, std::min(A.lc, 1e21), std::min(B.lc, 1e21));
    const int nseg = static_cast<int>(u.size()) - 1;
    std::vector<int> vnode(nseg + 1);
    vnode[0] = pnode.at(kv.second.first);
    vnode[nseg] = pnode.at(kv.second.second);
    for (int j = 1; j < nseg; ++j) {
      vnode[j] = static_cast<int>(coords.size() / 3);
      for (int k = 0; k < 3; ++k) coords.push_back(A.x[k] + u[j] * d[k]);
    }
    std::vector<int32_t> elems;
    for (int j = 0; j < nseg; ++j) {
      elems.push_back(vnode[j]);
      if (order == 2) {  // mid node of the segment
        const int mid = static_cast<int>(coords.size() / 3);
        for (int k = 0; k < 3; ++k) coords.push_back(A.x[k] + 0.5 * (u[j] + u[j + 1]) * d[k]);
        elems.push_back(mid);
      }
      elems.push_back(vnode[j + 1]);
    }
    line_elems.push_back(elems);
  }
}

void read_msh(const std::string &path, std::vector<double> &coords, std::vector<std::vector<int32_t>> &line_elems,
              int &nen, std::vector<int32_t> &point_nodes) {
  point_nodes.clear();
  std::ifstream f(path);
  if (!f) throw std::runtime_error("cannot open " + path);
  std::string tok;
  double version = 0.0;
  std::map<long, int> idx;
  std::map<int, std::vector<int32_t>> byEntity;
  nen = 0;
  coords.clear();
  while (f >> tok) {
    if (tok == "$MeshFormat") {
      int ft = 0, ds = 0;
      f >> version >> ft >> ds;
      if (ft != 0) throw std::runtime_error(path + ": binary .msh is not supported");
    } else if (tok == "$Nodes") {
      if (version >= 4.0) {
        long nb, nn, mn, mx;
        f >> nb >> nn >> mn >> mx;
        for (long b = 0; b < nb; ++b) {
          int edim, etag, param;
          long cnt;
          f >> edim >> etag >> param >> cnt;
          std::vector<long> tags(cnt);
          for (auto &t : tags) f >> t;
          for (long k = 0; k < cnt; ++k) {
            double x, y, z;
            f >> x >> y >> z;
            if (param)
              for (int p = 0; p < edim; ++p) {
                double dummy;
                f >> dummy;
              }
            idx[tags[k]] = static_cast<int>(coords.size() / 3);
            coords.push_back(x);
            coords.push_back(y);
            coords.push_back(z);
          }
        }
      } else {
        long nn;
        f >> nn;
        for (long k = 0; k < nn; ++k) {
          long id;
          double x, y, z;
          f >> id >> x >> y >> z;
          idx[id] = static_cast<int>(coords.size() / 3);
          coords.push_back(x);
          coords.push_back(y);
          coords.push_back(z);
        }
      }
    } else if (tok == "$Elements") {
      auto take = [&](int type, int entity, const std::vector<long> &nodes) {
        if (type == 15) {
          point_nodes.push_back(idx.at(nodes[0]));
          return;
        }
        if (type != 1 && type != 8) return;
        const int n = type == 1 ? 2 : 3;
        if (nen && nen != n) throw std::runtime_error(path + ": mixed element orders");
        nen = n;
        auto &v = byEntity[entity];
        // gmsh order (end, end, mid) -> along the line (end, mid, end)
        v.push_back(idx.at(nodes[0]));
        if (n == 3) v.push_back(idx.at(nodes[2]));
        v.push_back(idx.at(nodes[1]));
      };
      if (version >= 4.0) {
        long nb, ne, mn, mx;
        f >> nb >> ne >> mn >> mx;
        for (long b = 0; b < nb; ++b) {
          int edim, etag, type;
          long cnt;
          f >> edim >> etag >> type >> cnt;
          const int nn = type == 1 ? 2 : (type == 8 ? 3 : (type == 15 ? 1 : (type == 2 ? 3 : (type == 3 ? 4 : 4))));
          for (long k = 0; k < cnt; ++k) {
            long id;
            f >> id;
            std::vector<long> nodes(nn);
            for (auto &x : nodes) f >> x;
            take(type, etag, nodes);
          }
        }
      } else {
        long ne;
        f >> ne;
        std::string rest;
        std::getline(f, rest);
        for (long k = 0; k < ne; ++k) {
          std::getline(f, rest);
          std::istringstream ls(rest);
          long id;
          int type, ntags;
          ls >> id >> type >> ntags;
          std::vector<long> tags(ntags);
          for (auto &t : tags) ls >> t;
          std::vector<long> nodes;
          long x;
          while (ls >> x) nodes.push_back(x);
          take(type, ntags > 1 ? static_cast<int>(tags[1]) : 0, nodes);
        }
      }
    }
  }
  line_elems.clear();
  for (auto &kv : byEntity) line_elems.push_back(kv.second);
  if (line_elems.empty()) throw std::runtime_error(path + ": no line elements");
}

namespace {

// GroupInputModule::NGroup_ (GroupInputModule.cpp:165-500): per axis a value
// (xtype min/max/mid, xval, xvals) or bounds (xbounds, firstHalf/secondHalf),
// tolerance eps (1e-5); explicit "nodes"; "all"; restrictToGroup(s).
std::vector<int32_t> node_group(const View &v, const std::string &p, const std::vector<double> &X,
                                const std::map<std::string, std::vector<int32_t>> &elemGroupNodes) {
  const int N = static_cast<int>(X.size() / 3);
  if (v.has(p + ".nodes")) {
    std::vector<int32_t> out;
    for (double d : v.nums(p + ".nodes")) out.push_back(static_cast<int32_t>(d));
    return out;
  }
  std::vector<int32_t> cand;
  std::vector<std::string> restrict = v.strs(p + ".restrictToGroups");
  if (v.has(p + ".restrictToGroup")) restrict = {v.str(p + ".restrictToGroup")};
  if (restrict.empty()) {
    for (int i = 0; i < N; ++i) cand.push_back(i);
  } else {
    std::set<int32_t> s;
    for (auto &g : restrict) {
      auto it = elemGroupNodes.find(g);
      if (it == elemGroupNodes.end()) throw std::runtime_error("GroupInput: unknown element group " + g);
      s.insert(it->second.begin(), it->second.end());
    }
    cand.assign(s.begin(), s.end());
  }
  if (v.has(p + ".all") && v.num(p + ".all") != 0.0) return cand;
  const double eps = v.num(p + ".eps", 1e-5);
  const char *ax[3] = {"x", "y", "z"};
  enum { NONE, VALUE, BOUNDS };
  int mode[3];
  std::vector<double> vals[3];
  double lo[3], hi[3];
  for (int r = 0; r < 3; ++r) {
    mode[r] = NONE;
    double mn = 1e300, mx = -1e300;
    for (int i = 0; i < N; ++i) {
      mn = std::min(mn, X[3 * i + r]);
      mx = std::max(mx, X[3 * i + r]);
    }
    const std::string a = ax[r];
    if (v.has(p + "." + a + "type")) {
      const std::string ty = v.str(p + "." + a + "type");
      mode[r] = VALUE;
      if (ty == "min") vals[r] = {mn};
      else if (ty == "max") vals[r] = {mx};
      else if (ty == "mid") vals[r] = {0.5 * (mn + mx)};
      else if (ty == "firstHalf") {
        mode[r] = BOUNDS;
        lo[r] = mn - eps;
        hi[r] = mn - eps + (mx - mn) / 2.0;
      } else if (ty == "secondHalf") {
        mode[r] = BOUNDS;
        lo[r] = mn + eps + (mx - mn) / 2.0;
        hi[r] = mx + eps;
      } else {
        throw std::runtime_error("Unknown xtype: " + ty);
      }
    } else if (v.has(p + "." + a + "val")) {
      mode[r] = VALUE;
      vals[r] = {v.num(p + "." + a + "val")};
    } else if (v.has(p + "." + a + "vals")) {
      mode[r] = VALUE;
      vals[r] = v.nums(p + "." + a + "vals");
    } else if (v.has(p + "." + a + "bounds")) {
      const std::vector<double> b = v.nums(p + "." + a + "bounds");
      if (b.size() != 2) throw std::runtime_error(p + "." + a + "bounds does not have length 2!");
      mode[r] = BOUNDS;
      lo[r] = b[0] - eps;
      hi[r] = b[1] + eps;
    }
  }
  if (mode[0] == NONE && mode[1] == NONE && mode[2] == NONE)
    throw std::runtime_error("GroupInput " + p + ": radius/angle selections are not supported");
  std::vector<int32_t> out;
  for (int32_t i : cand) {
    bool inc = true;
    for (int r = 0; r < 3 && inc; ++r) {
      const double c = X[3 * i + r];
      if (mode[r] == VALUE) {
        bool any = false;
        for (double xv : vals[r]) any = any || std::fabs(xv - c) < eps;
        inc = any;
      } else if (mode[r] == BOUNDS) {
        inc = c > lo[r] && c < hi[r];
      }
    }
    if (inc) out.push_back(i);
  }
  return out;
}

std::string find_typed(const Store &st, const std::string &type, const std::string &under = "") {
  for (auto &kv : st.kv) {
    const std::string &k = kv.first;
    if (k.size() < 5 || k.compare(k.size() - 5, 5, ".type") != 0) continue;
    if (!under.empty() && k.rfind(under + ".", 0) != 0) continue;
    if (kv.second.kind == Val::STR && kv.second.str == type) return k.substr(0, k.size() - 5);
  }
  return "";
}

int dof_index(const std::vector<std::string> &names, const std::string &d) {
  for (size_t i = 0; i < names.size(); ++i)
    if (names[i] == d) return static_cast<int>(i);
  throw std::runtime_error("unknown DOF name " + d);
}

}  // namespace

std::unique_ptr<ProModel> load_pro(const std::string &path) {
  auto pm = std::make_unique<ProModel>();
  ProModel &M = *pm;
  {
    std::string base = path.substr(path.find_last_of('/') + 1);
    M.case_name = base.substr(0, base.rfind('.'));
  }
  Store st;
  Parser ps(st, M.case_name);
  ps.file(path, "");
  View v{st};
  const std::string dir = dir_of(path);

  // ---- input: mesh and groups
  const std::string gin = find_typed(st, "GMSHInput");
  if (gin.empty()) throw std::runtime_error("no GMSHInput module in " + path);
  std::string meshFile = v.str(gin + ".file");
  if (meshFile.empty()) throw std::runtime_error(gin + ".file is missing");
  if (meshFile[0] != '/') {
    std::ifstream probe(dir + "/" + meshFile);
    if (probe) meshFile = dir + "/" + meshFile;
  }
  const int order = static_cast<int>(v.num(gin + ".order", 1.0));
  std::map<std::string, double> onelab;
  for (auto &c : st.children(gin + ".onelab")) onelab[c] = v.num(gin + ".onelab." + c);
  std::vector<std::vector<int32_t>> lineElems;
  std::vector<int32_t> pointNodes;
  int nen = 2;
  if (meshFile.size() > 4 && meshFile.compare(meshFile.size() - 4, 4, ".msh") == 0)
    read_msh(meshFile, M.coords, lineElems, nen, pointNodes);
  else
    mesh_geo(meshFile, order, onelab, M.coords, lineElems, nen, pointNodes);
  const int N = static_cast<int>(M.coords.size() / 3);
  // element groups of GMSHInputModule::createElems_ (GMSHInputModule.cpp:
  // 342-413): one per entity ("beam_k", "point_k") and "points" for all
  // point elements (its node indices: the unique nodes, ascending)
  std::map<std::string, std::vector<int32_t>> egNodes;
  for (size_t l = 0; l < lineElems.size(); ++l) {
    std::set<int32_t> s(lineElems[l].begin(), lineElems[l].end());
    egNodes["beam_" + std::to_string(l + 1)] = std::vector<int32_t>(s.begin(), s.end());
  }
  if (!pointNodes.empty()) {
    for (size_t k = 0; k < pointNodes.size(); ++k) egNodes["point_" + std::to_string(k + 1)] = {pointNodes[k]};
    std::set<int32_t> s(pointNodes.begin(), pointNodes.end());
    egNodes["points"] = std::vector<int32_t>(s.begin(), s.end());
  }
  // ---- lattice model: rods = element groups <prefix>1, <prefix>2, ...
  const std::string lat = find_typed(st, "Lattice");
  if (lat.empty()) throw std::runtime_error("no Lattice model in " + path);
  const std::string prefix = v.str(lat + ".prefix", "beam_");
  if (prefix != "beam_")
    throw std::runtime_error(lat + ".prefix: the meshes name their line groups beam_1, beam_2, ...");
  for (size_t r = 0; r < lineElems.size(); ++r) {
    const auto &el = lineElems[r];
    for (size_t k = 0; k < el.size(); k += nen) {
      for (int a = 0; a < nen; ++a) M.conn.push_back(el[k + a]);
      M.elem_rod.push_back(static_cast<int32_t>(r));
    }
  }
  const std::string ch = lat + ".child";
  if (v.str(ch + ".type") != "specialCosseratRod")
    throw std::runtime_error(ch + ".type must be specialCosseratRod");
  std::vector<std::string> trans = v.strs(ch + ".dofNamesTrans"), rot = v.strs(ch + ".dofNamesRot");
  if (trans.empty()) trans = {"dx", "dy", "dz"};
  if (rot.empty()) rot = {"rx", "ry", "rz"};
  M.dof_names = trans;
  M.dof_names.insert(M.dof_names.end(), rot.begin(), rot.end());
  for (auto &s : M.dof_names) M.dof_ptrs.push_back(s.c_str());
  // material
  const std::string mp = ch + ".material";
  const std::string mtype = v.str(mp + ".type");
  dl_material_desc md{};
  if (mtype == "ElasticRod") md.type = DL_MAT_ELASTIC_ROD;
  else if (mtype == "ElastoPlasticRod") md.type = DL_MAT_ELASTOPLASTIC_ROD;
  else throw std::runtime_error("unsupported material type " + mtype);
  md.young = v.num(mp + ".young");
  if (v.has(mp + ".shear_modulus")) md.shear_modulus = v.num(mp + ".shear_modulus");
  else md.shear_modulus = md.young / 2.0 / (v.num(mp + ".poisson_ratio") + 1.0);
  const std::string cs = v.str(mp + ".cross_section", "");
  md.shear_correction = 5.0 / 6.0;
  if (cs == "circle") {
    const double r = v.num(mp + ".radius");
    md.circle = 1;
    md.radius = r;
    md.area = M_PI * r * r;
    md.area_moment[0] = md.area_moment[1] = M_PI * std::pow(r, 4) / 4.0;
    md.shear_correction = 9.0 / 10.0;
  } else if (cs == "square") {
    const double s = v.num(mp + ".side_length");
    md.area = s * s;
    md.area_moment[0] = md.area_moment[1] = std::pow(s, 4) / 12.0;
  } else if (cs == "rectangle") {
    const std::vector<double> sl = v.nums(mp + ".side_length");
    if (sl.size() != 2) throw std::runtime_error("A rectangle has only two sides!");
    md.area = sl[0] * sl[1];
    md.area_moment[0] = std::pow(sl[1], 3) * sl[0] / 12.0;
    md.area_moment[1] = std::pow(sl[0], 3) * sl[1] / 12.0;
  } else if (cs.empty()) {
    md.area = v.num(mp + ".area");
    const std::vector<double> am = v.nums(mp + ".area_moment");
    if (am.empty()) throw std::runtime_error(mp + ".area_moment is missing");
    md.area_moment[0] = am[0];
    md.area_moment[1] = am.size() > 1 ? am[1] : am[0];
  } else {
    throw std::runtime_error("unknown cross section, only 'rectangle', 'square' and 'circle' are supported");
  }
  md.polar_moment = v.num(mp + ".polar_moment", md.area_moment[0] + md.area_moment[1]);
  md.shear_correction = v.num(mp + ".shear_correction", md.shear_correction);
  md.density = v.num(mp + ".density", 0.0);
  md.inertia_correct = v.num(mp + ".inertia_correct", 1.0);
  if (md.type == DL_MAT_ELASTOPLASTIC_ROD) {
    M.strings.push_back(v.str(mp + ".yieldCond"));
    std::vector<std::string> der = v.strs(mp + ".yieldDeriv");
    const size_t first = M.strings.size();
    for (auto &d : der) M.strings.push_back(d);
    M.derivs.emplace_back();
    for (size_t k = 0; k < der.size(); ++k) M.derivs.back().push_back(nullptr);
    md.n_yield_deriv = static_cast<int32_t>(der.size());
    md.has_isotropic = v.has(mp + ".isotropicCoefficient") ? 1 : 0;
    md.isotropic_coefficient = v.num(mp + ".isotropicCoefficient", 0.0);
    if (v.has(mp + ".kinematicTensor")) {
      M.kin.push_back(v.nums(mp + ".kinematicTensor"));
      if (M.kin.back().size() != 36) throw std::runtime_error("kinematicTensor needs 36 values");
    }
    md.max_iter = static_cast<int32_t>(v.num(mp + ".maxIter", 20));
    md.precision = v.num(mp + ".precision", 1e-5);
    (void)first;
  }
  M.mats.push_back(md);
  // Gauss rule of the stiffness shape (Line3D default: Gauss(n-1))
  int G = nen - 1;
  for (const char *k : {".shape.intScheme", ".stiffShape.intScheme"}) {
    const std::string sch = v.str(ch + k, "");
    if (sch.rfind("Gauss", 0) == 0) G = std::atoi(sch.c_str() + 5);
  }
  if (v.has(ch + ".shape.numPoints")) G = static_cast<int>(v.num(ch + ".shape.numPoints"));
  if (G < 1 || G > 4) throw std::runtime_error("unsupported integration scheme");
  if (v.has(ch + ".material_ey")) {
    const std::vector<double> ey = v.nums(ch + ".material_ey");
    if (ey.size() != 3) throw std::runtime_error("material_ey needs three components");
    M.desc.has_material_ey = 1;
    for (int k = 0; k < 3; ++k) M.desc.material_ey[k] = ey[k];
  }
  if (v.has(ch + ".given_dir_nodes")) {
    for (double d : v.nums(ch + ".given_dir_nodes")) M.given_nodes.push_back(static_cast<int32_t>(d));
    M.given_dirs = v.nums(ch + ".given_dir_dirs");
    if (M.given_dirs.size() != 3 * M.given_nodes.size()) throw std::runtime_error("given_dir_dirs size mismatch");
  }
  // contact
  if (v.str(lat + ".contact.type") == "RodContact") {
    dl_contact_desc &c = M.desc.contact;
    c.enabled = 1;
    c.radius = v.num(lat + ".contact.radius");
    const double pen = v.num(lat + ".contact.penalty", 0.0);
    c.penalty_sts = v.num(lat + ".contact.penaltySTS", pen);
    c.penalty_nts = v.num(lat + ".contact.penaltyNTS", pen);
    c.margin = 2.0 * c.radius;
  }
  // joint contact (LatticeModel.cpp:99-101, JointContactModel.cpp:24-60):
  // the joints are the nodes of the element group "points"
  if (v.has(lat + ".jointContact.type")) {
    const std::string jt = v.str(lat + ".jointContact.type");
    if (jt != "JointContact") throw std::runtime_error(lat + ".jointContact.type: unsupported model type \"" + jt + "\"");
    dl_joint_contact_desc &j = M.desc.joint_contact;
    j.enabled = 1;
    j.radius = v.num(lat + ".jointContact.radius");
    j.penalty = v.num(lat + ".jointContact.penalty");
    auto it = egNodes.find("points");
    if (it == egNodes.end()) throw std::runtime_error(lat + ".jointContact: the mesh has no point elements (\"points\")");
    M.joints = it->second;
  }
  // ---- node groups (GroupInput) and "all"
  const std::string grp = find_typed(st, "GroupInput");
  if (!grp.empty())
    for (auto &g : v.strs(grp + ".nodeGroups")) M.groups[g] = node_group(v, grp + "." + g, M.coords, egNodes);
  {
    std::vector<int32_t> all(N);
    for (int i = 0; i < N; ++i) all[i] = i;
    M.groups["all"] = all;
  }
  for (auto &kv : egNodes) M.groups[kv.first] = kv.second;
  // ---- explicit module
  std::string integ;
  for (const char *t : {"LeapFrog", "MilneDevice", "EmbeddedRK", "Explicit"}) {
    integ = find_typed(st, t);
    if (!integ.empty()) {
      if (std::string(t) == "MilneDevice") {
        // ExplicitModule::configure (ExplicitModule.cpp:124-148); the JIVE
        // names of the dt bounds are not visible here: minDtime / maxDtime
        M.integ.kind = DL_INTEG_MILNE;
        M.integ.precision = v.num(integ + ".precision", kDefaultMilnePrecision);
        M.integ.min_dt = v.num(integ + ".minDtime", 0.0);
        M.integ.max_dt = v.num(integ + ".maxDtime", 0.0);
        M.integ.safety = v.num(integ + ".stepSaftey", 0.0);
        M.integ.increase = v.num(integ + ".increaseFactor", 0.0);
        M.integ.decrease = v.num(integ + ".decreaseFactor", 0.0);
        M.integ.length_scale = v.num(integ + ".lengthScale", 0.0);
      } else if (std::string(t) != "LeapFrog") {
        M.notes.push_back(std::string("integrator ") + t + " run as LeapFrog");
      }
      break;
    }
  }
  if (integ.empty()) throw std::runtime_error("no explicit integrator (LeapFrog/MilneDevice) in " + path);
  M.desc.dt = v.num(integ + ".deltaTime");
  // ExplicitModule rebuilds the mass matrix when updateWhen holds (default:
  // every step, ExplicitModule.cpp:121-126, 262-265); the engine forms the
  // rotational mass from the current rotation in every step
  if (v.has(integ + ".updateWhen")) {
    std::string uw = v.str(integ + ".updateWhen");
    uw.erase(0, uw.find_first_not_of(" \t"));
    uw.erase(uw.find_last_not_of(" \t") + 1);
    if (uw != "true" && uw != "1")
      M.notes.push_back(integ + ".updateWhen = \"" + uw + "\" not applied: the mass matrix is rebuilt every step");
  }
  M.desc.so3_update = v.has(integ + ".dofs_SO3") ? 1 : 0;
  M.desc.gyroscopic = 1;
  // ---- boundary-condition models, in the order of the Multi model's list
  std::string multi = find_typed(st, "Multi");
  std::vector<std::string> models;
  if (!multi.empty())
    for (auto &m : v.strs(multi + ".models")) models.push_back(multi + "." + m);
  struct PendingBc {
    int kind, dof;
    std::vector<int32_t> nodes;
    double factor;
    std::string scale;
  };
  std::vector<PendingBc> pend;
  std::function<void(const std::string &, const std::string &)> bcModel = [&](const std::string &m,
                                                                                const std::string &scale) {
    const std::string ty = v.str(m + ".type", "");
    if (ty == "LoadScale") {
      bcModel(m + ".model", v.str(m + ".scaleFunc", "1"));
      return;
    }
    if (ty == "Dirichlet" || ty == "Neumann") {
      const std::vector<std::string> gs = v.strs(m + ".nodeGroups"), ds = v.strs(m + ".dofs");
      std::vector<double> fs = v.nums(m + ".factors");
      if (ds.size() != gs.size()) throw std::runtime_error(m + ": dofs must have the same length as nodeGroups");
      if (fs.empty()) fs.assign(gs.size(), 0.0);
      if (ty == "Dirichlet" && !v.has(m + ".factors") && v.has(m + ".loaded"))
        fs[static_cast<size_t>(v.num(m + ".loaded"))] = 1.0;
      if (fs.size() != gs.size()) throw std::runtime_error(m + ": factors must have the same length as nodeGroups");
      std::string sc = scale;
      if (ty == "Dirichlet" && scale.empty()) {
        // DirichletModel.cpp:184-205: RATE (dispRate), INCREMENT (dispIncr), else unit
        if (v.has(m + ".dispRate")) {
          std::ostringstream os;
          os.precision(17);
          os << v.num(m + ".dispRate") << " * i * deltaTime";
          sc = os.str();
        } else if (v.has(m + ".dispIncr")) {
          std::ostringstream os;
          os.precision(17);
          os << v.num(m + ".initDisp", 0.0) << " + (i - 1) * " << v.num(m + ".dispIncr");
          sc = os.str();
        }
      }
      if (ty == "Neumann" && scale.empty()) {
        // NeumannModel.cpp:178-183, 365: initLoad + i * loadIncr
        std::ostringstream os;
        os.precision(17);
        os << v.num(m + ".initLoad", 0.0) << " + i * " << v.num(m + ".loadIncr", 0.0);
        sc = os.str();
      }
      for (size_t k = 0; k < gs.size(); ++k) {
        auto it = M.groups.find(gs[k]);
        if (it == M.groups.end()) throw std::runtime_error(m + ": unknown node group " + gs[k]);
        pend.push_back({ty == "Dirichlet" ? DL_BC_DIRICHLET : DL_BC_NEUMANN, dof_index(M.dof_names, ds[k]),
                        it->second, fs[k], sc});
      }
      return;
    }
    if (ty == "InitLoad") {
      for (const char *part : {"velo", "disp"}) {
        const std::string P = part;
        const std::vector<std::string> gs = v.strs(m + "." + P + "Groups"), ds = v.strs(m + "." + P + "Dofs");
        const std::vector<double> vs = v.nums(m + "." + P + "Vals");
        if (gs.size() != ds.size() || gs.size() != vs.size())
          throw std::runtime_error(m + ": " + P + "Groups/Dofs/Vals sizes differ");
        for (size_t k = 0; k < gs.size(); ++k) {
          auto it = M.groups.find(gs[k]);
          if (it == M.groups.end()) throw std::runtime_error(m + ": unknown node group " + gs[k]);
          pend.push_back({P == "velo" ? DL_BC_INIT_VELO : DL_BC_INIT_DISP, dof_index(M.dof_names, ds[k]),
                          it->second, vs[k], ""});
        }
      }
      return;
    }
    if (ty == "Mass") {  // MassModel (MassModel.cpp:24-36, 77-99): totalMass[i] spread over group i, on each DOF
      const std::vector<double> tm = v.nums(m + ".totalMass");
      const std::vector<std::string> gs = v.strs(m + ".nodeGroups"), ds = v.strs(m + ".dofs");
      if (tm.size() != gs.size()) throw std::runtime_error(m + ": NodeGroups and totalMass need to have the same length");
      for (size_t k = 0; k < gs.size(); ++k) {
        auto it = M.groups.find(gs[k]);
        if (it == M.groups.end()) throw std::runtime_error(m + ": unknown node group " + gs[k]);
        if (it->second.empty()) throw std::runtime_error(m + ": node group " + gs[k] + " is empty");
        for (const std::string &d : ds)
          pend.push_back({DL_BC_MASS, dof_index(M.dof_names, d), it->second,
                          tm[k] / static_cast<double>(it->second.size()), ""});
      }
      return;
    }
    if (ty == "None" || ty == "Lattice" || ty.empty()) return;
    M.notes.push_back("model " + m + " of type " + ty + " ignored");
  };
  for (auto &m : models) bcModel(m, "");
  for (auto &b : pend) {
    M.bc_nodes.push_back(b.nodes);
    M.strings.push_back(b.scale);
  }
  // strings are stable now: wire pointers
  size_t si = 0;
  if (md.type == DL_MAT_ELASTOPLASTIC_ROD) {
    M.mats[0].yield_cond = M.strings[0].c_str();
    for (int k = 0; k < M.mats[0].n_yield_deriv; ++k) M.derivs[0][k] = M.strings[1 + k].c_str();
    M.mats[0].yield_deriv = M.derivs[0].data();
    if (!M.kin.empty()) M.mats[0].kinematic_tensor = M.kin[0].data();
    si = 1 + M.mats[0].n_yield_deriv;
  }
  for (size_t k = 0; k < pend.size(); ++k) {
    dl_bc_desc b{};
    b.kind = pend[k].kind;
    b.dof = pend[k].dof;
    b.n_nodes = static_cast<int32_t>(M.bc_nodes[k].size());
    b.nodes = M.bc_nodes[k].data();
    b.factor = pend[k].factor;
    b.scale = M.strings[si + k].empty() ? nullptr : M.strings[si + k].c_str();
    M.bcs.push_back(b);
  }
  // ---- output modules (OutputModule chain of the .pro file)
  for (const std::string &name : v.strs("Output.modules")) {
    const std::string k = "Output." + name;
    ProOutput o;
    o.name = name;
    o.type = v.str(k + ".type");
    if (o.type == "GroupOutput") {
      o.node_groups = v.strs(k + ".nodeGroups");
      o.dofs = v.strs(k + ".dofs");
    } else if (o.type == "Sample") {
      o.file = v.str(k + ".file");
      o.data_sets = v.strs(k + ".dataSets");
      o.separator = v.str(k + ".separator", " ");
      o.when = v.str(k + ".sampleWhen", "");
    } else if (o.type == "CSVOutput") {
      o.file = v.str(k + ".file");
      o.vectors = v.strs(k + ".vectors");
      o.when = v.str(k + ".saveWhen", v.str(k + ".sampleWhen", ""));
    } else if (o.type == "ParaView") {
      o.format = v.str(k + ".output_format");
      o.when = v.str(k + ".sampleWhen", "");
      for (const std::string &g : v.strs(k + ".groups"))
      {
        for (const std::string &d : v.strs(k + "." + g + ".node_data")) {
          if (d != "fint" && d != "fext" && d != "fres")
            M.notes.push_back("ParaView node_data " + d + " not written (fint, fext and fres are)");
          o.node_data.push_back(d);
        }
        for (const std::string &d : v.strs(k + "." + g + ".el_data")) o.el_data.push_back(d);
      }
    } else {
      M.notes.push_back("output module " + name + " of type " + o.type + " ignored");
      continue;
    }
    M.outputs.push_back(o);
  }
  // ---- run length: control.runWhile "t <= T" / "t < T" / "i <= N" / "i < N"
  const std::string rw = v.str("control.runWhile", "");
  if (!rw.empty()) {
    std::string s;
    for (char c : rw)
      if (!std::isspace(static_cast<unsigned char>(c))) s += c;
    auto num_after = [&](size_t p) { return evalExpr(parseExpr(s.substr(p), {}).get(), nullptr); };
    if (s.rfind("t<=", 0) == 0) {
      M.t_end = num_after(3);
      M.steps = static_cast<int64_t>(std::floor(M.t_end / M.desc.dt + 1e-9));
    } else if (s.rfind("t<", 0) == 0) {
      M.t_end = num_after(2);
      M.steps = static_cast<int64_t>(std::ceil(M.t_end / M.desc.dt - 1e-9)) - 1;
    }
    else if (s.rfind("i<=", 0) == 0) M.steps = static_cast<int64_t>(num_after(3));
    else if (s.rfind("i<", 0) == 0) M.steps = static_cast<int64_t>(num_after(2)) - 1;
    else M.notes.push_back("control.runWhile not understood: " + rw);
  }
  // ---- rigid hinges: the rod model builds a HingeModel from its "hinges"
  // properties (SpecialCosseratRodModel.cpp:80-89), whose constructor splits
  // the rod (HingeModel::createHinges_, HingeModel.cpp:268-358): along each
  // rod, in element order, the first node of every element is copied and the
  // element takes the copy, then the last node of the last element; each
  // copy is tied to its original (HingeModel.cpp:172-199)
  if (v.has(ch + ".hinges.type")) {
    const std::string ht = v.str(ch + ".hinges.type");
    if (ht != "rigidHinge") throw std::runtime_error(ch + ".hinges.type: unsupported model type \"" + ht + "\"");
    const int R = M.elem_rod.empty() ? 0 : (*std::max_element(M.elem_rod.begin(), M.elem_rod.end()) + 1);
    std::vector<std::vector<int>> rodElems(R);
    for (size_t e = 0; e < M.elem_rod.size(); ++e) rodElems[M.elem_rod[e]].push_back(static_cast<int>(e));
    auto copy_node = [&](int32_t orig) {
      for (int k = 0; k < 3; ++k) M.coords.push_back(M.coords[static_cast<size_t>(orig) * 3 + k]);
      const int32_t nn = static_cast<int32_t>(M.coords.size() / 3) - 1;
      M.ties.push_back(orig);
      M.ties.push_back(nn);
      return nn;
    };
    for (auto &els : rodElems) {
      if (els.empty()) continue;
      for (int e : els) M.conn[static_cast<size_t>(e) * nen] = copy_node(M.conn[static_cast<size_t>(e) * nen]);
      const size_t last = static_cast<size_t>(els.back()) * nen + nen - 1;
      M.conn[last] = copy_node(M.conn[last]);
    }
    M.notes.push_back(ch + ".hinges: the reference's rod model creates the hinge model but passes it no actions "
                           "(the calls are commented out, SpecialCosseratRodModel.cpp:216-217, 302-303, 362-363, "
                           "396-397); the engine ties every copy to its original rigidly, as the hinge's "
                           "constraints do in an explicit run (zero plastic offset)");
    if (v.has(ch + ".hinges.yieldCond"))
      M.notes.push_back(ch + ".hinges.yieldCond: the hinge's plastic offsets change only in CHECK_COMMIT, which "
                             "explicit modules never issue; not applied");
  }
  // ---- description
  dl_model_desc &d = M.desc;
  d.n_nodes = static_cast<int32_t>(M.coords.size() / 3);
  d.coords = M.coords.data();
  d.n_elems = static_cast<int32_t>(M.elem_rod.size());
  d.nodes_per_elem = nen;
  d.conn = M.conn.data();
  d.elem_rod = M.elem_rod.data();
  d.n_rods = M.elem_rod.empty() ? 0 : (*std::max_element(M.elem_rod.begin(), M.elem_rod.end()) + 1);
  d.n_materials = 1;
  d.materials = M.mats.data();
  d.dof_names = M.dof_ptrs.data();
  d.n_gauss = G;
  d.n_given_dirs = static_cast<int32_t>(M.given_nodes.size());
  d.given_dir_nodes = M.given_nodes.empty() ? nullptr : M.given_nodes.data();
  d.given_dirs = M.given_dirs.empty() ? nullptr : M.given_dirs.data();
  d.n_bcs = static_cast<int32_t>(M.bcs.size());
  d.bcs = M.bcs.data();
  d.joint_contact.n_joints = static_cast<int32_t>(M.joints.size());
  d.joint_contact.joints = M.joints.empty() ? nullptr : M.joints.data();
  d.n_ties = static_cast<int32_t>(M.ties.size() / 2);
  d.ties = M.ties.empty() ? nullptr : M.ties.data();
  return pm;
}

}  // namespace dl
