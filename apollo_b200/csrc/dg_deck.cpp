// Apollo input-deck text (".pin" cryptset blocks) to the plugin calls of the C ABI.
//
// Apollo configures its sub-solver from nested cryptset blocks: the
// nodalDG2d block holds polynomialOrder, cfl, and the lists Equations,
// boundaryConditions and Limiter, each naming a block whose Kind selects the
// plugin and whose keys are that plugin's parameters
// (WxNodalDG2dMethod::setup, src/subsolvers/wxnodaldg2dmethod.cc:50-152;
// WxHyperbolicEqnSet::setup, src/hyper/wxhyperboliceqnset.cc:43-89; the
// plugins' setup(): wxeulereqn.cc:18-89, wxadvectioneqn.cc:12-30,
// wxphmaxwelleqn.cc:12-30, the BCs' setup() in src/hyperapps/*/*bc.cc, the
// limiter's wxhesthavenwarburtoneulerlimiter.cc:18-30).  A deck starts with a
// Python preamble (NAME = expression lines) whose names the blocks may use
// ("c0 = LIGHT", "cfl = 0.5/((2.*(P_ORDER+1)-1))").
//
// This file reads that text: blocks <name> ... </name>, "key = value" lines
// (with '\' continuations and '#' comments), values that are numbers,
// arithmetic over the preamble's names (+ - * / ** ^, parentheses), quoted or
// bare strings, and [lists].  Keys keep Apollo's names and defaults; a key
// written after a sub-block of its block is not read, as in Apollo.
#include <cctype>
#include <cmath>
#include <cstring>
#include <map>
#include <string>
#include <vector>

#include "apollo_dg.h"

namespace {

struct Block {
  std::string name;
  std::vector<std::pair<std::string, std::string>> kv;  // in deck order
  std::vector<Block> sub;
  const std::string* get(const std::string& k) const {
    for (const auto& p : kv)
      if (p.first == k) return &p.second;
    return nullptr;
  }
};

std::string trim(const std::string& s) {
  size_t a = 0, b = s.size();
  while (a < b && std::isspace((unsigned char)s[a])) ++a;
  while (b > a && std::isspace((unsigned char)s[b - 1])) --b;
  return s.substr(a, b - a);
}

// ---- arithmetic over numbers and preamble names
struct Expr {
  const std::string& s;
  const std::map<std::string, double>& defs;
  size_t i = 0;
  bool ok = true;
  Expr(const std::string& s_, const std::map<std::string, double>& d) : s(s_), defs(d) {}
  void ws() {
    while (i < s.size() && std::isspace((unsigned char)s[i])) ++i;
  }
  bool eat(const char* t) {
    ws();
    const size_t n = std::strlen(t);
    if (s.compare(i, n, t) == 0) {
      i += n;
      return true;
    }
    return false;
  }
  double primary() {
    ws();
    if (eat("(")) {
      const double v = sum();
      if (!eat(")")) ok = false;
      return v;
    }
    if (eat("-")) return -power();
    if (eat("+")) return power();
    if (i < s.size() && (std::isdigit((unsigned char)s[i]) || s[i] == '.')) {
      const char* b = s.c_str() + i;
      char* e = nullptr;
      const double v = std::strtod(b, &e);
      if (e == b) { ok = false; return 0.0; }
      i += (size_t)(e - b);
      return v;
    }
    size_t j = i;
    while (j < s.size() && (std::isalnum((unsigned char)s[j]) || s[j] == '_' || s[j] == '.')) ++j;
    if (j == i) { ok = false; return 0.0; }
    const std::string name = s.substr(i, j - i);
    i = j;
    auto it = defs.find(name);
    if (it != defs.end()) return it->second;
    if (name == "math.pi" || name == "pi" || name == "PI") return 3.14159265358979323846;
    ok = false;
    return 0.0;
  }
  double power() {
    const double b = primary();
    if (eat("**") || eat("^")) return std::pow(b, power());
    return b;
  }
  double product() {
    double v = power();
    for (;;) {
      ws();
      if (i + 1 < s.size() && s[i] == '*' && s[i + 1] == '*') break;  // handled by power()
      if (eat("*")) v *= power();
      else if (eat("/")) v /= power();
      else break;
    }
    return v;
  }
  double sum() {
    double v = product();
    for (;;) {
      if (eat("+")) v += product();
      else if (eat("-")) v -= product();
      else break;
    }
    return v;
  }
};

bool eval_number(const std::string& text, const std::map<std::string, double>& defs, double* out) {
  Expr e(text, defs);
  const double v = e.sum();
  e.ws();
  if (!e.ok || e.i != text.size()) return false;
  *out = v;
  return true;
}

std::string unquote(const std::string& v0) {
  const std::string v = trim(v0);
  if (v.size() >= 2 && (v[0] == '\'' || v[0] == '"') && v.back() == v[0]) return v.substr(1, v.size() - 2);
  return v;
}

std::vector<std::string> list_items(const std::string& v0) {
  std::vector<std::string> out;
  std::string v = trim(v0);
  if (v.size() < 2 || v[0] != '[' || v.back() != ']') return out;
  v = v.substr(1, v.size() - 2);
  size_t a = 0;
  while (a <= v.size()) {
    size_t b = v.find(',', a);
    if (b == std::string::npos) b = v.size();
    const std::string it = unquote(v.substr(a, b - a));
    if (!it.empty()) out.push_back(it);
    a = b + 1;
  }
  return out;
}

struct Deck {
  Block root;
  std::map<std::string, double> defs;
  std::string err;
};

// Parses the deck; false with d.err set on malformed structure.
bool parse(const char* text, Deck& d) {
  if (!text) {
    d.err = "no text";
    return false;
  }
  // logical lines: comments cut, '\' continuations joined
  std::vector<std::string> lines;
  std::string cur;
  const std::string all(text);
  size_t p = 0;
  while (p <= all.size()) {
    size_t e = all.find('\n', p);
    if (e == std::string::npos) e = all.size();
    std::string ln = all.substr(p, e - p);
    p = e + 1;
    // '#' starts a comment unless inside quotes
    bool q1 = false, q2 = false;
    for (size_t i = 0; i < ln.size(); ++i) {
      if (ln[i] == '\'' && !q2) q1 = !q1;
      else if (ln[i] == '"' && !q1) q2 = !q2;
      else if (ln[i] == '#' && !q1 && !q2) { ln.resize(i); break; }
    }
    ln = trim(ln);
    if (!ln.empty() && ln.back() == '\\') {
      cur += ln.substr(0, ln.size() - 1) + " ";
      continue;
    }
    cur += ln;
    if (!trim(cur).empty()) lines.push_back(trim(cur));
    cur.clear();
    if (e == all.size()) break;
  }
  std::vector<Block*> stack{&d.root};
  for (const std::string& ln : lines) {
    if (ln.size() >= 3 && ln[0] == '<' && ln.back() == '>') {
      if (ln[1] == '/') {
        const std::string nm = trim(ln.substr(2, ln.size() - 3));
        if (stack.size() < 2 || stack.back()->name != nm) {
          d.err = "unbalanced </" + nm + ">";
          return false;
        }
        stack.pop_back();
      } else {
        Block b;
        b.name = trim(ln.substr(1, ln.size() - 2));
        stack.back()->sub.push_back(b);
        stack.push_back(&stack.back()->sub.back());
      }
      continue;
    }
    if (ln.compare(0, 7, "import ") == 0 || ln.compare(0, 5, "from ") == 0) continue;
    const size_t eq = ln.find('=');
    if (eq == std::string::npos || eq == 0) continue;  // a line without '=' carries no key
    const std::string k = trim(ln.substr(0, eq)), v = trim(ln.substr(eq + 1));
    if (stack.size() == 1) {
      // the Python preamble (and top-level keys): numeric names become definitions
      double x;
      if (eval_number(v, d.defs, &x)) d.defs[k] = x;
    }
    // Apollo's reader does not see a key written after a sub-block of the
    // same block (each nested parse runs on its own copy of the lexer,
    // WxCryptSet::_WxParser::wx_decl_value, src/lib/wxcryptset.cc:337-367):
    // such a key is dropped here too, so a deck configures the same plugins
    if (stack.size() > 1 && !stack.back()->sub.empty()) continue;
    stack.back()->kv.emplace_back(k, v);
  }
  if (stack.size() != 1) {
    d.err = "block <" + stack.back()->name + "> not closed";
    return false;
  }
  return true;
}

const Block* find_block(const Block& b, const std::string& name) {
  for (const Block& s : b.sub) {
    if (s.name == name) return &s;
    if (const Block* r = find_block(s, name)) return r;
  }
  return nullptr;
}
// the first block (depth first) holding key k
const Block* find_with_key(const Block& b, const std::string& k) {
  if (b.get(k)) return &b;
  for (const Block& s : b.sub)
    if (const Block* r = find_with_key(s, k)) return r;
  return nullptr;
}
const Block* find_type(const Block& b, const std::string& type) {
  for (const Block& s : b.sub) {
    const std::string* t = s.get("Type");
    if (t && unquote(*t) == type) return &s;
    if (const Block* r = find_type(s, type)) return r;
  }
  return nullptr;
}

struct ParamSpec {
  const char* name;
  bool required;
  double dflt;
};
struct KindSpec {
  const char* kind;
  std::vector<ParamSpec> params;
};

const std::vector<KindSpec>& equation_kinds() {
  static const std::vector<KindSpec> k = {
      {"advectionEqn", {{"ux", false, 0.0}, {"uy", false, 0.0}, {"uz", false, 0.0}}},
      {"eulerEqn", {{"gas_gamma", true, 0.0}, {"minPressure", false, 0.0}, {"minDensity", false, 0.0}}},
      {"eulerEqn2d", {{"gas_gamma", true, 0.0}, {"minPressure", false, 0.0}, {"minDensity", false, 0.0}}},
      {"phMaxwellEqn", {{"c0", true, 0.0}, {"gamma", false, 0.0}, {"chi", false, 0.0}}},
      {"maxwellTM", {{"c0", true, 0.0}}},
  };
  return k;
}
const std::vector<KindSpec>& bc_kinds() {
  static const std::vector<KindSpec> k = {
      {"gridFixedBC", {{"value", true, 0.0}}},
      {"isentropicVortexBC",
       {{"u0", true, 0.0}, {"v0", true, 0.0}, {"x0", true, 0.0}, {"y0", true, 0.0}, {"gas_gamma", true, 0.0},
        {"beta", true, 0.0}}},
      {"maxwellTransverseMagneticBC", {}},
      {"phmConductingWallBC", {}},
      {"eulerWallBC", {}},
      {"eulerZeroGradientBC", {}},
      {"eulerInflowBC",
       {{"Mach_number", true, 0.0}, {"Flow_angle", true, 0.0}, {"gas_gamma", true, 0.0}, {"Pressure", true, 0.0},
        {"density", true, 0.0}}},
      {"eulerDirichletBC",
       {{"density", true, 0.0}, {"xvelocity", true, 0.0}, {"yvelocity", true, 0.0}, {"zvelocity", true, 0.0},
        {"gas_gamma", true, 0.0}, {"pressure", true, 0.0}}},
  };
  return k;
}
const std::vector<KindSpec>& source_kinds() {
  static const std::vector<KindSpec> k = {
      {"tranverseMagneticSrc", {}},
      {"pointCurrentSrc",
       {{"xLocation", true, 0.0}, {"yLocation", true, 0.0}, {"radius", true, 0.0}, {"currentDensity", true, 0.0},
        {"frequency", true, 0.0}, {"phase", true, 0.0}, {"charge", true, 0.0}, {"mass", true, 0.0},
        {"epsilon0", true, 0.0}}},
  };
  return k;
}
const std::vector<KindSpec>& limiter_kinds() {
  static const std::vector<KindSpec> k = {
      {"eulerLimiterHW", {{"gas_gamma", true, 0.0}, {"min_pressure", true, 0.0}, {"min_density", true, 0.0}}},
      {"tuAliabadiLimiter", {}},
  };
  return k;
}

// The parameters of `kind` from block b, in the C ABI's order.
bool block_params(const Block& b, const std::string& kind, const std::vector<KindSpec>& kinds, const Deck& d,
                  std::vector<double>& out, std::string& err) {
  const KindSpec* ks = nullptr;
  for (const KindSpec& k : kinds)
    if (kind == k.kind) ks = &k;
  if (!ks) {
    err = "unknown Kind " + kind;
    return false;
  }
  out.clear();
  for (const ParamSpec& p : ks->params) {
    const std::string* v = b.get(p.name);
    if (!v) {
      if (p.required) {
        err = kind + ": missing " + p.name;
        return false;
      }
      out.push_back(p.dflt);
      continue;
    }
    double x;
    if (!eval_number(*v, d.defs, &x)) {
      err = kind + ": " + p.name + " = " + *v + " is not a number";
      return false;
    }
    out.push_back(x);
  }
  return true;
}

// The block a list key names (its first entry, or entry `idx`) or, without the
// list, a block of the given Type, or the deck's top level when it has a Kind.
const Block* listed_block(const Deck& d, const char* list_key, const char* type, int idx, int* count,
                          std::string& err) {
  if (const Block* holder = find_with_key(d.root, list_key)) {
    const std::vector<std::string> items = list_items(*holder->get(list_key));
    if (count) *count = (int)items.size();
    if (items.empty()) {
      err = std::string(list_key) + " is not a list of block names";
      return nullptr;
    }
    if (idx >= (int)items.size()) return nullptr;
    const Block* b = find_block(d.root, items[idx]);
    if (!b) err = "no block <" + items[idx] + "> for " + list_key;
    return b;
  }
  if (count) *count = 1;
  if (idx > 0) return nullptr;
  if (d.root.get("Kind")) return &d.root;
  const Block* b = find_type(d.root, type);
  if (!b && d.root.sub.size() == 1) b = &d.root.sub[0];
  if (!b && !d.root.kv.empty()) b = &d.root;
  if (!b) err = std::string("no ") + list_key + " list and no block of Type " + type;
  return b;
}

void copy_err(const std::string& e, char* err, int err_len) {
  if (err && err_len > 0) {
    std::strncpy(err, e.c_str(), (size_t)err_len - 1);
    err[err_len - 1] = '\0';
  }
}

}  // namespace

extern "C" {

apollo_status apollo_dg_deck_config(const char* text, apollo_dg_config* cfg, char* err, int err_len) {
  if (!text || !cfg) return APOLLO_ERR_ARG;
  Deck d;
  if (!parse(text, d)) {
    copy_err(d.err, err, err_len);
    return APOLLO_ERR_CONFIG;
  }
  // the nodalDG2d block, else whichever block holds polynomialOrder
  const Block* b = nullptr;
  std::vector<const Block*> todo{&d.root};
  while (!todo.empty() && !b) {
    const Block* x = todo.back();
    todo.pop_back();
    const std::string* k = x->get("Kind");
    if (k && unquote(*k) == "nodalDG2d") b = x;
    for (const Block& s : x->sub) todo.push_back(&s);
  }
  if (!b) b = find_with_key(d.root, "polynomialOrder");
  if (!b || !b->get("polynomialOrder") || !b->get("cfl")) {
    copy_err("no block with polynomialOrder and cfl", err, err_len);
    return APOLLO_ERR_CONFIG;
  }
  double n = 0, c = 0;
  if (!eval_number(*b->get("polynomialOrder"), d.defs, &n) || !eval_number(*b->get("cfl"), d.defs, &c) ||
      n != std::floor(n)) {
    copy_err("polynomialOrder or cfl is not a number", err, err_len);
    return APOLLO_ERR_CONFIG;
  }
  cfg->polynomial_order = (int)n;
  cfg->cfl = c;
  return APOLLO_OK;
}

apollo_status apollo_dg_deck_equation(const char* kind, const char* text, char* kind_out, int kind_len,
                                      double* params, int* nparams, char* flux_out, int flux_len, char* err,
                                      int err_len) {
  if (!text || !params || !nparams) return APOLLO_ERR_ARG;
  Deck d;
  if (!parse(text, d)) {
    copy_err(d.err, err, err_len);
    return APOLLO_ERR_CONFIG;
  }
  std::string e;
  int count = 0;
  const Block* b = kind ? (d.root.sub.size() == 1 && d.root.kv.empty() ? &d.root.sub[0] : &d.root)
                        : listed_block(d, "Equations", "WxHyperbolicEqn", 0, &count, e);
  if (!b) {
    copy_err(e, err, err_len);
    return APOLLO_ERR_CONFIG;
  }
  if (count > 1) {
    copy_err("Equations lists more than one equation; this library takes one per handle", err, err_len);
    return APOLLO_ERR_CONFIG;
  }
  std::string k = kind ? std::string(kind) : (b->get("Kind") ? unquote(*b->get("Kind")) : std::string());
  std::vector<double> v;
  if (!block_params(*b, k, equation_kinds(), d, v, e)) {
    copy_err(e, err, err_len);
    return APOLLO_ERR_CONFIG;
  }
  for (size_t i = 0; i < v.size(); ++i) params[i] = v[i];
  *nparams = (int)v.size();
  if (kind_out && kind_len > 0) copy_err(k, kind_out, kind_len);
  const std::string* nf = b->get("Numerical_Flux");
  if (flux_out && flux_len > 0) copy_err(nf ? unquote(*nf) : std::string("LF"), flux_out, flux_len);
  return APOLLO_OK;
}

apollo_status apollo_dg_deck_bc(const char* kind, const char* text, int index, int* count, char* kind_out,
                                int kind_len, double* params, int* nparams, char* err, int err_len) {
  if (!text || !count) return APOLLO_ERR_ARG;
  Deck d;
  if (!parse(text, d)) {
    copy_err(d.err, err, err_len);
    return APOLLO_ERR_CONFIG;
  }
  std::string e;
  const Block* b = nullptr;
  if (kind) {
    *count = 1;
    b = (d.root.sub.size() == 1 && d.root.kv.empty()) ? &d.root.sub[0] : &d.root;
    if (index > 0) b = nullptr;
  } else if (const Block* holder = find_with_key(d.root, "Equations")) {
    // a sub-solver deck: its boundaryConditions list (none: no conditions;
    // the limiter block has a list of its own)
    const std::string* lst = holder->get("boundaryConditions");
    const std::vector<std::string> items = lst ? list_items(*lst) : std::vector<std::string>();
    *count = (int)items.size();
    if (index < (int)items.size()) {
      b = find_block(d.root, items[index]);
      if (!b) e = "no block <" + items[index] + "> for boundaryConditions";
    }
  } else {
    // one condition's block: the text's keys, or its only block
    *count = 1;
    if (d.root.get("Kind")) b = &d.root;
    else if (d.root.sub.size() == 1) b = &d.root.sub[0];
    else e = "no Equations list and no single boundary-condition block";
    if (index > 0) b = nullptr;
  }
  if (index >= *count) return APOLLO_OK;  // only the count was asked for
  if (!b) {
    copy_err(e, err, err_len);
    return APOLLO_ERR_CONFIG;
  }
  const std::string k = kind ? std::string(kind) : (b->get("Kind") ? unquote(*b->get("Kind")) : std::string());
  std::vector<double> v;
  if (!block_params(*b, k, bc_kinds(), d, v, e)) {
    copy_err(e, err, err_len);
    return APOLLO_ERR_CONFIG;
  }
  if (params)
    for (size_t i = 0; i < v.size(); ++i) params[i] = v[i];
  if (nparams) *nparams = (int)v.size();
  if (kind_out && kind_len > 0) copy_err(k, kind_out, kind_len);
  return APOLLO_OK;
}

apollo_status apollo_dg_deck_source(const char* kind, const char* text, int index, int* count, char* kind_out,
                                    int kind_len, int* out_range, int* nout, double* params, int* nparams, char* err,
                                    int err_len) {
  if (!text || !count) return APOLLO_ERR_ARG;
  Deck d;
  if (!parse(text, d)) {
    copy_err(d.err, err, err_len);
    return APOLLO_ERR_CONFIG;
  }
  std::string e;
  const Block* b = nullptr;
  if (kind) {
    *count = 1;
    b = (d.root.sub.size() == 1 && d.root.kv.empty()) ? &d.root.sub[0] : &d.root;
    if (index > 0) b = nullptr;
  } else if (const Block* holder = find_with_key(d.root, "Equations")) {
    // the sub-solver's Sources list (none: no sources)
    const std::string* lst = holder->get("Sources");
    const std::vector<std::string> items = lst ? list_items(*lst) : std::vector<std::string>();
    *count = (int)items.size();
    if (index < (int)items.size()) {
      b = find_block(d.root, items[index]);
      if (!b) e = "no block <" + items[index] + "> for Sources";
    }
  } else {
    *count = 1;
    if (d.root.get("Kind")) b = &d.root;
    else if (d.root.sub.size() == 1) b = &d.root.sub[0];
    else e = "no Equations list and no single source block";
    if (index > 0) b = nullptr;
  }
  if (index >= *count) return APOLLO_OK;
  if (!b) {
    copy_err(e, err, err_len);
    return APOLLO_ERR_CONFIG;
  }
  const std::string k = kind ? std::string(kind) : (b->get("Kind") ? unquote(*b->get("Kind")) : std::string());
  std::vector<double> v;
  if (!block_params(*b, k, source_kinds(), d, v, e)) {
    copy_err(e, err, err_len);
    return APOLLO_ERR_CONFIG;
  }
  const std::string* orng = b->get("OutRange");
  const std::vector<std::string> outs = orng ? list_items(*orng) : std::vector<std::string>();
  if (outs.empty()) {
    copy_err(k + ": missing OutRange", err, err_len);
    return APOLLO_ERR_CONFIG;
  }
  if (out_range && nout) {
    int n = 0;
    for (const std::string& o : outs) {
      double x;
      if (!eval_number(o, d.defs, &x) || x != std::floor(x) || x < 0) {
        copy_err(k + ": OutRange entry " + o + " is not a field index", err, err_len);
        return APOLLO_ERR_CONFIG;
      }
      if (n < 8) out_range[n++] = (int)x;
    }
    *nout = n;
  }
  if (params)
    for (size_t i = 0; i < v.size(); ++i) params[i] = v[i];
  if (nparams) *nparams = (int)v.size();
  if (kind_out && kind_len > 0) copy_err(k, kind_out, kind_len);
  return APOLLO_OK;
}

apollo_status apollo_dg_deck_limiter(const char* kind, const char* text, char* kind_out, int kind_len,
                                     double* params, int* nparams, char* err, int err_len) {
  if (!text || !params || !nparams) return APOLLO_ERR_ARG;
  Deck d;
  if (!parse(text, d)) {
    copy_err(d.err, err, err_len);
    return APOLLO_ERR_CONFIG;
  }
  std::string e;
  int count = 0;
  const Block* b = kind ? (d.root.sub.size() == 1 && d.root.kv.empty() ? &d.root.sub[0] : &d.root)
                        : (find_with_key(d.root, "Limiter") ? listed_block(d, "Limiter", "ApSubSolver", 0, &count, e)
                                                            : nullptr);
  if (!b) {
    if (!kind && e.empty()) {  // no Limiter list: no limiter
      *nparams = 0;
      if (kind_out && kind_len > 0) kind_out[0] = '\0';
      return APOLLO_OK;
    }
    copy_err(e, err, err_len);
    return APOLLO_ERR_CONFIG;
  }
  const std::string k = kind ? std::string(kind) : (b->get("Kind") ? unquote(*b->get("Kind")) : std::string());
  std::vector<double> v;
  if (!block_params(*b, k, limiter_kinds(), d, v, e)) {
    copy_err(e, err, err_len);
    return APOLLO_ERR_CONFIG;
  }
  for (size_t i = 0; i < v.size(); ++i) params[i] = v[i];
  *nparams = (int)v.size();
  if (kind_out && kind_len > 0) copy_err(k, kind_out, kind_len);
  return APOLLO_OK;
}

}  // extern "C"

namespace apollo {
void handle_set_error(apollo_dg* h, const char* msg);
}

extern "C" {

apollo_status apollo_dg_set_equation_text(apollo_dg* h, const char* kind, const char* text) {
  if (!h || !text) return APOLLO_ERR_ARG;
  char k[64], nf[32], err[256];
  double p[8];
  int np = 0;
  apollo_status r = apollo_dg_deck_equation(kind, text, k, sizeof k, p, &np, nf, sizeof nf, err, sizeof err);
  if (r) {
    apollo::handle_set_error(h, err);
    return r;
  }
  r = apollo_dg_set_equation(h, k, p, np);
  if (r) return r;
  return apollo_dg_set_numerical_flux(h, nf);
}

apollo_status apollo_dg_add_bc_text(apollo_dg* h, const char* kind, const char* text) {
  if (!h || !text) return APOLLO_ERR_ARG;
  char k[64], err[256];
  double p[8];
  int count = 0, np = 0;
  apollo_status r = apollo_dg_deck_bc(kind, text, 0, &count, nullptr, 0, nullptr, nullptr, err, sizeof err);
  if (r) {
    apollo::handle_set_error(h, err);
    return r;
  }
  for (int i = 0; i < count; ++i) {
    r = apollo_dg_deck_bc(kind, text, i, &count, k, sizeof k, p, &np, err, sizeof err);
    if (r) {
      apollo::handle_set_error(h, err);
      return r;
    }
    r = apollo_dg_add_bc(h, k, p, np);
    if (r) return r;
  }
  return APOLLO_OK;
}

apollo_status apollo_dg_add_source_text(apollo_dg* h, const char* kind, const char* text) {
  if (!h || !text) return APOLLO_ERR_ARG;
  char k[64], err[256];
  double p[9];
  int count = 0, np = 0, outs[8], nout = 0;
  apollo_status r = apollo_dg_deck_source(kind, text, 0, &count, nullptr, 0, nullptr, nullptr, nullptr, nullptr, err,
                                          sizeof err);
  if (r) {
    apollo::handle_set_error(h, err);
    return r;
  }
  for (int i = 0; i < count; ++i) {
    r = apollo_dg_deck_source(kind, text, i, &count, k, sizeof k, outs, &nout, p, &np, err, sizeof err);
    if (r) {
      apollo::handle_set_error(h, err);
      return r;
    }
    r = apollo_dg_add_source(h, k, outs, nout, p, np);
    if (r) return r;
  }
  return APOLLO_OK;
}

apollo_status apollo_dg_set_limiter_text(apollo_dg* h, const char* kind, const char* text) {
  if (!h || !text) return APOLLO_ERR_ARG;
  char k[64], err[256];
  double p[8];
  int np = 0;
  apollo_status r = apollo_dg_deck_limiter(kind, text, k, sizeof k, p, &np, err, sizeof err);
  if (r) {
    apollo::handle_set_error(h, err);
    return r;
  }
  return apollo_dg_set_limiter(h, k[0] ? k : nullptr, p, np);
}

}  // extern "C"
