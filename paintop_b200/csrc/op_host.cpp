// op_host.cpp -- C++ host side of the `cuda` backend, mirroring the reference's
// operator interface for the two Poisson ops and the two mask generators
// whose output they consume (mask.ellipse@1, mask.polygon@1).
//
// The reference's op body is `OpImplementation::compute(&InputValues, &Value)`
// (crates/paintop-core/src/executor/op_impl.rs:51-70), implemented by
// PoissonBlend (crates/paintop-cpu/src/poisson_blend.rs:534-600) and
// ScreenedPoisson (crates/paintop-cpu/src/screened_poisson.rs:361-430). This file
// restates that body in C++ -- the same validation order, the same error
// classes, codes and messages, the same defaults, the same SolverData mapping --
// and hands the numerical work to pt_poisson_solve. It is exported as
// pt_op_compute so a Rust FFI crate (or a test harness) can drive the op through
// the C ABI.
#include <cctype>
#include <cerrno>
#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <map>
#include <string>
#include <vector>

#include "../../include/paintop_cuda.h"
#include "abi_guard.h"

namespace pt_op {

// ---------------------------------------------------------------------------
// a minimal JSON reader: enough of serde_json's Value to read op params
// ---------------------------------------------------------------------------
struct JsonNumber {
  enum Kind { PosInt, NegInt, Float } kind = Float;
  uint64_t u = 0;
  int64_t i = 0;
  double f = 0.0;
};

struct JsonValue {
  enum Type { Null, Bool, Number, String, Array, Object } type = Null;
  bool b = false;
  JsonNumber num;
  std::string str;
  std::string lexeme;  // source text, for error context
  std::map<std::string, JsonValue> members;
  std::vector<JsonValue> items;  // array elements, in order

  // serde_json::Value::as_u64
  bool as_u64(uint64_t *out) const {
    if (type != Number || num.kind != JsonNumber::PosInt) return false;
    *out = num.u;
    return true;
  }
  // serde_json::Value::as_f64
  bool as_f64(double *out) const {
    if (type != Number) return false;
    switch (num.kind) {
      case JsonNumber::PosInt: *out = (double)num.u; break;
      case JsonNumber::NegInt: *out = (double)num.i; break;
      default: *out = num.f; break;
    }
    return true;
  }
  const JsonValue *get(const char *key) const {
    if (type != Object) return nullptr;
    auto it = members.find(key);
    return it == members.end() ? nullptr : &it->second;
  }
};

class JsonParser {
 public:
  explicit JsonParser(const char *s) : s_(s), p_(s) {}
  bool parse(JsonValue *v) {
    ws();
    if (!value(v, 0)) return false;
    ws();
    return *p_ == '\0';
  }

 private:
  const char *s_;
  const char *p_;
  void ws() {
    while (*p_ == ' ' || *p_ == '\t' || *p_ == '\n' || *p_ == '\r') ++p_;
  }
  bool lit(const char *w) {
    size_t n = std::strlen(w);
    if (std::strncmp(p_, w, n) != 0) return false;
    p_ += n;
    return true;
  }
  bool string(std::string *out) {
    if (*p_ != '"') return false;
    ++p_;
    while (*p_ && *p_ != '"') {
      if (*p_ == '\\') {
        ++p_;
        switch (*p_) {
          case '"': out->push_back('"'); break;
          case '\\': out->push_back('\\'); break;
          case '/': out->push_back('/'); break;
          case 'b': out->push_back('\b'); break;
          case 'f': out->push_back('\f'); break;
          case 'n': out->push_back('\n'); break;
          case 'r': out->push_back('\r'); break;
          case 't': out->push_back('\t'); break;
          case 'u': {
            for (int k = 1; k <= 4; ++k)
              if (!std::isxdigit((unsigned char)p_[k])) return false;
            out->push_back('?');
            p_ += 4;
          } break;
          default: return false;
        }
        ++p_;
      } else {
        out->push_back(*p_++);
      }
    }
    if (*p_ != '"') return false;
    ++p_;
    return true;
  }
  bool number(JsonValue *v) {
    const char *st = p_;
    bool neg = false, is_float = false;
    if (*p_ == '-') { neg = true; ++p_; }
    if (!std::isdigit((unsigned char)*p_)) return false;
    if (*p_ == '0') ++p_;
    else while (std::isdigit((unsigned char)*p_)) ++p_;
    if (*p_ == '.') {
      is_float = true;
      ++p_;
      if (!std::isdigit((unsigned char)*p_)) return false;
      while (std::isdigit((unsigned char)*p_)) ++p_;
    }
    if (*p_ == 'e' || *p_ == 'E') {
      is_float = true;
      ++p_;
      if (*p_ == '+' || *p_ == '-') ++p_;
      if (!std::isdigit((unsigned char)*p_)) return false;
      while (std::isdigit((unsigned char)*p_)) ++p_;
    }
    v->type = JsonValue::Number;
    v->lexeme.assign(st, p_);
    if (!is_float) {
      errno = 0;
      if (!neg) {
        unsigned long long u = std::strtoull(v->lexeme.c_str(), nullptr, 10);
        if (errno == 0) { v->num.kind = JsonNumber::PosInt; v->num.u = u; return true; }
      } else {
        long long i = std::strtoll(v->lexeme.c_str(), nullptr, 10);
        if (errno == 0) { v->num.kind = JsonNumber::NegInt; v->num.i = i; return true; }
      }
    }
    // serde_json parses fractions, exponents and out-of-range integers as f64
    v->num.kind = JsonNumber::Float;
    v->num.f = std::strtod(v->lexeme.c_str(), nullptr);
    return std::isfinite(v->num.f);
  }
  bool value(JsonValue *v, int depth) {
    if (depth > 64) return false;
    ws();
    const char *st = p_;
    if (*p_ == '{') {
      v->type = JsonValue::Object;
      ++p_;
      ws();
      if (*p_ == '}') { ++p_; v->lexeme.assign(st, p_); return true; }
      for (;;) {
        ws();
        std::string key;
        if (!string(&key)) return false;
        ws();
        if (*p_ != ':') return false;
        ++p_;
        JsonValue child;
        if (!value(&child, depth + 1)) return false;
        v->members[key] = std::move(child);
        ws();
        if (*p_ == ',') { ++p_; continue; }
        if (*p_ == '}') { ++p_; break; }
        return false;
      }
      v->lexeme.assign(st, p_);
      return true;
    }
    if (*p_ == '[') {
      v->type = JsonValue::Array;
      ++p_;
      ws();
      if (*p_ == ']') { ++p_; v->lexeme.assign(st, p_); return true; }
      for (;;) {
        JsonValue child;
        if (!value(&child, depth + 1)) return false;
        v->items.push_back(std::move(child));
        ws();
        if (*p_ == ',') { ++p_; continue; }
        if (*p_ == ']') { ++p_; break; }
        return false;
      }
      v->lexeme.assign(st, p_);
      return true;
    }
    if (*p_ == '"') {
      v->type = JsonValue::String;
      if (!string(&v->str)) return false;
      v->lexeme.assign(st, p_);
      return true;
    }
    if (lit("true")) { v->type = JsonValue::Bool; v->b = true; v->lexeme = "true"; return true; }
    if (lit("false")) { v->type = JsonValue::Bool; v->b = false; v->lexeme = "false"; return true; }
    if (lit("null")) { v->type = JsonValue::Null; v->lexeme = "null"; return true; }
    return number(v);
  }
};

// ---------------------------------------------------------------------------
// the op contract
// ---------------------------------------------------------------------------
constexpr uint32_t DEFAULT_MAX_ITERATIONS = 2000;   // poisson_blend.rs:68
constexpr uint32_t MAX_ITERATIONS_LIMIT = 100000;   // poisson_blend.rs:71
constexpr double DEFAULT_TOLERANCE = 1e-6;          // poisson_blend.rs:74
constexpr double OMEGA = 1.8;                       // poisson_blend.rs:78
constexpr double DEFAULT_LAMBDA = 0.0;              // screened_poisson.rs:63

struct OpError {
  std::string cls, code, message, actual;
};

struct BlendControls {
  uint32_t max_iterations = DEFAULT_MAX_ITERATIONS;
  double tolerance = DEFAULT_TOLERANCE;
  double lambda = 0.0;
};

struct OpSpec {
  const char *op;          // "repair.poisson_blend" / "repair.screened_poisson"
  const char *in_a;        // source / guidance
  const char *in_b;        // target / anchor
  const char *e_input, *e_param, *e_buffer;
  const char *kind;        // SolverData kind
  bool screened;
};

const OpSpec kBlend = {"repair.poisson_blend", "source", "target", "E_POISSON_BLEND_INPUT",
                       "E_POISSON_BLEND_PARAM", "E_POISSON_BLEND_BUFFER", "poisson", false};
const OpSpec kScreened = {"repair.screened_poisson", "guidance", "anchor", "E_SCREENED_POISSON_INPUT",
                          "E_SCREENED_POISSON_PARAM", "E_SCREENED_POISSON_BUFFER", "screened-poisson",
                          true};

OpError param_error(const OpSpec &s, const std::string &detail, const JsonValue &v) {
  // poisson_blend.rs:143-150 / screened_poisson.rs:116-123
  return OpError{"schema", s.e_param, std::string(s.op) + ": " + detail, v.lexeme};
}

// poisson_blend.rs:102-139 and screened_poisson.rs:66-112 (lambda first for the
// screened op, exactly as the reference reads it).
bool resolve_controls(const OpSpec &s, const JsonValue &params, BlendControls *c, OpError *err) {
  if (s.screened) {
    if (const JsonValue *v = params.get("lambda")) {
      double l;
      if (!v->as_f64(&l)) { *err = param_error(s, "lambda must be a number", *v); return false; }
      if (!std::isfinite(l) || l < 0.0) {
        *err = param_error(s, "lambda must be a finite value >= 0", *v);
        return false;
      }
      c->lambda = l;
    } else {
      c->lambda = DEFAULT_LAMBDA;
    }
  }
  if (const JsonValue *v = params.get("max_iterations")) {
    uint64_t n;
    if (!v->as_u64(&n) || n > 0xffffffffull) {
      *err = param_error(s, "max_iterations must be a positive integer", *v);
      return false;
    }
    if (n == 0 || n > MAX_ITERATIONS_LIMIT) {
      *err = param_error(s, "max_iterations must be in 1..=" + std::to_string(MAX_ITERATIONS_LIMIT), *v);
      return false;
    }
    c->max_iterations = (uint32_t)n;
  }
  if (const JsonValue *v = params.get("tolerance")) {
    double t;
    if (!v->as_f64(&t)) { *err = param_error(s, "tolerance must be a number", *v); return false; }
    if (!std::isfinite(t) || t <= 0.0 || t >= 1.0) {
      *err = param_error(s, "tolerance must be in (0, 1)", *v);
      return false;
    }
    c->tolerance = t;
  }
  return true;
}

const pt_port *find_port(const pt_port *inputs, uint32_t n, const char *name) {
  for (uint32_t k = 0; k < n; ++k)
    if (inputs[k].name && std::strcmp(inputs[k].name, name) == 0) return &inputs[k];
  return nullptr;
}

void set_error(pt_error *e, const OpError &o) {
  if (!e) return;
  std::snprintf(e->error_class, sizeof(e->error_class), "%s", o.cls.c_str());
  std::snprintf(e->code, sizeof(e->code), "%s", o.code.c_str());
  std::snprintf(e->message, sizeof(e->message), "%s", o.message.c_str());
  std::snprintf(e->actual, sizeof(e->actual), "%s", o.actual.c_str());
}

// ---------------------------------------------------------------------------
// mask.ellipse@1 and mask.polygon@1 (the generators the solve's masks come from)
// ---------------------------------------------------------------------------

// Rust's Display for f64: the shortest digits that round-trip, written out
// positionally (never an exponent), "-0" for negative zero.
std::string rust_f64(double v) {
  if (v == 0.0) return std::signbit(v) ? "-0" : "0";
  if (!std::isfinite(v)) return std::isnan(v) ? "NaN" : (v > 0 ? "inf" : "-inf");
  char buf[48];
  for (int p = 0; p < 17; ++p) {
    std::snprintf(buf, sizeof buf, "%.*e", p, v);
    if (std::strtod(buf, nullptr) == v) break;
  }
  std::string s(buf);
  const bool neg = s[0] == '-';
  if (neg) s.erase(0, 1);
  const size_t e = s.find('e');
  const int point = std::atoi(s.c_str() + e + 1) + 1;  // digits before the decimal point
  std::string digits;
  for (size_t k = 0; k < e; ++k)
    if (s[k] != '.') digits.push_back(s[k]);
  std::string out;
  if (point <= 0) out = "0." + std::string((size_t)-point, '0') + digits;
  else if (point >= (int)digits.size()) out = digits + std::string((size_t)point - digits.size(), '0');
  else out = digits.substr(0, (size_t)point) + "." + digits.substr((size_t)point);
  return (neg ? "-" : "") + out;
}

struct EllipseParams {
  double cx = 0, cy = 0, rx = 0, ry = 0, angle = 0, half = 0;
};

OpError ellipse_param_error(const std::string &name, const std::string &detail, const std::string &actual) {
  // ellipse.rs param_error
  return OpError{"schema", "E_ELLIPSE_PARAM", "mask.ellipse parameter `" + name + "`: " + detail, actual};
}

// finite_number (ellipse.rs): a number, and finite
bool ellipse_number(const JsonValue &v, const std::string &name, double *out, OpError *err) {
  if (!v.as_f64(out)) { *err = ellipse_param_error(name, "must be a number", v.lexeme); return false; }
  if (!std::isfinite(*out)) { *err = ellipse_param_error(name, "must be finite", v.lexeme); return false; }
  return true;
}

bool ellipse_pair(const JsonValue &params, const char *name, double *x, double *y, OpError *err) {
  const JsonValue *v = params.get(name);
  if (!v) { *err = ellipse_param_error(name, "missing required parameter", "null"); return false; }
  if (v->type != JsonValue::Array) { *err = ellipse_param_error(name, "must be a [x, y] array", v->lexeme); return false; }
  if (v->items.size() != 2) {
    *err = ellipse_param_error(name, "must have exactly two elements", v->lexeme);
    return false;
  }
  return ellipse_number(v->items[0], name, x, err) && ellipse_number(v->items[1], name, y, err);
}

// EllipseGeometry::resolve, pair_param, finite_number and parse_edge
// (ellipse.rs:119-159, :221-252, :261-297)
bool resolve_ellipse(const JsonValue &params, EllipseParams *g, OpError *err) {
  if (!ellipse_pair(params, "center_px", &g->cx, &g->cy, err)) return false;
  if (!ellipse_pair(params, "radii_px", &g->rx, &g->ry, err)) return false;
  const std::pair<const char *, double> radii[2] = {{"radii_px.x", g->rx}, {"radii_px.y", g->ry}};
  for (const auto &r : radii)
    if (!(std::isfinite(r.second) && r.second > 0.0)) {
      *err = OpError{"schema", "E_ELLIPSE_PARAM",
                     std::string("mask.ellipse `") + r.first + "` must be a strictly positive radius, got " +
                         rust_f64(r.second),
                     rust_f64(r.second)};
      return false;
    }
  g->angle = 0.0;
  if (const JsonValue *v = params.get("angle_rad"))
    if (!ellipse_number(*v, "angle_rad", &g->angle, err)) return false;
  if (const JsonValue *v = params.get("antialias")) {
    if (v->type != JsonValue::String) {
      *err = ellipse_param_error("antialias", "`antialias` must be a string", v->lexeme);
      return false;
    }
    if (v->str != "analytic") {
      *err = OpError{"schema", "E_ELLIPSE_PARAM",
                     "mask.ellipse only supports `antialias: analytic`, got `" + v->str + "`", ""};
      return false;
    }
  }
  g->half = 0.0;
  if (const JsonValue *edge = params.get("edge")) {
    if (edge->type != JsonValue::Object) {
      *err = ellipse_param_error("edge", "`edge` must be an object", edge->lexeme);
      return false;
    }
    const JsonValue *profile = edge->get("profile");
    if (!profile || profile->type != JsonValue::String) {
      *err = ellipse_param_error("edge.profile", "`edge.profile` must be a string", edge->lexeme);
      return false;
    }
    if (profile->str != "smoothstep") {
      *err = OpError{"schema", "E_ELLIPSE_PARAM",
                     "mask.ellipse only supports `edge.profile: smoothstep`, got `" + profile->str + "`", ""};
      return false;
    }
    const JsonValue *half = edge->get("half_width_px");
    if (!half) {
      *err = ellipse_param_error("edge.half_width_px", "`edge.half_width_px` is required", edge->lexeme);
      return false;
    }
    if (!ellipse_number(*half, "edge.half_width_px", &g->half, err)) return false;
    if (g->half < 0.0) {
      *err = ellipse_param_error("edge.half_width_px", "must be non-negative", half->lexeme);
      return false;
    }
  }
  return true;
}

OpError polygon_param_error(const std::string &detail, const std::string &actual) {
  // mask_polygon.rs param_error
  return OpError{"schema", "E_POLYGON_PARAM", "mask.polygon parameter: " + detail, actual};
}

// FillRule::resolve and Polygon::resolve (mask_polygon.rs:90-104, :124-152)
bool resolve_polygon(const JsonValue &params, std::vector<double> *pts, int32_t *rule, OpError *err) {
  const JsonValue *v = params.get("points");
  if (!v) {
    *err = OpError{"schema", "E_POLYGON_PARAM", "mask.polygon requires a `points` array of [x, y] vertices", ""};
    return false;
  }
  if (v->type != JsonValue::Array) {
    *err = polygon_param_error("`points` must be an array of [x, y] pairs", v->lexeme);
    return false;
  }
  for (const JsonValue &vertex : v->items) {
    if (vertex.type != JsonValue::Array) {
      *err = polygon_param_error("each vertex must be a [x, y] array", vertex.lexeme);
      return false;
    }
    if (vertex.items.size() != 2) {
      *err = polygon_param_error("each vertex must have exactly two elements", vertex.lexeme);
      return false;
    }
    for (const JsonValue &c : vertex.items) {
      double d;
      if (!c.as_f64(&d)) { *err = polygon_param_error("coordinates must be numbers", c.lexeme); return false; }
      if (!std::isfinite(d)) { *err = polygon_param_error("coordinates must be finite", c.lexeme); return false; }
      pts->push_back(d);
    }
  }
  *rule = PT_FILL_NONZERO;
  if (const JsonValue *f = params.get("fill_rule")) {
    if (f->type == JsonValue::String && f->str == "nonzero") *rule = PT_FILL_NONZERO;
    else if (f->type == JsonValue::String && f->str == "even-odd") *rule = PT_FILL_EVEN_ODD;
    else {
      *err = OpError{"schema", "E_POLYGON_PARAM", "mask.polygon `fill_rule` must be `nonzero` or `even-odd`",
                     f->lexeme};
      return false;
    }
  }
  return true;
}

// EllipseMask::compute (ellipse.rs:506-540) and PolygonMask::compute
// (mask_polygon.rs:427-452): the extent first, then the params, then the
// rasteriser; the output is the mask (width*height f32) in `candidate`.
pt_status mask_op_compute(pt_ctx *ctx, bool ellipse, const pt_port *inputs, uint32_t n_inputs,
                          const char *params_json, float *candidate, size_t candidate_count,
                          int32_t *all_finite, pt_error *err) {
  const char *op = ellipse ? "mask.ellipse" : "mask.polygon";
  const char *e_input = ellipse ? "E_ELLIPSE_INPUT" : "E_POLYGON_INPUT";
  const char *e_param = ellipse ? "E_ELLIPSE_PARAM" : "E_POLYGON_PARAM";
  const pt_port *src = find_port(inputs, n_inputs, "extent_from");
  if (!src) {
    set_error(err, OpError{"reference", e_input, std::string(op) + " requires an `extent_from` input value", ""});
    return PT_INVALID_ARG;
  }
  JsonValue params;
  if (params_json && *params_json) {
    JsonParser jp(params_json);
    if (!jp.parse(&params)) {
      set_error(err, OpError{"parse", e_param, std::string(op) + ": params are not valid JSON", ""});
      return PT_INVALID_ARG;
    }
  }
  OpError oe;
  EllipseParams g;
  std::vector<double> pts;
  int32_t rule = PT_FILL_NONZERO;
  if (ellipse ? !resolve_ellipse(params, &g, &oe) : !resolve_polygon(params, &pts, &rule, &oe)) {
    set_error(err, oe);
    return PT_INVALID_ARG;
  }
  const size_t count = (size_t)src->width * src->height;
  if ((count && !candidate) || candidate_count != count) {
    set_error(err, OpError{"execution", e_input,
                           std::string(op) + (ellipse ? " produced a sample buffer" : " produced a mask buffer") +
                               " of unexpected length " + std::to_string(candidate_count),
                           ""});
    return PT_INVALID_ARG;
  }
  if (!ctx) {
    set_error(err, OpError{"policy", "E_CUDA_UNAVAILABLE", std::string(op) + ": the cuda backend has no device context",
                           ""});
    return PT_NO_DEVICE;
  }
  const pt_status st =
      ellipse ? pt_mask_ellipse(ctx, src->width, src->height, g.cx, g.cy, g.rx, g.ry, g.angle, g.half, candidate, 0)
              : pt_mask_polygon(ctx, src->width, src->height, pts.data(), (uint32_t)(pts.size() / 2), rule,
                                candidate, 0);
  if (st != PT_OK) {
    set_error(err, OpError{st == PT_NO_DEVICE ? "policy" : "execution",
                           st == PT_NO_DEVICE ? "E_CUDA_UNAVAILABLE" : "E_CUDA_EXECUTION",
                           std::string(op) + ": " + pt_status_str(st) + ": " + pt_ctx_last_error(ctx), ""});
    return st;
  }
  if (all_finite) *all_finite = 1;  // coverage in [0, 1] by construction
  return PT_OK;
}

}  // namespace pt_op

using namespace pt_op;

extern "C" pt_status pt_op_compute_ex(pt_ctx *ctx, const char *op_id, const pt_port *inputs,
                                      uint32_t n_inputs, const char *params_json, float *candidate,
                                      size_t candidate_count, pt_solver_data *solver,
                                      double *residual_history, uint32_t history_cap,
                                      int32_t *all_finite, pt_error *err, uint32_t solve_flags) {
  return abi_guard(ctx, [&]() -> pt_status {
    if (err) std::memset(err, 0, sizeof(*err));
    if (!op_id || (n_inputs && !inputs)) return PT_INVALID_ARG;
    if (solve_flags & ~PT_FLAG_MULTIGRID) {
      set_error(err, OpError{"execution", "E_CUDA_SOLVE_FLAGS",
                             std::string("unsupported solve flags ") + std::to_string(solve_flags), ""});
      return PT_INVALID_ARG;
    }
    if (std::strcmp(op_id, "mask.ellipse@1") == 0 || std::strcmp(op_id, "mask.polygon@1") == 0)
      return mask_op_compute(ctx, op_id[5] == 'e', inputs, n_inputs, params_json, candidate, candidate_count,
                             all_finite, err);
    if (!solver) return PT_INVALID_ARG;
    const OpSpec *spec = nullptr;
    if (std::strcmp(op_id, "repair.poisson_blend@1") == 0) spec = &kBlend;
    else if (std::strcmp(op_id, "repair.screened_poisson@1") == 0) spec = &kScreened;
    else {
      set_error(err, OpError{"reference", "E_OP_UNKNOWN", std::string("unknown operation ") + op_id, ""});
      return PT_INVALID_ARG;
    }
    const OpSpec &s = *spec;

    JsonValue params;
    if (params_json && *params_json) {
      JsonParser jp(params_json);
      if (!jp.parse(&params)) {
        set_error(err, OpError{"parse", s.e_param, std::string(s.op) + ": params are not valid JSON", ""});
        return PT_INVALID_ARG;
      }
    }
    BlendControls controls;
    OpError oe;
    if (!resolve_controls(s, params, &controls, &oe)) { set_error(err, oe); return PT_INVALID_ARG; }

    // input_value (poisson_blend.rs:603-614): a missing port is a Reference error.
    const pt_port *pa = nullptr, *pb = nullptr, *pm = nullptr;
    const char *names[3] = {s.in_a, s.in_b, "mask"};
    const pt_port **slots[3] = {&pa, &pb, &pm};
    for (int k = 0; k < 3; ++k) {
      *slots[k] = find_port(inputs, n_inputs, names[k]);
      if (!*slots[k]) {
        set_error(err, OpError{"reference", s.e_input,
                               std::string(s.op) + " requires a `" + names[k] + "` input value", ""});
        return PT_INVALID_ARG;
      }
    }
    // descriptor kinds (poisson_blend.rs:545-553): the wrong kind is a Type error.
    const struct { const pt_port *p; const char *name; uint32_t kind; const char *word; } kinds[3] = {
        {pa, s.in_a, PT_KIND_IMAGE, "image"}, {pb, s.in_b, PT_KIND_IMAGE, "image"},
        {pm, "mask", PT_KIND_MASK, "mask"}};
    for (const auto &k : kinds) {
      if (k.p->kind != k.kind) {
        set_error(err, OpError{"type", s.e_input,
                               std::string(s.op) + " `" + k.name + "` input must be a " + k.word + " resource",
                               ""});
        return PT_INVALID_ARG;
      }
      const uint32_t ch = k.kind == PT_KIND_MASK ? 1u : k.p->channels;
      const size_t want = (size_t)k.p->width * k.p->height * ch;
      if (k.p->sample_count != want || (want && !k.p->samples)) {
        // a ResourceValue whose buffer disagrees with its descriptor cannot be
        // built in the reference (value.rs:50-69)
        set_error(err, OpError{"type", s.e_input,
                               std::string(s.op) + " `" + k.name +
                                   "` input buffer length does not match its descriptor",
                               std::to_string(k.p->sample_count)});
        return PT_INVALID_ARG;
      }
    }
    // check_shapes (poisson_blend.rs:417-445); shape errors use E_POISSON_BLEND_SHAPE
    // for both ops since the screened op reuses the blend's check.
    auto shape = [&](const char *detail, const std::string &actual) {
      set_error(err, OpError{"semantic", "E_POISSON_BLEND_SHAPE", std::string(s.op) + ": " + detail, actual});
      return PT_INVALID_ARG;
    };
    char buf[96];
    if (pa->width != pb->width || pa->height != pb->height) {
      std::snprintf(buf, sizeof buf, "%s %ux%u vs %s %ux%u", s.in_a, pa->width, pa->height, s.in_b, pb->width,
                    pb->height);
      return shape("the source and target images must share an extent", buf);
    }
    if (pa->channels != pb->channels) {
      std::snprintf(buf, sizeof buf, "%s %u channels vs %s %u channels", s.in_a, pa->channels, s.in_b,
                    pb->channels);
      return shape("the source and target images must share a channel layout", buf);
    }
    if (pm->width != pb->width || pm->height != pb->height) {
      std::snprintf(buf, sizeof buf, "mask %ux%u vs image %ux%u", pm->width, pm->height, pb->width, pb->height);
      return shape("the mask must share the images' extent", buf);
    }
    const size_t count = (size_t)pb->width * pb->height * pb->channels;
    if (!candidate || candidate_count != count) {
      set_error(err, OpError{"execution", s.e_buffer,
                             std::string(s.op) + " produced a candidate buffer of unexpected length " +
                                 std::to_string(candidate_count),
                             ""});
      return PT_INVALID_ARG;
    }

    pt_problem p{};
    p.width = pb->width;
    p.height = pb->height;
    p.channels = pb->channels;
    p.source_or_guidance = pa->samples;
    p.target_or_anchor = pb->samples;
    p.mask = pm->samples;
    p.lambda = controls.lambda;
    p.max_iterations = controls.max_iterations;
    p.tolerance = controls.tolerance;
    p.omega = OMEGA;
    p.flags = solve_flags;
    if (!ctx) {
      // validation passed but there is no device context: the backend is
      // unavailable (the E_GPU_UNAVAILABLE analogue, a Policy error)
      set_error(err, OpError{"policy", "E_CUDA_UNAVAILABLE",
                             std::string(s.op) + ": the cuda backend has no device context", ""});
      return PT_NO_DEVICE;
    }
    std::vector<pt_report> reps(p.channels + 1);
    std::vector<double> hist((size_t)p.channels * p.max_iterations);
    const pt_status st = pt_poisson_solve(ctx, &p, candidate, reps.data(), hist.empty() ? nullptr : hist.data());
    if (st != PT_OK) {
      set_error(err, OpError{st == PT_NO_DEVICE ? "policy" : "execution",
                             st == PT_NO_DEVICE ? "E_CUDA_UNAVAILABLE" : "E_CUDA_EXECUTION",
                             std::string(s.op) + ": " + pt_status_str(st) + ": " + pt_ctx_last_error(ctx), ""});
      return st;
    }
    const pt_report &w = reps[p.channels];  // worst channel (blend_channels' report)
    std::memset(solver, 0, sizeof(*solver));
    std::snprintf(solver->kind, sizeof(solver->kind), "%s", s.kind);
    // solver_data (poisson_blend.rs:249-266)
    solver->steps = w.iterations;
    solver->stability_number = 0.0;
    solver->stability_limit = 0.0;
    solver->stable = 1;
    solver->total_energy = 0.0;
    solver->iterations = w.iterations;
    solver->stop_reason = w.stop_reason;
    solver->converged = w.converged;
    solver->tolerance = w.tolerance;
    solver->final_residual = w.final_residual;
    solver->history_len = w.history_len;
    if (residual_history && w.channel >= 0) {
      const uint32_t m = w.history_len < history_cap ? w.history_len : history_cap;
      std::memcpy(residual_history, hist.data() + (size_t)w.channel * p.max_iterations, m * sizeof(double));
    }
    if (all_finite) {
      int32_t f = 1;
      for (size_t k = 0; k < count; ++k)
        if (!std::isfinite(candidate[k])) { f = 0; break; }
      *all_finite = f;
    }
    return PT_OK;
  });
}

extern "C" pt_status pt_op_compute(pt_ctx *ctx, const char *op_id, const pt_port *inputs,
                                   uint32_t n_inputs, const char *params_json, float *candidate,
                                   size_t candidate_count, pt_solver_data *solver,
                                   double *residual_history, uint32_t history_cap,
                                   int32_t *all_finite, pt_error *err) {
  return pt_op_compute_ex(ctx, op_id, inputs, n_inputs, params_json, candidate, candidate_count, solver,
                          residual_history, history_cap, all_finite, err, 0);
}
