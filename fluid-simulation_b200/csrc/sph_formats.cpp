// Checkpoint (RON / bincode) and recording-frame (bincode) encoders and
// decoders, and their C ABI. Host code only; the device readbacks that fill
// a checkpoint or a frame live in sph_system.cu.
#include "sph_formats.hpp"

#include <cerrno>
#include <charconv>
#include <cmath>
#include <cstdlib>
#include <cstring>
#include <limits>
#include <memory>
#include <new>
#include <utility>

#include "sph_host.hpp"

namespace sph {
namespace fmt {

// ---------------------------------------------------------------------------
// Rust `Display` for f64: the shortest digits that round-trip, placed in
// positional notation (no exponent), "-" for negative values including -0,
// "inf" / "-inf" / "NaN".
// ---------------------------------------------------------------------------
std::string rust_display(double v) {
  if (std::isnan(v)) return "NaN";
  if (std::isinf(v)) return v < 0 ? "-inf" : "inf";
  char buf[64];
  auto r = std::to_chars(buf, buf + sizeof buf, v, std::chars_format::scientific);
  std::string s(buf, r.ptr);
  std::string out;
  size_t i = 0;
  if (s[0] == '-') {
    out += '-';
    i = 1;
  }
  const size_t e = s.find('e');
  std::string digits;
  for (size_t k = i; k < e; ++k)
    if (s[k] != '.') digits += s[k];
  const int exp10 = std::atoi(s.c_str() + e + 1);
  const int point = exp10 + 1;  // digits before the decimal point
  const int nd = (int)digits.size();
  if (point <= 0) {
    out += "0.";
    out.append((size_t)(-point), '0');
    out += digits;
  } else if (point >= nd) {
    out += digits;
    out.append((size_t)(point - nd), '0');
  } else {
    out += digits.substr(0, (size_t)point);
    out += '.';
    out += digits.substr((size_t)point);
  }
  return out;
}

static std::string ron_f64(double v) {
  std::string s = rust_display(v);
  if (std::isfinite(v) && std::trunc(v) == v) s += ".0";
  return s;
}

// ---------------------------------------------------------------------------
// bincode 2, standard configuration
// ---------------------------------------------------------------------------
struct BinWriter {
  std::vector<uint8_t> b;
  void raw(const void* p, size_t n) {
    const uint8_t* q = (const uint8_t*)p;
    b.insert(b.end(), q, q + n);
  }
  void u8(uint8_t v) { b.push_back(v); }
  void varint(uint64_t v) {  // unsigned integers wider than u8, and usize
    if (v < 251) {
      u8((uint8_t)v);
    } else if (v <= 0xffffu) {
      u8(251);
      const uint16_t x = (uint16_t)v;
      le(&x, 2);
    } else if (v <= 0xffffffffu) {
      u8(252);
      const uint32_t x = (uint32_t)v;
      le(&x, 4);
    } else {
      u8(253);
      le(&v, 8);
    }
  }
  void le(const void* p, size_t n) {  // this library only builds for little-endian hosts
    raw(p, n);
  }
  void f64(double v) { le(&v, 8); }
  void f32(float v) { le(&v, 4); }
  void vec3_f64(const double* x, size_t n) {
    varint(n);
    for (size_t i = 0; i < 3 * n; ++i) f64(x[i]);
  }
  void vec3_f32(const float* x, size_t n) {
    varint(n);
    for (size_t i = 0; i < 3 * n; ++i) f32(x[i]);
  }
  void vec_f32(const float* x, size_t n) {
    varint(n);
    for (size_t i = 0; i < n; ++i) f32(x[i]);
  }
  void vec_u32(const uint32_t* x, size_t n) {
    varint(n);
    for (size_t i = 0; i < n; ++i) varint(x[i]);
  }
};

struct BinReader {
  const uint8_t* p;
  size_t n, i = 0;
  BinReader(const uint8_t* d, size_t len) : p(d), n(len) {}
  [[noreturn]] void fail(const char* what) const {
    throw Error(SPH_ERR_INVALID, std::string("bincode: ") + what + " at byte " + std::to_string(i));
  }
  void need(size_t k) {
    if (n - i < k) fail("unexpected end of input");
  }
  uint8_t u8() {
    need(1);
    return p[i++];
  }
  template <class T>
  T le() {
    need(sizeof(T));
    T v;
    std::memcpy(&v, p + i, sizeof(T));
    i += sizeof(T);
    return v;
  }
  uint64_t varint(uint64_t max) {
    const uint8_t b = u8();
    uint64_t v;
    if (b < 251) v = b;
    else if (b == 251) v = le<uint16_t>();
    else if (b == 252) v = le<uint32_t>();
    else if (b == 253) v = le<uint64_t>();
    else fail("invalid integer encoding");
    if (v > max) fail("integer out of range");
    return v;
  }
  uint64_t u64() { return varint(std::numeric_limits<uint64_t>::max()); }
  uint32_t u32() { return (uint32_t)varint(0xffffffffu); }
  size_t len(size_t min_elem_bytes) {
    const uint64_t k = u64();
    if (min_elem_bytes && k > (n - i) / min_elem_bytes) fail("sequence longer than the input");
    return (size_t)k;
  }
  double f64() { return le<double>(); }
  void vec3_f64(std::vector<double>& out) {
    const size_t k = len(24);
    out.resize(3 * k);
    for (auto& x : out) x = f64();
  }
};

void Checkpoint::check() const {
  const size_t N = mass.size();
  if (fluid_id.size() != N || position.size() != 3 * N || velocity.size() != 3 * N)
    throw Error(SPH_ERR_INVALID, "checkpoint arrays disagree in length");
  for (const auto& s : integrator_position)
    if (s.size() != 3 * N) throw Error(SPH_ERR_INVALID, "integrator position slot length");
  for (const auto& s : integrator_velocity)
    if (s.size() != 3 * N) throw Error(SPH_ERR_INVALID, "integrator velocity slot length");
}

// SerRigidBodyMotionCheckpoint field order: center_of_mass, orientation
// (i, j, k, w), linear_velocity, angular_momentum, force, torque.
static void rigid_to_ser(const RigidState& r, double out[19]) {
  const double* s = r.s.data();
  out[0] = s[0]; out[1] = s[1]; out[2] = s[2];
  out[3] = s[4]; out[4] = s[5]; out[5] = s[6]; out[6] = s[3];  // (i,j,k,w) from (w,i,j,k)
  for (int k = 7; k < 19; ++k) out[k] = s[k];
}
static void rigid_from_ser(const double in[19], RigidState& r) {
  double* s = r.s.data();
  s[0] = in[0]; s[1] = in[1]; s[2] = in[2];
  s[3] = in[6]; s[4] = in[3]; s[5] = in[4]; s[6] = in[5];
  for (int k = 7; k < 19; ++k) s[k] = in[k];
  r.dynamic = true;
}

std::vector<uint8_t> checkpoint_to_bincode(const Checkpoint& c) {
  c.check();
  BinWriter w;
  w.varint(c.time_steps_propagated);
  w.f64(c.current_time);
  const size_t N = c.n();
  w.vec_u32(c.fluid_id.data(), N);
  w.vec3_f64(c.position.data(), N);
  w.vec3_f64(c.velocity.data(), N);
  w.varint(N);
  for (double m : c.mass) w.f64(m);
  for (const auto* slots : {&c.integrator_position, &c.integrator_velocity}) {
    w.varint(slots->size());
    for (const auto& s : *slots) w.vec3_f64(s.data(), s.size() / 3);
  }
  w.varint(c.boundaries.size());
  for (const auto& r : c.boundaries) {
    w.u8(r.dynamic ? 1 : 0);
    if (r.dynamic) {
      double ser[19];
      rigid_to_ser(r, ser);
      for (double x : ser) w.f64(x);
    }
  }
  return std::move(w.b);
}

Checkpoint checkpoint_from_bincode(const uint8_t* data, size_t len) {
  BinReader r(data, len);
  Checkpoint c;
  c.time_steps_propagated = r.u64();
  c.current_time = r.f64();
  const size_t N = r.len(1);
  c.fluid_id.resize(N);
  for (auto& x : c.fluid_id) x = r.u32();
  r.vec3_f64(c.position);
  r.vec3_f64(c.velocity);
  c.mass.resize(r.len(8));
  for (auto& x : c.mass) x = r.f64();
  for (auto* slots : {&c.integrator_position, &c.integrator_velocity}) {
    slots->resize(r.len(1));
    for (auto& s : *slots) r.vec3_f64(s);
  }
  c.boundaries.resize(r.len(1));
  for (auto& b : c.boundaries) {
    const uint8_t tag = r.u8();
    if (tag > 1) r.fail("invalid Option tag");
    if (tag) {
      double ser[19];
      for (double& x : ser) x = r.f64();
      rigid_from_ser(ser, b);
    }
  }
  c.check();
  return c;
}

// ---------------------------------------------------------------------------
// RON writer (ron::to_string layout)
// ---------------------------------------------------------------------------
static void ron_tuple(std::string& o, const double* x, int k) {
  o += '(';
  for (int i = 0; i < k; ++i) {
    if (i) o += ',';
    o += ron_f64(x[i]);
  }
  o += ')';
}
static void ron_vec3_seq(std::string& o, const std::vector<double>& x) {
  o += '[';
  for (size_t i = 0; i < x.size() / 3; ++i) {
    if (i) o += ',';
    ron_tuple(o, &x[3 * i], 3);
  }
  o += ']';
}

std::string checkpoint_to_ron(const Checkpoint& c) {
  c.check();
  std::string o;
  o.reserve(64 + c.n() * 160);
  o += "(time_steps_propagated:" + std::to_string(c.time_steps_propagated);
  o += ",current_time:" + ron_f64(c.current_time);
  o += ",fluid:(fluid_id:[";
  for (size_t i = 0; i < c.fluid_id.size(); ++i) {
    if (i) o += ',';
    o += std::to_string(c.fluid_id[i]);
  }
  o += "],position:";
  ron_vec3_seq(o, c.position);
  o += ",velocity:";
  ron_vec3_seq(o, c.velocity);
  o += ",mass:[";
  for (size_t i = 0; i < c.mass.size(); ++i) {
    if (i) o += ',';
    o += ron_f64(c.mass[i]);
  }
  o += ']';
  const char* names[2] = {",integrator_position_slots:[", ",integrator_velocity_slots:["};
  const std::vector<std::vector<double>>* slots[2] = {&c.integrator_position, &c.integrator_velocity};
  for (int k = 0; k < 2; ++k) {
    o += names[k];
    for (size_t s = 0; s < slots[k]->size(); ++s) {
      if (s) o += ',';
      ron_vec3_seq(o, (*slots[k])[s]);
    }
    o += ']';
  }
  o += "),boundary:(dynamic_states:[";
  for (size_t b = 0; b < c.boundaries.size(); ++b) {
    if (b) o += ',';
    const RigidState& r = c.boundaries[b];
    if (!r.dynamic) {
      o += "None";
      continue;
    }
    double ser[19];
    rigid_to_ser(r, ser);
    o += "Some((center_of_mass:";
    ron_tuple(o, ser, 3);
    o += ",orientation:";
    ron_tuple(o, ser + 3, 4);
    o += ",linear_velocity:";
    ron_tuple(o, ser + 7, 3);
    o += ",angular_momentum:";
    ron_tuple(o, ser + 10, 3);
    o += ",force:";
    ron_tuple(o, ser + 13, 3);
    o += ",torque:";
    ron_tuple(o, ser + 16, 3);
    o += "))";
  }
  o += "]))";
  return o;
}

// ---------------------------------------------------------------------------
// RON reader: a small recursive-descent parser into a value tree, then the
// checkpoint's fields taken from it by name (any order; unknown fields are
// ignored as serde's derive does).
// ---------------------------------------------------------------------------
struct RonValue {
  enum Kind { Number, Ident, Seq, Tuple, Struct, Some, None } kind = Number;
  std::string text;                                     // Number / Ident
  std::vector<RonValue> items;                          // Seq / Tuple / Some
  std::vector<std::pair<std::string, RonValue>> fields;  // Struct
};

struct RonParser {
  const char* s;
  size_t n, i = 0;
  int depth = 0;
  RonParser(const char* t, size_t len) : s(t), n(len) {}
  [[noreturn]] void fail(const std::string& what) const {
    throw Error(SPH_ERR_INVALID, "RON: " + what + " at offset " + std::to_string(i));
  }
  void skip() {
    for (;;) {
      while (i < n && (s[i] == ' ' || s[i] == '\t' || s[i] == '\n' || s[i] == '\r')) ++i;
      if (i + 1 < n && s[i] == '/' && s[i + 1] == '/') {
        while (i < n && s[i] != '\n') ++i;
      } else if (i + 1 < n && s[i] == '/' && s[i + 1] == '*') {
        i += 2;
        while (i + 1 < n && !(s[i] == '*' && s[i + 1] == '/')) ++i;
        if (i + 1 >= n) fail("unterminated comment");
        i += 2;
      } else if (i + 1 < n && s[i] == '#' && s[i + 1] == '!') {  // #![enable(...)] attributes
        while (i < n && s[i] != ']') ++i;
        if (i >= n) fail("unterminated attribute");
        ++i;
      } else {
        return;
      }
    }
  }
  bool peek(char c) {
    skip();
    return i < n && s[i] == c;
  }
  void expect(char c) {
    if (!peek(c)) fail(std::string("expected '") + c + "'");
    ++i;
  }
  static bool ident_start(char c) { return (c >= 'a' && c <= 'z') || (c >= 'A' && c <= 'Z') || c == '_'; }
  static bool ident_char(char c) { return ident_start(c) || (c >= '0' && c <= '9'); }
  std::string ident() {
    skip();
    size_t b = i;
    if (i >= n || !ident_start(s[i])) fail("expected an identifier");
    while (i < n && ident_char(s[i])) ++i;
    return std::string(s + b, i - b);
  }
  // After '(' : a struct if an identifier and ':' follow, else a tuple.
  bool struct_ahead() {
    skip();
    size_t save = i;
    if (i >= n || !ident_start(s[i])) return false;
    while (i < n && ident_char(s[i])) ++i;
    skip();
    const bool is = i < n && s[i] == ':';
    i = save;
    return is;
  }
  RonValue value() {
    if (++depth > 64) fail("nesting too deep");
    skip();
    if (i >= n) fail("unexpected end of input");
    RonValue v;
    const char c = s[i];
    if (c == '[') {
      ++i;
      v.kind = RonValue::Seq;
      while (!peek(']')) {
        v.items.push_back(value());
        if (!peek(',')) break;
        ++i;
      }
      expect(']');
    } else if (c == '(') {
      v = paren();
    } else if (c == '-' || c == '+' || c == '.' || (c >= '0' && c <= '9')) {
      size_t b = i++;
      while (i < n && (ident_char(s[i]) || s[i] == '.' ||
                       ((s[i] == '-' || s[i] == '+') && (s[i - 1] == 'e' || s[i - 1] == 'E'))))
        ++i;
      v.kind = RonValue::Number;
      v.text.assign(s + b, i - b);
    } else if (ident_start(c)) {
      std::string id = ident();
      if (id == "Some") {
        expect('(');
        v.kind = RonValue::Some;
        v.items.push_back(value());
        if (peek(',')) ++i;
        expect(')');
      } else if (id == "None") {
        v.kind = RonValue::None;
      } else if (id == "inf" || id == "NaN") {
        v.kind = RonValue::Number;
        v.text = id;
      } else if (peek('(')) {
        v = paren();  // named struct or tuple struct: the name is not checked
      } else {
        v.kind = RonValue::Ident;
        v.text = id;
      }
    } else {
      fail(std::string("unexpected character '") + c + "'");
    }
    --depth;
    return v;
  }
  RonValue paren() {
    expect('(');
    RonValue v;
    if (struct_ahead()) {
      v.kind = RonValue::Struct;
      while (!peek(')')) {
        std::string k = ident();
        expect(':');
        v.fields.emplace_back(std::move(k), value());
        if (!peek(',')) break;
        ++i;
      }
    } else {
      v.kind = RonValue::Tuple;
      while (!peek(')')) {
        v.items.push_back(value());
        if (!peek(',')) break;
        ++i;
      }
    }
    expect(')');
    return v;
  }
};

static const RonValue& field(const RonValue& v, const char* name) {
  if (v.kind != RonValue::Struct) throw Error(SPH_ERR_INVALID, std::string("RON: expected a struct with '") + name + "'");
  for (const auto& f : v.fields)
    if (f.first == name) return f.second;
  throw Error(SPH_ERR_INVALID, std::string("RON: missing field '") + name + "'");
}
static double ron_to_f64(const RonValue& v) {
  if (v.kind != RonValue::Number) throw Error(SPH_ERR_INVALID, "RON: expected a number");
  const std::string& t = v.text;
  if (t == "inf" || t == "+inf") return std::numeric_limits<double>::infinity();
  if (t == "-inf") return -std::numeric_limits<double>::infinity();
  if (t == "NaN" || t == "-NaN" || t == "+NaN") return std::numeric_limits<double>::quiet_NaN();
  std::string u;
  for (char ch : t)
    if (ch != '_') u += ch;  // RON allows digit separators
  char* end = nullptr;
  const double d = std::strtod(u.c_str(), &end);
  if (end != u.c_str() + u.size() || u.empty()) throw Error(SPH_ERR_INVALID, "RON: bad number '" + t + "'");
  return d;
}
static uint64_t ron_to_u64(const RonValue& v, uint64_t max) {
  if (v.kind != RonValue::Number) throw Error(SPH_ERR_INVALID, "RON: expected an integer");
  std::string u;
  for (char ch : v.text)
    if (ch != '_') u += ch;
  if (!u.empty() && u[0] == '+') u.erase(0, 1);
  if (u.empty() || u.find_first_not_of("0123456789") != std::string::npos)
    throw Error(SPH_ERR_INVALID, "RON: bad unsigned integer '" + v.text + "'");
  errno = 0;
  const unsigned long long x = std::strtoull(u.c_str(), nullptr, 10);
  if (errno == ERANGE || x > max) throw Error(SPH_ERR_INVALID, "RON: integer out of range '" + v.text + "'");
  return x;
}
static const std::vector<RonValue>& ron_items(const RonValue& v, RonValue::Kind want, const char* what) {
  if (v.kind != want && !(want == RonValue::Tuple && v.kind == RonValue::Seq))
    throw Error(SPH_ERR_INVALID, std::string("RON: expected ") + what);
  return v.items;
}
static void ron_fixed(const RonValue& v, double* out, size_t k) {
  const auto& it = ron_items(v, RonValue::Tuple, "a tuple");
  if (it.size() != k) throw Error(SPH_ERR_INVALID, "RON: tuple of the wrong length");
  for (size_t j = 0; j < k; ++j) out[j] = ron_to_f64(it[j]);
}
static void ron_vec3(const RonValue& v, std::vector<double>& out) {
  const auto& it = ron_items(v, RonValue::Seq, "a sequence");
  out.resize(3 * it.size());
  for (size_t j = 0; j < it.size(); ++j) ron_fixed(it[j], &out[3 * j], 3);
}

Checkpoint checkpoint_from_ron(const char* text, size_t len) {
  RonParser p(text, len);
  RonValue root = p.value();
  p.skip();
  if (p.i != p.n) p.fail("trailing characters");
  Checkpoint c;
  c.time_steps_propagated = ron_to_u64(field(root, "time_steps_propagated"), std::numeric_limits<uint64_t>::max());
  c.current_time = ron_to_f64(field(root, "current_time"));
  const RonValue& f = field(root, "fluid");
  for (const auto& x : ron_items(field(f, "fluid_id"), RonValue::Seq, "a sequence"))
    c.fluid_id.push_back((uint32_t)ron_to_u64(x, 0xffffffffu));
  ron_vec3(field(f, "position"), c.position);
  ron_vec3(field(f, "velocity"), c.velocity);
  for (const auto& x : ron_items(field(f, "mass"), RonValue::Seq, "a sequence")) c.mass.push_back(ron_to_f64(x));
  const char* names[2] = {"integrator_position_slots", "integrator_velocity_slots"};
  std::vector<std::vector<double>>* slots[2] = {&c.integrator_position, &c.integrator_velocity};
  for (int k = 0; k < 2; ++k)
    for (const auto& s : ron_items(field(f, names[k]), RonValue::Seq, "a sequence")) {
      slots[k]->emplace_back();
      ron_vec3(s, slots[k]->back());
    }
  for (const auto& d : ron_items(field(field(root, "boundary"), "dynamic_states"), RonValue::Seq, "a sequence")) {
    RigidState r;
    if (d.kind == RonValue::Some) {
      const RonValue& b = d.items[0];
      double ser[19];
      ron_fixed(field(b, "center_of_mass"), ser, 3);
      ron_fixed(field(b, "orientation"), ser + 3, 4);
      ron_fixed(field(b, "linear_velocity"), ser + 7, 3);
      ron_fixed(field(b, "angular_momentum"), ser + 10, 3);
      ron_fixed(field(b, "force"), ser + 13, 3);
      ron_fixed(field(b, "torque"), ser + 16, 3);
      rigid_from_ser(ser, r);
    } else if (d.kind != RonValue::None) {
      throw Error(SPH_ERR_INVALID, "RON: expected Some(...) or None");
    }
    c.boundaries.push_back(r);
  }
  c.check();
  return c;
}

// ---------------------------------------------------------------------------
// TimeStepInfo (render_info.rs:71-81): time_step_number, Measurement
// (measurement.rs:51-75), FluidVisualization, BoundaryVisualization.
// ---------------------------------------------------------------------------
std::vector<uint8_t> time_step_info_to_bincode(const sph_frame_view& f) {
  BinWriter w;
  w.varint(f.time_step_number);
  const sph_measurement& m = f.measurement;
  for (double x : {m.time, m.density, m.density_error, m.kinetic_energy, m.stiffness, m.fluid_viscosity,
                   m.boundary_viscosity, m.fluid_depth, m.rest_density_grid_spacing, m.kernel_support_radius,
                   m.time_step_size, m.target_density_error})
    w.f64(x);
  w.varint(m.solver_iterations);
  for (double x : {m.relaxation_factor, m.time_step_wall_clock_time, m.predicted_density_error}) w.f64(x);
  auto quantity = [&](int q) {
    if (q < SPH_Q_SPEED || q > SPH_Q_KINETIC_ENERGY) throw Error(SPH_ERR_INVALID, "unknown quantity");
    w.varint((uint64_t)q);  // ScalarQuantity variant index
  };
  if (f.fluid == SPH_FLUID_TRIANGLE_MESH) {
    // TriangleMesh { meshes: Vec<(u32, RenderMesh)>, max_fluid_id, coloring }
    w.varint(0);
    const size_t nm = f.meshes ? f.meshes->m.size() : 0;
    w.varint(nm);
    for (size_t k = 0; k < nm; ++k) {
      const SurfaceMeshOut& m = f.meshes->m[k];
      w.varint(m.fluid_id);
      w.varint(m.vertices.size() / 6);  // RenderVertex { position, normal }
      for (double x : m.vertices) w.f64(x);
      w.vec_u32(m.indices.data(), m.indices.size());
    }
    w.varint(f.max_fluid_id);
    if (f.fluid_coloring != SPH_COLORING_UNIFORM && f.fluid_coloring != SPH_COLORING_ID)
      throw Error(SPH_ERR_INVALID, "unknown fluid mesh coloring");
    w.varint(f.fluid_coloring == SPH_COLORING_ID ? 1 : 0);  // FluidMeshColoring
  } else if (f.fluid == SPH_FLUID_SAMPLES) {
    w.varint(1);
    if (f.n && !f.fluid_positions) throw Error(SPH_ERR_INVALID, "null fluid positions");
    w.vec3_f32(f.fluid_positions, f.n);
    if (f.fluid_coloring == SPH_COLORING_UNIFORM) {
      w.varint(0);
    } else if (f.fluid_coloring == SPH_COLORING_ID) {
      if (f.n && !f.fluid_ids) throw Error(SPH_ERR_INVALID, "null fluid ids");
      uint32_t mx = 0;
      for (size_t i = 0; i < f.n; ++i) mx = f.fluid_ids[i] > mx ? f.fluid_ids[i] : mx;
      w.varint(1);
      w.vec_u32(f.fluid_ids, f.n);
      w.varint(mx);
    } else if (f.fluid_coloring == SPH_COLORING_QUANTITY) {
      if (f.n && !f.fluid_data) throw Error(SPH_ERR_INVALID, "null fluid data");
      w.varint(2);
      quantity(f.quantity);
      w.vec_f32(f.fluid_data, f.n);
    } else {
      throw Error(SPH_ERR_INVALID, "unknown fluid sample coloring");
    }
  } else if (f.fluid == SPH_FLUID_SENSOR_PLANE) {
    w.varint(2);
    quantity(f.quantity);
    if (f.num_planes && !f.planes) throw Error(SPH_ERR_INVALID, "null planes");
    w.varint(f.num_planes);
    for (size_t k = 0; k < f.num_planes; ++k) {
      const sph_sensor_plane& pl = f.planes[k];
      const size_t np = pl.rows * pl.cols;
      if (np && (!pl.positions || !pl.data)) throw Error(SPH_ERR_INVALID, "null plane arrays");
      w.vec3_f32(pl.positions, np);
      w.vec_f32(pl.data, np);
      w.varint(pl.rows);
      w.varint(pl.cols);
    }
  } else {
    throw Error(SPH_ERR_INVALID, "unknown fluid visualization");
  }
  if (f.boundary_visualization == SPH_BOUNDARY_TRIANGLE_MESH) {
    // TriangleMesh { meshes: Vec<(RenderMesh, RenderPose)>, coloring }
    w.varint(0);
    if (f.num_boundary_meshes && (!f.boundary_meshes || !f.boundary_poses))
      throw Error(SPH_ERR_INVALID, "null boundary meshes or poses");
    w.varint(f.num_boundary_meshes);
    for (size_t k = 0; k < f.num_boundary_meshes; ++k) {
      const sph_render_mesh& m = f.boundary_meshes[k];
      if ((m.num_vertices && !m.vertices) || (m.num_indices && !m.indices))
        throw Error(SPH_ERR_INVALID, "null render mesh arrays");
      w.varint(m.num_vertices);
      for (size_t i = 0; i < 6 * m.num_vertices; ++i) w.f64(m.vertices[i]);
      w.vec_u32(m.indices, m.num_indices);
      for (int c = 0; c < 7; ++c) w.f32(f.boundary_poses[7 * k + c]);  // RenderPose
    }
    switch (f.boundary_mesh_coloring) {  // BoundaryMeshColoring
      case SPH_MESH_ORIGINAL: w.varint(0); break;
      case SPH_MESH_UNIFORM: w.varint(1); break;
      case SPH_MESH_BOUNDARY_ID: {
        if (f.num_mesh_ids && !f.mesh_ids) throw Error(SPH_ERR_INVALID, "null mesh ids");
        uint32_t mx = 0;
        for (size_t i = 0; i < f.num_mesh_ids; ++i) mx = f.mesh_ids[i] > mx ? f.mesh_ids[i] : mx;
        w.varint(2);
        w.vec_u32(f.mesh_ids, f.num_mesh_ids);
        w.varint(mx);
        break;
      }
      default: throw Error(SPH_ERR_INVALID, "unknown boundary mesh coloring");
    }
    return std::move(w.b);
  }
  if (f.boundary_visualization != SPH_BOUNDARY_SAMPLES) throw Error(SPH_ERR_INVALID, "unknown boundary visualization");
  // BoundaryVisualization::Samples
  w.varint(1);
  if (f.num_boundary_samples && !f.boundary_positions) throw Error(SPH_ERR_INVALID, "null boundary positions");
  w.vec3_f32(f.boundary_positions, f.num_boundary_samples);
  if (f.boundary_coloring == SPH_COLORING_UNIFORM) {
    w.varint(0);
  } else if (f.boundary_coloring == SPH_COLORING_ID) {
    if (f.num_boundary_samples && !f.boundary_ids) throw Error(SPH_ERR_INVALID, "null boundary ids");
    uint32_t mx = 0;
    for (size_t i = 0; i < f.num_boundary_samples; ++i) mx = f.boundary_ids[i] > mx ? f.boundary_ids[i] : mx;
    w.varint(1);
    w.vec_u32(f.boundary_ids, f.num_boundary_samples);
    w.varint(mx);
  } else {
    throw Error(SPH_ERR_INVALID, "unknown boundary sample coloring");
  }
  return std::move(w.b);
}

}  // namespace fmt
}  // namespace sph

// ---------------------------------------------------------------------------
// C ABI
// ---------------------------------------------------------------------------
using sph::Error;

template <class F>
static int guarded_fmt(F&& f) {
  try {
    f();
    return SPH_OK;
  } catch (const Error& e) {
    sph::g_last_error = e.what();
    return e.code;
  } catch (const std::bad_alloc&) {
    sph::g_last_error = "host allocation failed";
    return SPH_ERR_OOM;
  } catch (const std::exception& e) {
    sph::g_last_error = e.what();
    return SPH_ERR_INVALID;
  }
}

namespace sph {
namespace fmt {
sph_bytes_t* new_bytes(std::vector<uint8_t>&& b) {
  auto* out = new sph_bytes;
  out->b = std::move(b);
  return out;
}
sph_checkpoint_t* new_checkpoint(Checkpoint&& c) {
  c.check();
  auto* out = new sph_checkpoint;
  out->c = std::move(c);
  return out;
}
}  // namespace fmt
}  // namespace sph

extern "C" {

int sph_bytes_get(const sph_bytes_t* b, const uint8_t** data, size_t* len) {
  return guarded_fmt([&] {
    if (!b || !data || !len) throw Error(SPH_ERR_INVALID, "null argument");
    *data = b->b.data();
    *len = b->b.size();
  });
}
void sph_bytes_free(sph_bytes_t* b) { delete b; }

int sph_checkpoint_from_view(const sph_checkpoint_view* v, sph_checkpoint_t** out) {
  return guarded_fmt([&] {
    if (!v || !out) throw Error(SPH_ERR_INVALID, "null argument");
    const size_t N = v->n;
    if (N && (!v->position || !v->velocity || !v->mass)) throw Error(SPH_ERR_INVALID, "null fluid arrays");
    if ((v->integrator_position_slots && N && !v->integrator_position) ||
        (v->integrator_velocity_slots && N && !v->integrator_velocity) ||
        (v->num_boundaries && !v->dynamic))
      throw Error(SPH_ERR_INVALID, "null slot or boundary arrays");
    sph::fmt::Checkpoint c;
    c.time_steps_propagated = v->time_steps_propagated;
    c.current_time = v->current_time;
    c.fluid_id.assign(N, 0u);
    if (v->fluid_id) c.fluid_id.assign(v->fluid_id, v->fluid_id + N);
    c.position.assign(v->position, v->position + 3 * N);
    c.velocity.assign(v->velocity, v->velocity + 3 * N);
    c.mass.assign(v->mass, v->mass + N);
    for (size_t s = 0; s < v->integrator_position_slots; ++s)
      c.integrator_position.emplace_back(v->integrator_position + s * 3 * N, v->integrator_position + (s + 1) * 3 * N);
    for (size_t s = 0; s < v->integrator_velocity_slots; ++s)
      c.integrator_velocity.emplace_back(v->integrator_velocity + s * 3 * N, v->integrator_velocity + (s + 1) * 3 * N);
    c.boundaries.resize(v->num_boundaries);
    for (size_t b = 0; b < v->num_boundaries; ++b) {
      c.boundaries[b].dynamic = v->dynamic[b] != 0;
      if (c.boundaries[b].dynamic) {
        if (!v->rigid_state) throw Error(SPH_ERR_INVALID, "null rigid states");
        std::memcpy(c.boundaries[b].s.data(), v->rigid_state + 19 * b, 19 * sizeof(double));
      }
    }
    *out = sph::fmt::new_checkpoint(std::move(c));
  });
}

int sph_checkpoint_view_of(const sph_checkpoint_t* cc, sph_checkpoint_view* v) {
  return guarded_fmt([&] {
    if (!cc || !v) throw Error(SPH_ERR_INVALID, "null argument");
    auto* k = const_cast<sph_checkpoint_t*>(cc);
    const sph::fmt::Checkpoint& c = k->c;
    const size_t N = c.n();
    k->xi.clear();
    for (const auto& s : c.integrator_position) k->xi.insert(k->xi.end(), s.begin(), s.end());
    k->vi.clear();
    for (const auto& s : c.integrator_velocity) k->vi.insert(k->vi.end(), s.begin(), s.end());
    k->dyn.assign(c.boundaries.size(), 0);
    k->rigid.assign(19 * c.boundaries.size(), 0.0);
    for (size_t b = 0; b < c.boundaries.size(); ++b) {
      k->dyn[b] = c.boundaries[b].dynamic ? 1 : 0;
      std::memcpy(&k->rigid[19 * b], c.boundaries[b].s.data(), 19 * sizeof(double));
    }
    v->time_steps_propagated = c.time_steps_propagated;
    v->current_time = c.current_time;
    v->n = N;
    v->fluid_id = c.fluid_id.data();
    v->position = c.position.data();
    v->velocity = c.velocity.data();
    v->mass = c.mass.data();
    v->integrator_position_slots = c.integrator_position.size();
    v->integrator_position = k->xi.data();
    v->integrator_velocity_slots = c.integrator_velocity.size();
    v->integrator_velocity = k->vi.data();
    v->num_boundaries = c.boundaries.size();
    v->dynamic = k->dyn.data();
    v->rigid_state = k->rigid.data();
  });
}

void sph_checkpoint_free(sph_checkpoint_t* c) { delete c; }

int sph_checkpoint_encode(const sph_checkpoint_t* c, int format, sph_bytes_t** out) {
  return guarded_fmt([&] {
    if (!c || !out) throw Error(SPH_ERR_INVALID, "null argument");
    if (format == SPH_FORMAT_RON) {
      std::string t = sph::fmt::checkpoint_to_ron(c->c);
      *out = sph::fmt::new_bytes(std::vector<uint8_t>(t.begin(), t.end()));
    } else if (format == SPH_FORMAT_BINCODE) {
      *out = sph::fmt::new_bytes(sph::fmt::checkpoint_to_bincode(c->c));
    } else {
      throw Error(SPH_ERR_INVALID, "unknown format");
    }
  });
}

int sph_checkpoint_decode(const uint8_t* data, size_t len, int format, sph_checkpoint_t** out) {
  return guarded_fmt([&] {
    if ((!data && len) || !out) throw Error(SPH_ERR_INVALID, "null argument");
    if (format == SPH_FORMAT_RON)
      *out = sph::fmt::new_checkpoint(sph::fmt::checkpoint_from_ron((const char*)data, len));
    else if (format == SPH_FORMAT_BINCODE)
      *out = sph::fmt::new_checkpoint(sph::fmt::checkpoint_from_bincode(data, len));
    else
      throw Error(SPH_ERR_INVALID, "unknown format");
  });
}

int sph_frame_encode(const sph_frame_view* f, sph_bytes_t** out) {
  return guarded_fmt([&] {
    if (!f || !out) throw Error(SPH_ERR_INVALID, "null argument");
    *out = sph::fmt::new_bytes(sph::fmt::time_step_info_to_bincode(*f));
  });
}

}  // extern "C"
