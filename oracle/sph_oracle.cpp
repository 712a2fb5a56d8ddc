// SPH oracle — TEST INFRASTRUCTURE ONLY (see sph_oracle.hpp for the scope and
// pinning statement). f64 restatement of the reference's CPU algorithms.
#include "sph_oracle.hpp"

#include <algorithm>
#include <limits>
#include <chrono>
#include <cstring>
#include <stdexcept>
#include <atomic>


namespace oracle {

static const double PI = 3.14159265358979323846;

static int g_threads = 0;
int num_threads() {
  if (g_threads > 0) return g_threads;
  unsigned hc = std::thread::hardware_concurrency();
  return hc ? (int)hc : 1;
}
void set_num_threads(int n) { g_threads = n; }
void parallel_for(size_t n, const std::function<void(size_t, size_t)>& body) {
  size_t t = (size_t)num_threads();
  if (t <= 1 || n < 2048) { if (n) body(0, n); return; }
  if (t > n) t = n;
  std::vector<std::thread> pool;
  size_t chunk = (n + t - 1) / t;
  for (size_t k = 0; k < t; ++k) {
    size_t b = k * chunk, e = std::min(n, b + chunk);
    if (b >= e) break;
    pool.emplace_back([&body, b, e] { body(b, e); });
  }
  for (auto& th : pool) th.join();
}

// ---------------------------------------------------------------------------
// small linear algebra (nalgebra semantics)
// ---------------------------------------------------------------------------
M3 mul(const M3& a, const M3& b) {
  M3 r;
  for (int i = 0; i < 3; ++i)
    for (int j = 0; j < 3; ++j)
      r.m[i][j] = (a.m[i][0] * b.m[0][j] + a.m[i][1] * b.m[1][j]) + a.m[i][2] * b.m[2][j];
  return r;
}
V3 mul(const M3& a, V3 v) {
  return {(a.m[0][0] * v.x + a.m[0][1] * v.y) + a.m[0][2] * v.z,
          (a.m[1][0] * v.x + a.m[1][1] * v.y) + a.m[1][2] * v.z,
          (a.m[2][0] * v.x + a.m[2][1] * v.y) + a.m[2][2] * v.z};
}
M3 transpose(const M3& a) {
  M3 r;
  for (int i = 0; i < 3; ++i)
    for (int j = 0; j < 3; ++j) r.m[i][j] = a.m[j][i];
  return r;
}
// Hamilton product
Quat qmul(Quat a, Quat b) {
  return {a.w * b.w - a.x * b.x - a.y * b.y - a.z * b.z,
          a.w * b.x + a.x * b.w + a.y * b.z - a.z * b.y,
          a.w * b.y - a.x * b.z + a.y * b.w + a.z * b.x,
          a.w * b.z + a.x * b.y - a.y * b.x + a.z * b.w};
}
// nalgebra UnitQuaternion * Vector3: t = 2 q.v x v; v + w t + q.v x t
V3 qrotate(Quat q, V3 v) {
  V3 qv{q.x, q.y, q.z};
  V3 t = cross(qv, v) * 2.0;
  V3 c = cross(qv, t);
  return (t * q.w + c) + v;
}
M3 qto_matrix(Quat q) {
  double ww = q.w * q.w, ii = q.x * q.x, jj = q.y * q.y, kk = q.z * q.z;
  double ij = q.x * q.y * 2.0, wk = q.w * q.z * 2.0, wj = q.w * q.y * 2.0;
  double ik = q.x * q.z * 2.0, jk = q.y * q.z * 2.0, wi = q.w * q.x * 2.0;
  M3 r;
  r.m[0][0] = ww + ii - jj - kk; r.m[0][1] = ij - wk;           r.m[0][2] = wj + ik;
  r.m[1][0] = wk + ij;           r.m[1][1] = ww - ii + jj - kk; r.m[1][2] = jk - wi;
  r.m[2][0] = ik - wj;           r.m[2][1] = wi + jk;           r.m[2][2] = ww - ii - jj + kk;
  return r;
}
// nalgebra UnitQuaternion::from_scaled_axis = exp of the pure quaternion v/2
Quat qfrom_scaled_axis(V3 v) {
  V3 h = v / 2.0;
  double nn = norm_squared(h);
  const double eps = std::numeric_limits<double>::epsilon();
  if (nn <= eps * eps) return Quat{};
  double n = std::sqrt(nn);
  double s = std::sin(n) / n;
  return {std::cos(n), h.x * s, h.y * s, h.z * s};
}

// ---------------------------------------------------------------------------
// Kernel (SL/sph/kernel/cubic_spline.rs:7-17, kernel/mod.rs:22-46)
// ---------------------------------------------------------------------------
static const double ALPHA = 16.0 / PI;
static inline double powi3(double x) { return (x * x) * x; }
static inline double powi2(double x) { return x * x; }
static inline double powi4(double x) { double x2 = x * x; return x2 * x2; }

double kernel_w(double q) {
  return powi3(std::max(1. - q, 0.)) - 4. * powi3(std::max(1. / 2. - q, 0.));
}
double kernel_dqw(double q) {
  return -3. * powi2(std::max(1. - q, 0.)) + 12. * powi2(std::max(1. / 2. - q, 0.));
}
double kernel_function(V3 r, double h) {
  return ALPHA / powi3(h) * kernel_w(norm(r) / h);
}
V3 kernel_gradient(V3 r, double h) {
  double rn = norm(r);
  if (rn == 0.0) return {0, 0, 0};
  double c = ALPHA / powi4(h);
  double d = kernel_dqw(rn / h);
  return {((c * r.x) / rn) * d, ((c * r.y) / rn) * d, ((c * r.z) / rn) * d};
}

// ---------------------------------------------------------------------------
// SpatialHashing (SL/neighbor_search/spatial_hashing.rs:27-158)
// ---------------------------------------------------------------------------
int32_t SpatialHashing::saturating_i32(double v) {  // Rust `as i32`
  if (std::isnan(v)) return 0;
  if (v >= 2147483647.0) return 2147483647;
  if (v <= -2147483648.0) return (int32_t)-2147483648LL;
  return (int32_t)v;
}
void SpatialHashing::get_cell(V3 p, double cs, int32_t out[3]) {  // :40-46
  out[0] = saturating_i32(std::floor(p.x / cs));
  out[1] = saturating_i32(std::floor(p.y / cs));
  out[2] = saturating_i32(std::floor(p.z / cs));
}
uint64_t SpatialHashing::map_int_to_uint(int32_t k) {  // :49-55
  if (k >= 0) return (uint64_t)k * 2;
  return (uint64_t)(-(int64_t)k) * 2 + 1;
}
uint64_t SpatialHashing::hash(int32_t k, int32_t l, int32_t m) {  // :61-71
  const uint64_t P1 = 73856093, P2 = 19349663, P3 = 83492791;
  return (map_int_to_uint(k) * P1) ^ (map_int_to_uint(l) * P2) ^ (map_int_to_uint(m) * P3);
}
void SpatialHashing::populate(const std::vector<V3>& samples) {  // :27-37 (sequential)
  for (size_t id = 0; id < samples.size(); ++id) {
    int32_t c[3];
    get_cell(samples[id], cell_size, c);
    cells[hash(c[0], c[1], c[2])].push_back(id);
  }
}
void SpatialHashing::find_samples(double range, const std::vector<V3>& positions,
                                  const std::vector<V3>& samples, NeighborList& nl) {
  cells.clear();
  populate(samples);
  const size_t n = positions.size();
  std::vector<std::vector<size_t>> per(n);
  const int32_t m = (int32_t)std::ceil(range / cell_size);  // :84
  std::atomic<size_t> dup_total{0};
parallel_for((size_t)(n), [&](size_t b__, size_t e__) {
  for (long long ii = (long long)b__; ii < (long long)e__; ++ii) {
    size_t id = (size_t)ii;
    V3 p = positions[id];
    int32_t c[3];
    get_cell(p, cell_size, c);
    std::vector<size_t>& out = per[id];
    std::vector<uint64_t> seen;
    for (int32_t dx = -m; dx <= m; ++dx)
      for (int32_t dy = -m; dy <= m; ++dy)
        for (int32_t dz = -m; dz <= m; ++dz) {
          uint64_t h = hash(c[0] + dx, c[1] + dy, c[2] + dz);
          auto it = cells.find(h);
          if (it == cells.end()) continue;
          bool repeat = std::find(seen.begin(), seen.end(), h) != seen.end();
          seen.push_back(h);
          for (size_t nb : it->second) {
            if (norm(p - samples[nb]) < range) {  // distance(sample, pos) = (pos - sample).norm()
              out.push_back(nb);
              if (repeat) ++dup_total;
            }
          }
        }
  }
  });
  last_duplicates = dup_total.load();
  // NeighborList::flatten (neighbor_search/mod.rs:118-133)
  nl.indices.clear();
  nl.offsets.assign(1, 0);
  size_t total = 0;
  for (auto& v : per) total += v.size();
  nl.indices.reserve(total);
  nl.offsets.reserve(n + 1);
  for (auto& v : per) {
    nl.indices.insert(nl.indices.end(), v.begin(), v.end());
    nl.offsets.push_back(nl.indices.size());
  }
}

// ---------------------------------------------------------------------------
// Fluid (SL/sph/fluid.rs:113-210)
// ---------------------------------------------------------------------------
void Fluid::resize_slots(size_t ip, size_t iv, size_t sp, size_t sv) {
  size_t n = position.size();
  integrator_position_slots.assign(ip, std::vector<V3>(n));
  integrator_velocity_slots.assign(iv, std::vector<V3>(n));
  solver_position_slots.assign(sp, std::vector<V3>(n));
  solver_velocity_slots.assign(sv, std::vector<V3>(n));
}
void Fluid::swap(size_t a, size_t b) {
  if (a == b) return;
  std::swap(fluid_id[a], fluid_id[b]);
  std::swap(position[a], position[b]);
  std::swap(velocity[a], velocity[b]);
  std::swap(acceleration[a], acceleration[b]);
  std::swap(mass[a], mass[b]);
  std::swap(volume[a], volume[b]);
  std::swap(pressure[a], pressure[b]);
  std::swap(origin[a], origin[b]);
  for (auto* pool : {&integrator_position_slots, &integrator_velocity_slots,
                     &solver_position_slots, &solver_velocity_slots})
    for (auto& s : *pool) std::swap(s[a], s[b]);
}
void Fluid::disable(size_t id) {  // fluid.rs:159-163
  if (id >= num_active) throw std::out_of_range("Fluid::disable: id >= num_active");
  num_active -= 1;
  swap(id, num_active);
}
void Fluid::drop_inactive() {
  size_t n = num_active;
  fluid_id.resize(n); position.resize(n); velocity.resize(n); acceleration.resize(n);
  mass.resize(n); volume.resize(n); pressure.resize(n); origin.resize(n);
  for (auto* pool : {&integrator_position_slots, &integrator_velocity_slots,
                     &solver_position_slots, &solver_velocity_slots})
    for (auto& s : *pool) s.resize(n);
}

// ---------------------------------------------------------------------------
// RigidBodyMotion (rigid_body_motion.rs:38-201)
// ---------------------------------------------------------------------------
RigidBodyMotion::RigidBodyMotion(double m, const M3& inertia_body, const M3& inv_body, V3 com,
                                 Quat q, V3 lv, V3 av)
    : mass(m), inertia_tensor_inv_body(inv_body), center_of_mass(com), orientation(q),
      linear_velocity(lv) {
  M3 r = qto_matrix(q);
  M3 iw = mul(mul(r, inertia_body), transpose(r));
  angular_momentum = mul(iw, av);
  update_derived_variables();
}
void RigidBodyMotion::update_derived_variables() {  // :72-77
  M3 r = qto_matrix(orientation);
  inertia_tensor_inv_world = mul(mul(r, inertia_tensor_inv_body), transpose(r));
  angular_velocity = mul(inertia_tensor_inv_world, angular_momentum);
}
V3 RigidBodyMotion::local_to_world(V3 p) const { return qrotate(orientation, p) + center_of_mass; }
V3 RigidBodyMotion::world_to_local(V3 p) const {
  Quat inv{orientation.w, -orientation.x, -orientation.y, -orientation.z};
  return qrotate(inv, p - center_of_mass);
}
V3 RigidBodyMotion::local_to_world_vector(V3 v) const { return qrotate(orientation, v); }
V3 RigidBodyMotion::velocity_at_point(V3 p) const {  // :135-140
  return linear_velocity + cross(angular_velocity, p - center_of_mass);
}
void RigidBodyMotion::add_force(V3 f, V3 location) {  // :147-150
  force += f;
  torque += cross(location - center_of_mass, f);
}
void RigidBodyMotion::reset_forces() {  // :141-144
  force = {0, 0, 0};
  torque = {0, 0, 0};
}
void RigidBodyMotion::restore_from_checkpoint(V3 com, Quat q, V3 lv, V3 am, V3 f,
                                              V3 t) {  // :214-222
  center_of_mass = com;
  orientation = q;
  linear_velocity = lv;
  angular_momentum = am;
  force = f;
  torque = t;
  update_derived_variables();
}
void RigidBodyMotion::step_forward_in_time(double dt) {  // :183-201
  V3 lin_acc = force / mass;
  linear_velocity += lin_acc * dt;
  center_of_mass += linear_velocity * dt;
  angular_momentum += torque * dt;
  angular_velocity = mul(inertia_tensor_inv_world, angular_momentum);
  orientation = qmul(qfrom_scaled_axis(angular_velocity * dt), orientation);
  reset_forces();
  update_derived_variables();
}

void BoundaryHandling::add_force_onto_boundary(size_t id, V3 force, V3 location) {
  if (id >= count()) return;
  RigidBodyMotion* m = at(id).motion();
  if (m) m->add_force(force, location);
}

// ---------------------------------------------------------------------------
// StaticSampleBoundary (static_sample_boundary.rs:142-168, 354-412, 544-552)
// ---------------------------------------------------------------------------
void SampleBoundary::update_positions_and_velocities() {
  if (!dynamic) return;
  for (size_t i = 0; i < xb_body.size(); ++i) {
    xb[i] = state.local_to_world(xb_body[i]);
    vb[i] = state.velocity_at_point(xb[i]);
  }
}
void StaticSampleBoundary::initialize(double h, double gamma_v) {
  cell_size = h;
  for (auto& b : boundaries) {
    b.update_positions_and_velocities();
    NeighborList bb;
    SpatialHashing sh(h);
    sh.find_samples(h, b.xb, b.xb, bb);
    b.vol.assign(b.xb.size(), 0.0);
    for (size_t i = 0; i < b.xb.size(); ++i) {
      double inv = 0;
      for (const size_t* it = bb.begin(i); it != bb.end(i); ++it)
        inv += kernel_function(b.xb[*it] - b.xb[i], h);
      b.vol[i] = gamma_v / inv;
    }
  }
}
void StaticSampleBoundary::find_boundary_samples(double range, const std::vector<V3>& positions,
                                                 double) {
  for (auto& b : boundaries) {
    SpatialHashing sh(cell_size);
    sh.find_samples(range, positions, b.xb, b.nl);
  }
}
void StaticSampleBoundary::step_forward_in_time(double dt) {
  for (auto& b : boundaries) {
    if (!b.dynamic) continue;
    b.state.step_forward_in_time(dt);
    b.update_positions_and_velocities();
  }
}

// ---------------------------------------------------------------------------
// CubicSerendipityDiscretization (discretization.rs:81-557)
// ---------------------------------------------------------------------------
// reference_nodes (:267-300) as lattice offsets {0..3} and reference coords
struct RefNode {
  double x, y, z;
  int ox, oy, oz;
};
static std::vector<RefNode> make_ref_nodes() {
  std::vector<RefNode> nodes;
  const double signs[2] = {-1.0, 1.0};
  const double thirds[2] = {-1. / 3., 1. / 3.};
  auto off = [](double r) { return (int)std::llround((r + 1.0) * 1.5); };
  auto push = [&](double x, double y, double z) {
    nodes.push_back({x, y, z, off(x), off(y), off(z)});
  };
  for (double z : signs) for (double y : signs) for (double x : signs) push(x, y, z);
  for (double z : signs) for (double y : signs) for (double t : thirds) push(t, y, z);
  for (double z : signs) for (double x : signs) for (double t : thirds) push(x, t, z);
  for (double y : signs) for (double x : signs) for (double t : thirds) push(x, y, t);
  return nodes;
}
static const std::vector<RefNode>& ref_nodes() {
  static const std::vector<RefNode> n = make_ref_nodes();
  return n;
}
static inline bool is_corner(double c) { return std::fabs(std::fabs(c) - 1.0) < 1e-9; }
static inline double shape(const RefNode& p, double xi, double eta, double zeta, double r2) {
  bool cx = is_corner(p.x), cy = is_corner(p.y), cz = is_corner(p.z);
  if (cx && cy && cz)
    return (1.0 / 64.0) * (1.0 + xi * p.x) * (1.0 + eta * p.y) * (1.0 + zeta * p.z) *
           (9.0 * r2 - 19.0);
  if (!cx && cy && cz)
    return (9.0 / 64.0) * (1.0 - xi * xi) * (1.0 + 9.0 * xi * p.x) * (1.0 + eta * p.y) *
           (1.0 + zeta * p.z);
  if (cx && !cy && cz)
    return (9.0 / 64.0) * (1.0 - eta * eta) * (1.0 + 9.0 * eta * p.y) * (1.0 + xi * p.x) *
           (1.0 + zeta * p.z);
  if (cx && cy && !cz)
    return (9.0 / 64.0) * (1.0 - zeta * zeta) * (1.0 + 9.0 * zeta * p.z) * (1.0 + xi * p.x) *
           (1.0 + eta * p.y);
  return 0.0;
}
bool Serendipity::function(V3 p, double& out) const {  // :437-483
  double pc[3] = {p.x, p.y, p.z}, mn[3] = {x_min.x, x_min.y, x_min.z},
         mx[3] = {x_max.x, x_max.y, x_max.z};
  int64_t c[3];
  for (int d = 0; d < 3; ++d) {
    double fi = std::floor((pc[d] - mn[d]) / dx);
    if (pc[d] < mn[d] || pc[d] > mx[d]) return false;  // OutOfBounds
    int64_t idx = (int64_t)fi;
    c[d] = std::min(idx, n[d] - 1);
  }
  const auto& rn = ref_nodes();
  const int64_t nx = NX(), ny = NY();
  double vals[32];
  for (int a = 0; a < 32; ++a) {
    int64_t kx = 3 * c[0] + rn[a].ox, ky = 3 * c[1] + rn[a].oy, kz = 3 * c[2] + rn[a].oz;
    double v = nodes[(size_t)((kz * ny + ky) * nx + kx)];
    if (std::isnan(v)) return false;  // PrunedCell
    vals[a] = v;
  }
  double o[3] = {mn[0] + (double)c[0] * dx, mn[1] + (double)c[1] * dx, mn[2] + (double)c[2] * dx};
  double xi = 2.0 * (pc[0] - o[0]) / dx - 1.0;
  double eta = 2.0 * (pc[1] - o[1]) / dx - 1.0;
  double zeta = 2.0 * (pc[2] - o[2]) / dx - 1.0;
  double r2 = xi * xi + eta * eta + zeta * zeta;
  double s = -0.0;
  for (int a = 0; a < 32; ++a) s += vals[a] * shape(rn[a], xi, eta, zeta, r2);
  out = s;
  return true;
}
bool Serendipity::gradient(V3 p, V3& out) const {  // :509-557
  double h = dx / 6.0;
  double g[3];
  for (int axis = 0; axis < 3; ++axis) {
    V3 pp = p, pm = p;
    if (axis == 0) { pp.x += h; pm.x -= h; }
    if (axis == 1) { pp.y += h; pm.y -= h; }
    if (axis == 2) { pp.z += h; pm.z -= h; }
    double fp, fm;
    if (!function(pp, fp)) return false;
    if (!function(pm, fm)) return false;
    g[axis] = (fp - fm) / (2.0 * h);
  }
  out = {g[0], g[1], g[2]};
  return true;
}

// ---------------------------------------------------------------------------
// VolumeMapBoundary sampling (volume_map_boundary.rs:1259-1424, 1936-1994)
// ---------------------------------------------------------------------------
bool VMBoundary::signed_distance(V3 p, double& out) const {
  return sdf.function(dynamic ? state.world_to_local(p) : p, out);
}
bool VMBoundary::signed_distance_gradient(V3 p, V3& out) const {
  if (!dynamic) return sdf.gradient(p, out);
  V3 gl;
  if (!sdf.gradient(state.world_to_local(p), gl)) return false;
  out = state.local_to_world_vector(gl);
  return true;
}
bool VMBoundary::volume_map_value(V3 p, double& out) const {
  return vm.function(dynamic ? state.world_to_local(p) : p, out);
}
V3 VMBoundary::velocity_at_point_on_boundary(V3 p) const {
  return dynamic ? state.velocity_at_point(p) : V3{0, 0, 0};
}
static inline double ball_volume(double r) { return 4.0 / 3.0 * PI * powi3(r); }

void VolumeMapBoundary::find_boundary_samples(double range, const std::vector<V3>& positions,
                                              double spacing) {
  const size_t n = positions.size();
  for (auto& b : boundaries) {
    std::vector<char> has(n, 0);
    std::vector<V3> xb(n), vb(n), vis_p(4 * n), vis_v(4 * n);
    std::vector<double> vol(n);
parallel_for((size_t)(n), [&](size_t b__, size_t e__) {
    for (long long ii = (long long)b__; ii < (long long)e__; ++ii) {
      size_t i = (size_t)ii;
      V3 pos = positions[i];
      double sd;
      if (!b.signed_distance(pos, sd) || !(sd < range)) continue;
      V3 g;
      if (!b.signed_distance_gradient(pos, g)) continue;
      double gn = norm(g);
      if (!(gn > 0.5 && gn < 2.0)) continue;
      double v;
      if (!b.volume_map_value(pos, v) || !(v > 0.)) continue;
      double volume = std::min(v, ball_volume(range));
      double d = std::max(sd + 0.25 * spacing, spacing);
      V3 pob = pos - (g / norm(g)) * d;
      has[i] = 1;
      xb[i] = pob;
      vb[i] = b.velocity_at_point_on_boundary(pob);
      vol[i] = volume;
      V3 u = pob - pos;
      V3 tmp{1., 0., 0.};
      if (std::fabs(dot(u / norm(u), tmp)) > 0.9) tmp = {0., 1., 0.};
      V3 t1 = cross(u, tmp);
      V3 t2 = cross(u, t1);
      t1 = t1 / norm(t1);
      t2 = t2 / norm(t2);
      double dd = 0.5 * range;
      V3 q[4] = {pob + t1 * dd, pob - t1 * dd, pob + t2 * dd, pob - t2 * dd};
      for (int k = 0; k < 4; ++k) {
        vis_p[4 * i + k] = q[k];
        vis_v[4 * i + k] = b.velocity_at_point_on_boundary(q[k]);
      }
    }
  });
    // sequential write-back (:1383-1422): Normal entries first, then viscosity
    b.spos.clear(); b.svel.clear(); b.svol.clear();
    b.nl_normal.indices.clear(); b.nl_normal.offsets.assign(1, 0);
    for (size_t i = 0; i < n; ++i) {
      if (has[i]) {
        b.nl_normal.indices.push_back(b.spos.size());
        b.spos.push_back(xb[i]); b.svel.push_back(vb[i]); b.svol.push_back(vol[i]);
      }
      b.nl_normal.offsets.push_back(b.nl_normal.indices.size());
    }
    b.nl_visc.indices.clear(); b.nl_visc.offsets.assign(1, 0);
    for (size_t i = 0; i < n; ++i) {
      if (has[i])
        for (int k = 0; k < 4; ++k) {
          b.nl_visc.indices.push_back(b.spos.size());
          b.spos.push_back(vis_p[4 * i + k]); b.svel.push_back(vis_v[4 * i + k]);
          b.svol.push_back(0.25 * vol[i]);
        }
      b.nl_visc.offsets.push_back(b.nl_visc.indices.size());
    }
  }
}
// ---------------------------------------------------------------------------
// Rigid-rigid contact of VolumeMapBoundary (volume_map_boundary.rs:55-1102):
// broad phase on world AABBs, contact cells from the overlap boxes, the
// contact volume of each cell by 8^3 Gauss-Legendre quadrature of the
// product of both bodies' cubic extension functions of the signed distance,
// and a projected Jacobi iteration with nonlinear conjugate-gradient
// acceleration (NNCG) for the contact pressures p_c >= 0 and the friction
// impulses lambda_c inside the Coulomb cone.
// ---------------------------------------------------------------------------
namespace {

constexpr double kContactCellSizeFactor = 0.5;   // :60
constexpr int kContactQuadratureDegree = 8;       // :57
constexpr double kFrictionCoefficient = 0.5;      // :62
constexpr double kRelaxation = 0.5;               // :64
constexpr double kMinDiagonal = 1e-35;            // :65
constexpr double kFbTolPressure = 1e-6;           // :67
constexpr double kFbTolFriction = 1e-3;           // :68

M3 m3_identity() {
  M3 m;
  m.m[0][0] = m.m[1][1] = m.m[2][2] = 1.0;
  return m;
}
M3 m3_add(const M3& a, const M3& b) {
  M3 r;
  for (int i = 0; i < 3; ++i)
    for (int j = 0; j < 3; ++j) r.m[i][j] = a.m[i][j] + b.m[i][j];
  return r;
}
M3 m3_sub(const M3& a, const M3& b) {
  M3 r;
  for (int i = 0; i < 3; ++i)
    for (int j = 0; j < 3; ++j) r.m[i][j] = a.m[i][j] - b.m[i][j];
  return r;
}
M3 m3_scale(const M3& a, double s) {
  M3 r;
  for (int i = 0; i < 3; ++i)
    for (int j = 0; j < 3; ++j) r.m[i][j] = a.m[i][j] * s;
  return r;
}
M3 m3_outer(V3 a, V3 b) {
  const double x[3] = {a.x, a.y, a.z}, y[3] = {b.x, b.y, b.z};
  M3 r;
  for (int i = 0; i < 3; ++i)
    for (int j = 0; j < 3; ++j) r.m[i][j] = x[i] * y[j];
  return r;
}
M3 m3_cross_matrix(V3 v) {
  M3 r;
  r.m[0][1] = -v.z; r.m[0][2] = v.y;
  r.m[1][0] = v.z;  r.m[1][2] = -v.x;
  r.m[2][0] = -v.y; r.m[2][1] = v.x;
  return r;
}
M3 m3_abs(const M3& a) {
  M3 r;
  for (int i = 0; i < 3; ++i)
    for (int j = 0; j < 3; ++j) r.m[i][j] = std::fabs(a.m[i][j]);
  return r;
}

struct WorldBox {
  V3 min, max;
};

// BoundaryType::world_aabb (:2122-2151): |R| applied to the local half extents.
WorldBox world_aabb(const VMBoundary& b) {
  if (!b.dynamic) return {b.aabb_center - b.aabb_half, b.aabb_center + b.aabb_half};
  const M3 r = qto_matrix(b.state.orientation);
  const V3 he = mul(m3_abs(r), b.aabb_half);
  const V3 c = b.state.local_to_world(b.aabb_center);
  return {c - he, c + he};
}
bool boxes_overlap(const WorldBox& a, const WorldBox& b) {  // :1783-1790
  return a.min.x <= b.max.x && a.max.x >= b.min.x && a.min.y <= b.max.y && a.max.y >= b.min.y &&
         a.min.z <= b.max.z && a.max.z >= b.min.z;
}
bool boxes_intersection(const WorldBox& a, const WorldBox& b, WorldBox& out) {  // :1792-1805
  out.min = {std::max(a.min.x, b.min.x), std::max(a.min.y, b.min.y), std::max(a.min.z, b.min.z)};
  out.max = {std::min(a.max.x, b.max.x), std::min(a.max.y, b.max.y), std::min(a.max.z, b.max.z)};
  return out.min.x <= out.max.x && out.min.y <= out.max.y && out.min.z <= out.max.z;
}

// cubic_extension_fn and its derivative (:1717-1745): W(x)/W(0) on (0, h).
double cubic_extension(double x, double h) {
  if (x >= h) return 0.;
  if (x <= 0.) return 1.;
  return kernel_function(V3{x, 0., 0.}, h) / kernel_function(V3{0., 0., 0.}, h);
}
double cubic_extension_derivative(double x, double h) {
  if (x >= h || x <= 0.0) return 0.0;
  return kernel_gradient(V3{x, 0., 0.}, h).x / kernel_function(V3{0., 0., 0.}, h);
}

struct QuadPoint {  // QuadPointData (:784-793)
  V3 pos;
  double weight;
  V3 grad_a, grad_b;
  double s_a, s_b, sp_a, sp_b;
};
struct Cell {  // ContactCell (:678-697)
  size_t a, b;
  std::vector<QuadPoint> q;
  double volume;
  V3 center, f_a, tau_a, f_b, tau_b;
  M3 tproj;
  double acc_p = 0, acc_f = 0;
};

const RigidBodyMotion* motion_of(const VMBoundary& b) { return b.dynamic ? &b.state : nullptr; }

// build_contact_cell (:700-782) with quadrature_points (:805-833).
bool build_cell(size_t ia, size_t ib, V3 from, V3 to, const std::vector<VMBoundary>& bs, double h,
                const std::vector<double>& gx, const std::vector<double>& gw, Cell& cell) {
  const V3 half = (to - from) * 0.5;
  const V3 center = from + half;
  const double scaling = 2.0;
  double v_c = 0.0;
  cell.q.clear();
  const int n = (int)gx.size();
  for (int i = 0; i < n; ++i)
    for (int j = 0; j < n; ++j)
      for (int k = 0; k < n; ++k) {
        const V3 pos = center + V3{gx[i] * half.x, gx[j] * half.y, gx[k] * half.z};
        const double w = gw[i] * gw[j] * gw[k] * half.x * half.y * half.z;
        double phi_a, phi_b;
        if (!bs[ia].signed_distance(pos, phi_a)) continue;
        if (!bs[ib].signed_distance(pos, phi_b)) continue;
        const double s_a = cubic_extension(scaling * phi_a + h, h);
        const double s_b = cubic_extension(scaling * phi_b + h, h);
        if (s_a <= 0.0 || s_b <= 0.0) continue;
        V3 ga, gb;
        if (!bs[ia].signed_distance_gradient(pos, ga)) continue;
        if (!bs[ib].signed_distance_gradient(pos, gb)) continue;
        v_c += w * s_a * s_b;
        cell.q.push_back(QuadPoint{pos, w, ga, gb, s_a, s_b,
                                   scaling * cubic_extension_derivative(scaling * phi_a + h, h),
                                   scaling * cubic_extension_derivative(scaling * phi_b + h, h)});
      }
  if (v_c <= 0.0 || cell.q.empty()) return false;
  cell.a = ia;
  cell.b = ib;
  cell.volume = v_c;
  return true;
}

// compute_diagonal (:835-926).
void compute_diagonal(Cell& c, const std::vector<VMBoundary>& bs, double dt) {
  const RigidBodyMotion* ma = motion_of(bs[c.a]);
  const RigidBodyMotion* mb = motion_of(bs[c.b]);
  V3 xv{0, 0, 0}, f_a{0, 0, 0}, t_a{0, 0, 0}, f_b{0, 0, 0}, t_b{0, 0, 0};
  for (const QuadPoint& q : c.q) {
    const double w_g = q.weight * q.s_a * q.s_b;
    xv += w_g * q.pos;
    const double w_a = q.weight * q.sp_a * q.s_b;
    f_a += w_a * q.grad_a;
    if (ma) t_a += w_a * cross(q.pos - ma->center_of_mass, q.grad_a);
    const double w_b = q.weight * q.sp_b * q.s_a;
    f_b += w_b * q.grad_b;
    if (mb) t_b += w_b * cross(q.pos - mb->center_of_mass, q.grad_b);
  }
  c.center = xv / c.volume;
  c.f_a = f_a;
  c.tau_a = t_a;
  c.f_b = f_b;
  c.tau_b = t_b;
  const V3 n = c.f_a / std::max(norm(c.f_a), 1e-15);
  c.tproj = m3_sub(m3_identity(), m3_outer(n, n));
  auto pressure_term = [](const RigidBodyMotion* m, V3 f, V3 t) {
    return m ? dot(f, f) / m->mass + dot(t, mul(m->inertia_tensor_inv_world, t)) : 0.0;
  };
  c.acc_p = dt * dt * (pressure_term(ma, f_a, t_a) + pressure_term(mb, f_b, t_b));
  auto friction_term = [&](const RigidBodyMotion* m) {
    if (!m) return M3{};
    const M3 rx = m3_cross_matrix(c.center - m->center_of_mass);
    return m3_sub(m3_scale(m3_identity(), 1.0 / m->mass), mul(mul(rx, m->inertia_tensor_inv_world), rx));
  };
  const M3 k = mul(m3_scale(c.tproj, dt), m3_add(friction_term(ma), friction_term(mb)));
  c.acc_f = 1. / 3. * ((k.m[0][0] + k.m[1][1]) + k.m[2][2]);
}

// mean_fischer_burmeister (utilities/mod.rs:27-41).
double mean_fischer_burmeister(const std::vector<double>& a, const std::vector<double>& b) {
  double sum = 0.0;
  for (size_t i = 0; i < a.size(); ++i) sum += std::fabs(a[i] + b[i] - std::sqrt(a[i] * a[i] + b[i] * b[i]));
  return sum / (double)a.size();
}

}  // namespace

ContactResult VolumeMapBoundary::solve_contacts(double dt, bool commit) {
  ContactResult res;
  const size_t nb = boundaries.size();
  res.force.assign(nb, V3{0, 0, 0});
  res.torque.assign(nb, V3{0, 0, 0});
  const double h = kernel_support_radius;
  // broad_phase (:70-96) and generate_contact_cells (:98-161)
  std::vector<WorldBox> boxes(nb);
  for (size_t i = 0; i < nb; ++i)
    if (boundaries[i].has_aabb) boxes[i] = world_aabb(boundaries[i]);
  std::vector<double> gx, gw;
  gauss_legendre(kContactQuadratureDegree, gx, gw);
  std::vector<Cell> cells;
  for (size_t i = 0; i < nb; ++i) {
    if (!boundaries[i].has_aabb) continue;
    for (size_t j = i + 1; j < nb; ++j) {
      if (!boundaries[j].has_aabb) continue;
      if (!boundaries[i].dynamic && !boundaries[j].dynamic) continue;
      if (!boxes_overlap(boxes[i], boxes[j])) continue;
      WorldBox ov;
      if (!boxes_intersection(boxes[i], boxes[j], ov)) continue;
      // subdivide_overlap (:1813-1844)
      const double target = h * kContactCellSizeFactor;
      const V3 ext = ov.max - ov.min;
      const size_t n[3] = {std::max<size_t>((size_t)std::ceil(ext.x / target), 1),
                           std::max<size_t>((size_t)std::ceil(ext.y / target), 1),
                           std::max<size_t>((size_t)std::ceil(ext.z / target), 1)};
      const V3 cs{ext.x / (double)n[0], ext.y / (double)n[1], ext.z / (double)n[2]};
      for (size_t iz = 0; iz < n[2]; ++iz)
        for (size_t iy = 0; iy < n[1]; ++iy)
          for (size_t ix = 0; ix < n[0]; ++ix) {
            const V3 from = ov.min + V3{(double)ix * cs.x, (double)iy * cs.y, (double)iz * cs.z};
            const V3 to = from + cs;
            const V3 center = from + (to - from) * 0.5;
            const double bound = 2.0 * (norm(to - from) * 0.5);
            double pa, pb;
            if (!boundaries[i].signed_distance(center, pa) || !boundaries[j].signed_distance(center, pb)) continue;
            if (!(pa - bound < 0. && pb - bound < 0.)) continue;
            Cell c;
            if (build_cell(i, j, from, to, boundaries, h, gx, gw, c)) cells.push_back(std::move(c));
          }
    }
  }
  const size_t n = cells.size();
  res.cells = n;
  if (n == 0) return res;
  // solve_for_p_c (:186-645)
  for (Cell& c : cells) compute_diagonal(c, boundaries, dt);
  std::vector<std::vector<std::pair<size_t, bool>>> touching(nb);  // BodyCellIndex (:647-676)
  for (size_t c = 0; c < n; ++c) {
    touching[cells[c].a].push_back({c, true});
    touching[cells[c].b].push_back({c, false});
  }
  std::vector<double> p(n, 0.0), v_err(n, 0.0), s_p(n, 0.0);
  std::vector<V3> lambda(n, V3{0, 0, 0}), v_tang(n, V3{0, 0, 0}), s_l(n, V3{0, 0, 0});
  std::vector<V3> ef(nb), et(nb), vt(nb), wt(nb);
  auto accumulate = [&]() {  // accumulate_extra_forces (:928-965)
    for (size_t b = 0; b < nb; ++b) {
      V3 f{0, 0, 0}, t{0, 0, 0};
      for (auto [ci, is_a] : touching[b]) {
        const Cell& c = cells[ci];
        const RigidBodyMotion* ma = motion_of(boundaries[c.a]);
        const RigidBodyMotion* mb = motion_of(boundaries[c.b]);
        if (is_a) {
          f += p[ci] * c.f_a + lambda[ci];
          if (ma) t += p[ci] * c.tau_a + cross(c.center - ma->center_of_mass, lambda[ci]);
        } else {
          f += p[ci] * c.f_b - lambda[ci];
          if (mb) t += p[ci] * c.tau_b - cross(c.center - mb->center_of_mass, lambda[ci]);
        }
      }
      ef[b] = f;
      et[b] = t;
    }
  };
  auto predict = [&]() {
    for (size_t b = 0; b < nb; ++b) {  // compute_trial_velocities (:967-994)
      const RigidBodyMotion* m = motion_of(boundaries[b]);
      if (!m) {
        vt[b] = wt[b] = V3{0, 0, 0};
        continue;
      }
      vt[b] = m->linear_velocity + dt / m->mass * (m->force + ef[b]);
      wt[b] = mul(m->inertia_tensor_inv_world, m->angular_momentum + dt * (m->torque + et[b]));
    }
    for (size_t c = 0; c < n; ++c) {
      const Cell& k = cells[c];
      // predicted_volume_error (:996-1009)
      v_err[c] = -k.volume + dt * (((dot(vt[k.a], k.f_a) + dot(wt[k.a], k.tau_a)) + dot(vt[k.b], k.f_b)) +
                                   dot(wt[k.b], k.tau_b));
      // predicted_tangential_velocity (:1011-1033)
      const RigidBodyMotion* ma = motion_of(boundaries[k.a]);
      const RigidBodyMotion* mb = motion_of(boundaries[k.b]);
      if (ma && mb) {
        const V3 v_rel = ((vt[k.a] + cross(wt[k.a], k.center - ma->center_of_mass)) - vt[k.b]) -
                         cross(wt[k.b], k.center - mb->center_of_mass);
        v_tang[c] = mul(k.tproj, v_rel);
      } else {
        v_tang[c] = V3{0, 0, 0};
      }
    }
  };
  // projected_jacobi (:1035-1102)
  auto jacobi = [&](std::vector<double>& p_out, std::vector<V3>& l_out) {
    std::vector<uint32_t> active(nb, 0);
    for (size_t b = 0; b < nb; ++b)
      for (auto [ci, is_a] : touching[b])
        if (v_err[ci] < 0.0 || p[ci] > 0.0) ++active[b];
    p_out.resize(n);
    l_out.resize(n);
    for (size_t c = 0; c < n; ++c) {
      const Cell& k = cells[c];
      const double n_max = (double)std::max<uint32_t>(std::max(active[k.a], active[k.b]), 1);
      const double alpha = kRelaxation / n_max / std::max(k.acc_p, kMinDiagonal);
      p_out[c] = std::max(p[c] - alpha * v_err[c], 0.0);
      const double lmax = kFrictionCoefficient * p[c] * norm(k.f_a);
      V3 star = -v_tang[c] / std::max(k.acc_f, kMinDiagonal);
      const double sn = norm(star);
      if (sn > lmax) star = lmax * star / sn;
      V3 ln = lambda[c] + kRelaxation / n_max * star;
      const double lnn = norm(ln);
      l_out[c] = lnn > lmax ? lmax * ln / lnn : ln;
    }
  };
  std::vector<double> pp(n), vtn(n), dev(n);
  auto merits = [&]() {
    for (size_t c = 0; c < n; ++c) {
      pp[c] = p[c] * std::max(cells[c].acc_p, kMinDiagonal);
      vtn[c] = norm(v_tang[c]);
      dev[c] = std::max(cells[c].acc_f, kMinDiagonal) *
               (kFrictionCoefficient * p[c] * norm(cells[c].f_a) - norm(lambda[c]));
    }
  };
  accumulate();
  predict();
  std::vector<double> pj, gp(n);
  std::vector<V3> lj, gl(n);
  jacobi(pj, lj);
  double prev_gp = 0, prev_gl = 0;
  for (size_t c = 0; c < n; ++c) {
    gp[c] = -(pj[c] - p[c]);
    gl[c] = -(lj[c] - lambda[c]);
    s_p[c] = -gp[c];
    s_l[c] = -gl[c];
    prev_gp += gp[c] * gp[c];
    prev_gl += dot(gl[c], gl[c]);
  }
  p = pj;
  lambda = lj;
  accumulate();
  predict();
  merits();
  uint32_t it = 0;
  auto more = [&]() {
    if (contact_fixed_sweeps) return it < contact_fixed_sweeps;
    return !(mean_fischer_burmeister(pp, v_err) < kFbTolPressure &&
             mean_fischer_burmeister(vtn, dev) < kFbTolFriction) &&
           it < contact_iteration_cap;
  };
  while (more()) {
    jacobi(pj, lj);
    double gpn = 0, gln = 0;
    for (size_t c = 0; c < n; ++c) {
      gp[c] = -(pj[c] - p[c]);
      gl[c] = -(lj[c] - lambda[c]);
      gpn += gp[c] * gp[c];
      gln += dot(gl[c], gl[c]);
    }
    const double beta = (gpn + gln) / std::max(prev_gp + prev_gl, std::numeric_limits<double>::min());
    if (beta > 1.0) {
      std::fill(s_p.begin(), s_p.end(), 0.0);
      std::fill(s_l.begin(), s_l.end(), V3{0, 0, 0});
      p = pj;
      lambda = lj;
    } else {
      std::vector<double> p_out(n), sp_out(n);
      std::vector<V3> l_out(n), sl_out(n);
      for (size_t c = 0; c < n; ++c) {
        const double p_nncg = pj[c] + beta * s_p[c];
        if (p_nncg < 0.0) {
          p_out[c] = pj[c];
          sp_out[c] = 0.0;
        } else {
          p_out[c] = p_nncg;
          sp_out[c] = beta * s_p[c] - gp[c];
        }
        // the friction cone of the iterate before this update (:452-467)
        const V3 l_nncg = lj[c] + beta * s_l[c];
        const V3 tp = mul(cells[c].tproj, l_nncg);
        const double lmax = kFrictionCoefficient * p[c] * norm(cells[c].f_a);
        if (norm(tp) > lmax) {
          l_out[c] = lj[c];
          sl_out[c] = V3{0, 0, 0};
        } else {
          l_out[c] = tp;
          sl_out[c] = beta * s_l[c] - gl[c];
        }
      }
      p = p_out;
      s_p = sp_out;
      lambda = l_out;
      s_l = sl_out;
    }
    prev_gp = gpn;
    prev_gl = gln;
    accumulate();
    predict();
    merits();
    ++it;
  }
  res.iterations = it;
  accumulate();
  for (size_t b = 0; b < nb; ++b) {
    res.force[b] = ef[b];
    res.torque[b] = et[b];
    if (commit && boundaries[b].dynamic) {  // add_force_and_torque (rigid_body_motion.rs:156-159)
      boundaries[b].state.force += ef[b];
      boundaries[b].state.torque += et[b];
    }
  }
  return res;
}

// :1440-1453: contact forces first, then every body integrates.
void VolumeMapBoundary::step_forward_in_time(double dt) {
  solve_contacts(dt, true);
  for (auto& b : boundaries)
    if (b.dynamic) b.state.step_forward_in_time(dt);
}

// ---------------------------------------------------------------------------
// Volume-map / SDF field construction
// ---------------------------------------------------------------------------
// Closest point on a triangle (Ericson, Real-Time Collision Detection 5.1.5);
// returns the feature: 0 face, 1..3 vertex a,b,c, 4 edge ab, 5 edge bc, 6 edge ca.
static V3 closest_on_triangle(V3 p, V3 a, V3 b, V3 c, int& feat) {
  V3 ab = b - a, ac = c - a, ap = p - a;
  double d1 = dot(ab, ap), d2 = dot(ac, ap);
  if (d1 <= 0 && d2 <= 0) { feat = 1; return a; }
  V3 bp = p - b;
  double d3 = dot(ab, bp), d4 = dot(ac, bp);
  if (d3 >= 0 && d4 <= d3) { feat = 2; return b; }
  double vc = d1 * d4 - d3 * d2;
  if (vc <= 0 && d1 >= 0 && d3 <= 0) { feat = 4; double v = d1 / (d1 - d3); return a + ab * v; }
  V3 cp = p - c;
  double d5 = dot(ab, cp), d6 = dot(ac, cp);
  if (d6 >= 0 && d5 <= d6) { feat = 3; return c; }
  double vb = d5 * d2 - d1 * d6;
  if (vb <= 0 && d2 >= 0 && d6 <= 0) { feat = 6; double w = d2 / (d2 - d6); return a + ac * w; }
  double va = d3 * d6 - d5 * d4;
  if (va <= 0 && (d4 - d3) >= 0 && (d5 - d6) >= 0) {
    feat = 5;
    double w = (d4 - d3) / ((d4 - d3) + (d5 - d6));
    return b + (c - b) * w;
  }
  feat = 0;
  double denom = 1.0 / (va + vb + vc);
  double v = vb * denom, w = vc * denom;
  return a + ab * v + ac * w;
}

// Signed distance to a closed triangle mesh: distance to the closest point,
// negative where (p - proj) points against the closest feature's angle-weighted
// pseudo-normal (volume_map_boundary.rs:1655-1671; the mesh's outward side is
// the side its face winding points to).
double mesh_signed_distance(const TriMeshD& mesh, V3 p) {
  size_t nt = mesh.f.size() / 3;
  double best = std::numeric_limits<double>::infinity();
  size_t bt = 0;
  int bf = 0;
  V3 bproj;
  for (size_t t = 0; t < nt; ++t) {
    V3 a = mesh.v[mesh.f[3 * t]], b = mesh.v[mesh.f[3 * t + 1]], c = mesh.v[mesh.f[3 * t + 2]];
    int feat;
    V3 q = closest_on_triangle(p, a, b, c, feat);
    double d2 = norm_squared(p - q);
    if (d2 < best) { best = d2; bt = t; bf = feat; bproj = q; }
  }
  auto face_normal = [&](size_t t) {
    V3 a = mesh.v[mesh.f[3 * t]], b = mesh.v[mesh.f[3 * t + 1]], c = mesh.v[mesh.f[3 * t + 2]];
    V3 nn = cross(b - a, c - a);
    return nn / norm(nn);
  };
  auto angle_at = [&](size_t t, uint32_t vid) {
    uint32_t i0 = mesh.f[3 * t], i1 = mesh.f[3 * t + 1], i2 = mesh.f[3 * t + 2];
    uint32_t o1, o2;
    if (vid == i0) { o1 = i1; o2 = i2; } else if (vid == i1) { o1 = i2; o2 = i0; } else { o1 = i0; o2 = i1; }
    V3 e1 = mesh.v[o1] - mesh.v[vid], e2 = mesh.v[o2] - mesh.v[vid];
    double cs = dot(e1, e2) / (norm(e1) * norm(e2));
    cs = std::max(-1.0, std::min(1.0, cs));
    return std::acos(cs);
  };
  V3 nrm;
  if (bf == 0) {
    nrm = face_normal(bt);
  } else if (bf <= 3) {
    uint32_t vid = mesh.f[3 * bt + (bf - 1)];
    V3 acc{0, 0, 0};
    for (size_t t = 0; t < nt; ++t)
      if (mesh.f[3 * t] == vid || mesh.f[3 * t + 1] == vid || mesh.f[3 * t + 2] == vid)
        acc += face_normal(t) * angle_at(t, vid);
    nrm = acc;
  } else {
    uint32_t ea, eb;
    uint32_t i0 = mesh.f[3 * bt], i1 = mesh.f[3 * bt + 1], i2 = mesh.f[3 * bt + 2];
    if (bf == 4) { ea = i0; eb = i1; } else if (bf == 5) { ea = i1; eb = i2; } else { ea = i2; eb = i0; }
    V3 acc{0, 0, 0};
    for (size_t t = 0; t < nt; ++t) {
      bool ha = false, hb = false;
      for (int k = 0; k < 3; ++k) { ha |= mesh.f[3 * t + k] == ea; hb |= mesh.f[3 * t + k] == eb; }
      if (ha && hb) acc += face_normal(t);
    }
    nrm = acc;
  }
  V3 diff = p - bproj;
  double dist = norm(diff);
  return dot(diff, nrm) < 0.0 ? -dist : dist;
}

// Gauss-Legendre nodes/weights on [-1,1] by Newton iteration on P_n.
bool gauss_legendre(int deg, std::vector<double>& x, std::vector<double>& w) {
  x.assign(deg, 0); w.assign(deg, 0);
  for (int i = 0; i < deg; ++i) {
    double z = std::cos(PI * (i + 0.75) / (deg + 0.5)), pp = 0;
    for (int it = 0; it < 100; ++it) {
      double p1 = 1, p2 = 0;
      for (int j = 1; j <= deg; ++j) { double p3 = p2; p2 = p1; p1 = ((2.0 * j - 1) * z * p2 - (j - 1.0) * p3) / j; }
      pp = deg * (z * p1 - p2) / (z * z - 1.0);
      double z1 = z;
      z = z1 - p1 / pp;
      if (std::fabs(z - z1) < 1e-16) break;
    }
    double p1 = 1, p2 = 0;
    for (int j = 1; j <= deg; ++j) { double p3 = p2; p2 = p1; p1 = ((2.0 * j - 1) * z * p2 - (j - 1.0) * p3) / j; }
    pp = deg * (z * p1 - p2) / (z * z - 1.0);
    x[i] = -z;
    w[i] = 2.0 / ((1.0 - z * z) * pp * pp);
  }
  return true;
}

static void grid_dims(V3 mn, V3 mx, double dx, int64_t n[3]) {  // discretization.rs:108-112
  n[0] = (int64_t)std::llround((mx.x - mn.x) / dx);
  n[1] = (int64_t)std::llround((mx.y - mn.y) / dx);
  n[2] = (int64_t)std::llround((mx.z - mn.z) / dx);
}

// Shared pruning pass (discretization.rs:186-236): keep the 32 nodes of every
// cell whose nodes are all valid and not all beyond the prune bounds.
template <class F>
static void discretize(Serendipity& out, V3 mn, V3 mx, double dx, bool has_lo, double lo,
                       bool has_hi, double hi, F f) {
  out.x_min = mn; out.x_max = mx; out.dx = dx;
  grid_dims(mn, mx, dx, out.n);
  const int64_t NX = out.NX(), NY = out.NY(), NZ = out.NZ();
  const double NaN = std::numeric_limits<double>::quiet_NaN();
  std::vector<double> raw((size_t)(NX * NY * NZ), NaN);
  std::vector<char> used((size_t)(NX * NY * NZ), 0);
  const auto& rn = ref_nodes();
  for (int64_t cz = 0; cz < out.n[2]; ++cz)
    for (int64_t cy = 0; cy < out.n[1]; ++cy)
      for (int64_t cx = 0; cx < out.n[0]; ++cx)
        for (const auto& r : rn)
          used[(size_t)(((3 * cz + r.oz) * NY + 3 * cy + r.oy) * NX + 3 * cx + r.ox)] = 1;
  std::vector<size_t> keys;
  for (size_t k = 0; k < used.size(); ++k) if (used[k]) keys.push_back(k);
parallel_for((size_t)(keys.size()), [&](size_t b__, size_t e__) {
  for (long long ii = (long long)b__; ii < (long long)e__; ++ii) {
    size_t k = keys[(size_t)ii];
    int64_t kx = (int64_t)(k % (size_t)NX), ky = (int64_t)((k / (size_t)NX) % (size_t)NY),
            kz = (int64_t)(k / (size_t)(NX * NY));
    V3 p{mn.x + (double)kx / 3.0 * dx, mn.y + (double)ky / 3.0 * dx, mn.z + (double)kz / 3.0 * dx};
    double v;
    if (f(p, v)) raw[k] = v;
  }
  });
  out.nodes.assign(raw.size(), NaN);
  for (int64_t cz = 0; cz < out.n[2]; ++cz)
    for (int64_t cy = 0; cy < out.n[1]; ++cy)
      for (int64_t cx = 0; cx < out.n[0]; ++cx) {
        size_t idx[32];
        bool ok = true, all_lo = true, all_hi = true;
        for (int a = 0; a < 32; ++a) {
          idx[a] = (size_t)(((3 * cz + rn[a].oz) * NY + 3 * cy + rn[a].oy) * NX + 3 * cx + rn[a].ox);
          double v = raw[idx[a]];
          if (std::isnan(v)) { ok = false; break; }
          if (!(v < lo)) all_lo = false;
          if (!(v > hi)) all_hi = false;
        }
        if (!ok) continue;
        bool prune = (has_lo && all_lo) || (has_hi && all_hi);
        if (prune) continue;
        for (int a = 0; a < 32; ++a) out.nodes[idx[a]] = raw[idx[a]];
      }
}

static void mesh_aabb(const TriMeshD& mesh, V3& mn, V3& mx) {
  mn = {1e300, 1e300, 1e300}; mx = {-1e300, -1e300, -1e300};
  for (V3 v : mesh.v) {
    mn.x = std::min(mn.x, v.x); mn.y = std::min(mn.y, v.y); mn.z = std::min(mn.z, v.z);
    mx.x = std::max(mx.x, v.x); mx.y = std::max(mx.y, v.y); mx.z = std::max(mx.z, v.z);
  }
}

void build_sdf_field(const TriMeshD& mesh, double dx, double r, Serendipity& out) {
  V3 mn, mx;  // volume_map_boundary.rs:1554-1576
  mesh_aabb(mesh, mn, mx);
  double pad = 3.1 * r;
  V3 pv{pad, pad, pad};
  discretize(out, mn - pv, mx + pv, dx, true, -pad, true, pad, [&](V3 p, double& v) {
    v = mesh_signed_distance(mesh, p);
    return true;
  });
}

static inline double cubic_extension_fn(double sd, double r) {  // :1717-1727
  if (sd >= r) return 0.;
  if (sd <= 0.) return 1.;
  return kernel_function(V3{sd, 0., 0.}, r) / kernel_function(V3{0, 0, 0}, r);
}

// SDFnWrapper::volume (:1684-1715) with gauss_legendre_integrate_ball
// (discretization.rs:33-79).
double volume_at(const Serendipity& sdf, V3 p, double r, int degree, bool& ok) {
  ok = true;
  double sdc;
  if (!sdf.function(p, sdc)) return 0.0;
  if (sdc >= 2.0 * r) return 0.0;
  if (sdc <= -r) return 4.0 / 3.0 * PI * powi3(r);
  static thread_local std::vector<double> gx, gw;
  static thread_local int gdeg = -1;
  if (gdeg != degree) { gauss_legendre(degree, gx, gw); gdeg = degree; }
  auto integrate = [&](double a, double b, auto fn) {
    double s = -0.0;
    for (int i = 0; i < degree; ++i) s += fn(0.5 * ((b - a) * gx[i] + (b + a))) * gw[i];
    return 0.5 * (b - a) * s;
  };
  bool err = false;
  double res = integrate(0.0, r, [&](double rr) {
    if (err) return 0.0;
    return powi2(rr) * integrate(0.0, PI, [&](double th) {
      if (err) return 0.0;
      return std::sin(th) * integrate(0.0, 2. * PI, [&](double ph) {
        if (err) return 0.0;
        V3 q{p.x + rr * std::sin(th) * std::cos(ph), p.y + rr * std::sin(th) * std::sin(ph),
             p.z + rr * std::cos(th)};
        double sd;
        if (!sdf.function(q, sd)) { err = true; return 0.0; }
        return cubic_extension_fn(sd, r);
      });
    });
  });
  if (err) { ok = false; return 0.0; }
  return res;
}

void build_volume_map_field(const TriMeshD& mesh, const Serendipity& sdf, double dx, double r,
                            int degree, Serendipity& out) {
  V3 mn, mx;  // volume_map_boundary.rs:1599-1618
  mesh_aabb(mesh, mn, mx);
  double pad = 2. * r + dx / 6.0;
  V3 pv{pad, pad, pad};
  discretize(out, mn - pv, mx + pv, dx, true, 0., false, 0., [&](V3 p, double& v) {
    bool ok;
    double vol = volume_at(sdf, p, r, degree, ok);
    if (!ok) return false;
    v = std::min(std::max(vol, 0.0), 4.0 / 3.0 * PI * powi3(r));
    return true;
  });
}

// ---------------------------------------------------------------------------
// System (SL/sph/mod.rs)
// ---------------------------------------------------------------------------
System::System(const System& o)
    : params(o.params), sp(o.sp), solver(o.solver), integrator(o.integrator), fluid(o.fluid),
      fluid_nl(o.fluid_nl), boundary(o.boundary ? o.boundary->clone() : nullptr), ns(o.ns),
      iisph(o.iisph), density_pred(o.density_pred),
      time_steps_propagated(o.time_steps_propagated), average_density(o.average_density),
      wall_clock(o.wall_clock), hash_duplicates(o.hash_duplicates) {}

double System::time() const {  // :107-116
  if (params.cfl) return params.current_time;
  return params.time_offset +
         (double)(time_steps_propagated - params.time_offset_steps) * params.time_increment;
}

void System::new_boxed() {  // :389-421
  size_t ip = integrator == Integrator::TakePredicted ? 1 : 0;
  size_t sp_slots = (solver == Solver::IISPH || solver == Solver::IISPHwOST) ? 1 : 0;
  size_t sv_slots = solver == Solver::SESPH ? 0 : 1;
  fluid.resize_slots(ip, ip, sp_slots, sv_slots);
  ns = SpatialHashing(params.kernel_support_radius);
  update();
}

void integrate(Integrator scheme, Fluid& fluid, size_t n, double dt) {
  if (scheme == Integrator::EulerCromer) {  // euler_cromer.rs:12-25
    parallel_for(n, [&](size_t b, size_t e) {
      for (size_t i = b; i < e; ++i) {
        V3 v = fluid.velocity[i] + fluid.acceleration[i] * dt;
        fluid.velocity[i] = v;
        fluid.position[i] = fluid.position[i] + v * dt;
      }
    });
  } else {  // take_predicted.rs:14-27: dt unused
    std::swap(fluid.position, fluid.integrator_position_slots[0]);
    std::swap(fluid.velocity, fluid.integrator_velocity_slots[0]);
  }
}

void System::step_forward_in_time() {  // :125-144
  auto t0 = std::chrono::steady_clock::now();
  double dt = params.time_increment;
  const size_t n = fluid.len();
  integrate(integrator, fluid, n, dt);
  boundary->step_forward_in_time(dt);
  time_steps_propagated += 1;
  if (params.cfl) params.current_time += params.time_increment;
  update();
  wall_clock = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
}

void System::update() {  // :674-731
  size_t id = 0;
  while (id < fluid.len()) {
    if (fluid.position[id].z < params.disable_particles_below) fluid.disable(id);
    else ++id;
  }
  fluid.drop_inactive();
  if (params.cfl) {  // :825-829
    double max_speed = calc_max_speed();
    double cfl_dt = params.cfl_number * params.rest_density_grid_spacing / max_speed;
    params.time_increment = std::min(params.max_time_increment, cfl_dt);
  }
  ns.find_samples(params.kernel_support_radius, fluid.position, fluid.position, fluid_nl);
  hash_duplicates = ns.last_duplicates;
  boundary->find_boundary_samples(params.kernel_support_radius, fluid.position,
                                  params.rest_density_grid_spacing);
  get_volume();
  calc_acceleration();
  average_density = calc_average_mass_density();
}

void System::calc_acceleration() {  // :658-671
  for (auto& a : fluid.acceleration) a = {0, 0, 0};
  add_gravity_acceleration();
  add_viscosity_acceleration();
  switch (solver) {
    case Solver::SESPH: sesph(); break;
    case Solver::SESPHwSplitting: sesph_w_splitting(); break;
    case Solver::IISPH: iisph_solve(); break;
    case Solver::IISPHwOST: iisph_w_ost(); break;
  }
}

double System::calc_max_speed() const {  // :424-441
  double m = 0.0;
  for (size_t i = 0; i < fluid.len(); ++i) m = std::max(m, norm(fluid.velocity[i]));
  return m;
}
double System::calc_average_mass_density() const {  // :444-486
  const size_t n = fluid.len();
  if (n == 0) return 0.0;
  double s = 0;
  for (size_t i = 0; i < n; ++i) {
    double v = fluid.volume[i];
    s += v < params.rest_volume ? fluid.mass[i] / v : fluid.mass[i] / params.rest_volume;
  }
  return s / (double)n;
}
double System::calc_average_mass_density_error() const {  // :489-529
  const size_t n = fluid.len();
  if (n == 0) return 0.0;
  double s = 0;
  for (size_t i = 0; i < n; ++i) {
    double v = fluid.volume[i];
    s += v < params.rest_volume ? params.rest_volume / v : 1.;
  }
  return 100. * (s / (double)n - 1.);
}
double System::calc_average_kinetic_energy() const {  // :532-564
  const size_t n = fluid.len();
  if (n == 0) return 0.0;
  double s = 0;
  for (size_t i = 0; i < n; ++i) s += 0.5 * fluid.mass[i] * norm_squared(fluid.velocity[i]);
  return s / (double)n;
}
Measurement System::take_measurement() const {  // :147-184
  Measurement m{};
  m.time = time();
  m.density = average_density;
  m.density_error = calc_average_mass_density_error();
  m.kinetic_energy = calc_average_kinetic_energy();
  bool sesph_like = solver == Solver::SESPH || solver == Solver::SESPHwSplitting;
  m.stiffness = sesph_like ? sp.stiffness : 0.0;
  m.fluid_viscosity = params.fluid_viscosity;
  m.boundary_viscosity = params.boundary_viscosity;
  m.fluid_depth = 0.0;
  m.rest_density_grid_spacing = params.rest_density_grid_spacing;
  m.kernel_support_radius = params.kernel_support_radius;
  m.time_step_size = params.time_increment;
  m.target_density_error = sesph_like ? 0.0 : sp.target_density_error;
  m.solver_iterations = sesph_like ? 0 : iisph.last_solver_iterations;
  m.relaxation_factor = sesph_like ? 0.0 : sp.relaxation_factor;
  m.time_step_wall_clock_time = wall_clock;
  m.predicted_density_error = sesph_like ? 0.0 : iisph.predicted_density_error;
  return m;
}

// quantities.rs:14-61
void System::get_volume() {
  const size_t n = fluid.len();
  const double h = params.kernel_support_radius, V0 = params.rest_volume;
parallel_for((size_t)(n), [&](size_t b__, size_t e__) {
  for (long long ii = (long long)b__; ii < (long long)e__; ++ii) {
    size_t id = (size_t)ii;
    double accu = 0.;
    for (const size_t* it = fluid_nl.begin(id); it != fluid_nl.end(id); ++it)
      accu += V0 * kernel_function(fluid.position[id] - fluid.position[*it], h);
    for (size_t bi = 0; bi < boundary->count(); ++bi) {
      const Boundary& b = boundary->at(bi);
      auto r = b.get_neighbors(id, RequestMode::Normal);
      for (const size_t* it = r.first; it != r.second; ++it)
        accu += b.volume(*it) * kernel_function(fluid.position[id] - b.position(*it), h);
    }
    fluid.volume[id] = V0 / accu;
  }
  });
}

// sph/mod.rs:241-341 (get_quantity_at_positions) with the sums of
// quantities.rs:14-330: fluid samples of each evaluation position by the
// system's spatial hashing, boundary samples searched for the evaluation
// positions (Normal mode; speed and volume only), f64 sums cast to f32.
// Quantity codes follow ScalarQuantity: 0 speed, 1 volume, 2 density,
// 3 density error, 4 pressure, 5 kinetic energy. As in the reference, the
// boundary's per-particle sample lists then describe the evaluation
// positions until the next update rebuilds them.
std::vector<float> System::quantity_at_positions(int q, const std::vector<V3>& eval) {
  if (q < 0 || q > 5) throw std::invalid_argument("unknown quantity");
  const double h = params.kernel_support_radius, V0 = params.rest_volume;
  NeighborList nl;
  ns.find_samples(h, eval, fluid.position, nl);
  boundary->find_boundary_samples(h, eval, params.rest_density_grid_spacing);
  std::vector<float> out(eval.size());
  parallel_for(eval.size(), [&](size_t b__, size_t e__) {
    for (size_t id = b__; id < e__; ++id) {
      const V3 x = eval[id];
      double s = 0.;
      V3 sv{0., 0., 0.};
      for (const size_t* it = nl.begin(id); it != nl.end(id); ++it) {
        const size_t j = *it;
        const double w = kernel_function(x - fluid.position[j], h);
        switch (q) {
          case 0: sv += fluid.velocity[j] * fluid.volume[j] * w; break;       // :89-99
          case 1: s += V0 * w; break;                                         // :33-40
          case 2: s += fluid.mass[j] * w; break;                              // :139-148
          case 3: {                                                           // :195-211
            // called with the fluid MASSES in the volume slot (sph/mod.rs:302-311)
            const double m = fluid.mass[j];
            if (m < V0) s += (V0 / m - 1.) * m * w;
            break;
          }
          case 4: s += fluid.pressure[j] * fluid.volume[j] * w; break;        // :255-264
          case 5:                                                             // :309-319
            s += 0.5 * fluid.mass[j] * norm_squared(fluid.velocity[j]) * fluid.volume[j] * w;
            break;
        }
      }
      if (q == 0 || q == 1) {
        for (size_t bi = 0; bi < boundary->count(); ++bi) {
          const Boundary& b = boundary->at(bi);
          auto r = b.get_neighbors(id, RequestMode::Normal);
          for (const size_t* it = r.first; it != r.second; ++it) {
            const double w = kernel_function(x - b.position(*it), h);
            if (q == 0) sv += b.velocity(*it) * b.volume(*it) * w;
            else s += b.volume(*it) * w;
          }
        }
      }
      double val;
      switch (q) {
        case 0: val = norm(sv); break;
        case 1: val = V0 / s; break;
        case 3: val = 100. * s; break;
        default: val = s;
      }
      out[id] = (float)val;
    }
  });
  return out;
}

// non_pressure_accelerations.rs:64-103
void System::add_gravity_acceleration() {
  const double g = 9.81;
  const size_t n = fluid.len();
  if (params.gravity == Gravity::Uniform) {
    for (size_t i = 0; i < n; ++i) fluid.acceleration[i] += V3{0.0, 0.0, -g};
    for (size_t bi = 0; bi < boundary->count(); ++bi) {
      RigidBodyMotion* m = boundary->at(bi).motion();
      if (m) m->add_force(V3{0.0, 0.0, -g} * m->mass, m->center_of_mass);
    }
  } else {
    V3 c = params.gravity_center;
    for (size_t i = 0; i < n; ++i) {
      V3 d = c - fluid.position[i];
      double dist = std::sqrt(norm_squared(d) + 1e-4);
      fluid.acceleration[i] += (g * d) / dist;
    }
    for (size_t bi = 0; bi < boundary->count(); ++bi) {
      RigidBodyMotion* m = boundary->at(bi).motion();
      if (!m) continue;
      V3 d = c - m->center_of_mass;
      double dist = std::sqrt(norm_squared(d) + 1e-4);
      V3 acc = (g * d) / dist;
      m->add_force(acc * m->mass, m->center_of_mass);
    }
  }
}

struct ForceRec { size_t id; V3 force, loc; };

// non_pressure_accelerations.rs:106-185
void System::add_viscosity_acceleration() {
  const size_t n = fluid.len();
  const double h = params.kernel_support_radius;
  const double eps = 0.01 * powi2(params.rest_density_grid_spacing);
  std::vector<std::vector<ForceRec>> forces(n);
parallel_for((size_t)(n), [&](size_t b__, size_t e__) {
  for (long long ii = (long long)b__; ii < (long long)e__; ++ii) {
    size_t id = (size_t)ii;
    V3 xi = fluid.position[id], vi = fluid.velocity[id];
    V3 accu{0, 0, 0};
    for (const size_t* it = fluid_nl.begin(id); it != fluid_nl.end(id); ++it) {
      size_t j = *it;
      V3 xij = xi - fluid.position[j];
      accu += params.fluid_viscosity * 2. * (3. + 2.) * fluid.volume[j] *
              dot(vi - fluid.velocity[j], xij) / (norm_squared(xij) + eps) *
              kernel_gradient(xij, h);
    }
    for (size_t bi = 0; bi < boundary->count(); ++bi) {
      const Boundary& b = boundary->at(bi);
      auto r = b.get_neighbors(id, RequestMode::ViscosityAcceleration);
      for (const size_t* it = r.first; it != r.second; ++it) {
        V3 xb = b.position(*it);
        V3 xib = xi - xb;
        V3 acc = params.boundary_viscosity * 2. * (3. + 2.) * b.volume(*it) *
                 dot(vi - b.velocity(*it), xib) / (norm_squared(xib) + eps) *
                 kernel_gradient(xib, h);
        V3 force = fluid.mass[id] * acc;
        if (b.is_dynamic()) forces[id].push_back({bi, -force, xb});
        accu += acc;
      }
    }
    fluid.acceleration[id] += accu;
  }
  });
  for (auto& fl : forces)
    for (auto& f : fl) boundary->add_force_onto_boundary(f.id, f.force, f.loc);
}

// pressure_solver/mod.rs:90-108
void System::set_pred_vel_by_applying_acc(bool to_pred) {
  const size_t n = fluid.len();
  const double dt = params.time_increment;
  auto& vp = fluid.solver_velocity_slots[0];
  for (size_t i = 0; i < n; ++i) {
    V3 base = to_pred ? vp[i] : fluid.velocity[i];
    vp[i] = base + dt * fluid.acceleration[i];
  }
}

// pressure_solver/mod.rs:121-195
void System::add_pressure_acceleration(std::vector<V3>* custom, bool pred_pos, bool overwrite,
                                       bool mirror) {
  std::vector<V3>& target = custom ? *custom : fluid.acceleration;
  const std::vector<V3>& pos = pred_pos ? fluid.solver_position_slots[0] : fluid.position;
  const size_t n = fluid.len();
  const double h = params.kernel_support_radius;
  const double wgt = params.boundary_pressure_acceleration_weighting;
  std::vector<std::vector<ForceRec>> forces(mirror ? n : 0);
parallel_for((size_t)(n), [&](size_t b__, size_t e__) {
  for (long long ii = (long long)b__; ii < (long long)e__; ++ii) {
    size_t id = (size_t)ii;
    V3 accu{0, 0, 0};
    double vi = fluid.volume[id], mi = fluid.mass[id], pi = fluid.pressure[id];
    for (const size_t* it = fluid_nl.begin(id); it != fluid_nl.end(id); ++it) {
      size_t j = *it;
      V3 r = pos[id] - pos[j];
      accu -= vi / mi * fluid.volume[j] * (pi + fluid.pressure[j]) * kernel_gradient(r, h);
    }
    for (size_t bi = 0; bi < boundary->count(); ++bi) {
      const Boundary& b = boundary->at(bi);
      auto rr = b.get_neighbors(id, RequestMode::Normal);
      for (const size_t* it = rr.first; it != rr.second; ++it) {
        V3 xb = b.position(*it);
        V3 force = 2. * wgt * vi * b.volume(*it) * pi * kernel_gradient(pos[id] - xb, h);
        if (mirror && b.is_dynamic()) forces[id].push_back({bi, force, xb});
        accu -= force / mi;
      }
    }
    if (overwrite) target[id] = accu;
    else target[id] += accu;
  }
  });
  if (mirror)
    for (auto& fl : forces)
      for (auto& f : fl) boundary->add_force_onto_boundary(f.id, f.force, f.loc);
}

// sesph.rs:31-67
void System::sesph() {
  const size_t n = fluid.len();
  for (size_t i = 0; i < n; ++i)
    fluid.pressure[i] = sp.stiffness * std::max(params.rest_volume / fluid.volume[i] - 1., 0.);
  add_pressure_acceleration(nullptr, false, false, true);
}

// sesph_with_splitting.rs:33-152
void System::sesph_w_splitting() {
  const size_t n = fluid.len();
  density_pred.assign(n, 0.0);
  set_pred_vel_by_applying_acc(false);
  const double h = params.kernel_support_radius, dt = params.time_increment;
  const auto& vp = fluid.solver_velocity_slots[0];
parallel_for((size_t)(n), [&](size_t b__, size_t e__) {
  for (long long ii = (long long)b__; ii < (long long)e__; ++ii) {
    size_t id = (size_t)ii;
    double accu = 0.;
    for (const size_t* it = fluid_nl.begin(id); it != fluid_nl.end(id); ++it) {
      size_t j = *it;
      V3 r = fluid.position[id] - fluid.position[j];
      accu += fluid.mass[j] * kernel_function(r, h) + dt * dot(vp[id] - vp[j], kernel_gradient(r, h));
    }
    for (size_t bi = 0; bi < boundary->count(); ++bi) {
      const Boundary& b = boundary->at(bi);
      auto rr = b.get_neighbors(id, RequestMode::Normal);
      for (const size_t* it = rr.first; it != rr.second; ++it) {
        V3 r = fluid.position[id] - b.position(*it);
        accu += b.volume(*it) * fluid.mass[id] / params.rest_volume * kernel_function(r, h) +
                dt * dot(vp[id], kernel_gradient(r, h));
      }
    }
    density_pred[id] = accu;
  }
  });
  for (size_t i = 0; i < n; ++i) {
    double vol = fluid.mass[i] / density_pred[i];
    fluid.pressure[i] = sp.stiffness * std::max(params.rest_volume / vol - 1., 0.);
  }
  add_pressure_acceleration(nullptr, false, false, true);
}

// iisph.rs:117-172
void System::set_source_term_vde() {
  const size_t n = fluid.len();
  const double h = params.kernel_support_radius, dt = params.time_increment;
  const auto& vp = fluid.solver_velocity_slots[0];
parallel_for((size_t)(n), [&](size_t b__, size_t e__) {
  for (long long ii = (long long)b__; ii < (long long)e__; ++ii) {
    size_t id = (size_t)ii;
    double accu = 0.;
    for (const size_t* it = fluid_nl.begin(id); it != fluid_nl.end(id); ++it) {
      size_t j = *it;
      V3 r = fluid.position[id] - fluid.position[j];
      accu -= dt * fluid.volume[j] * dot(vp[id] - vp[j], kernel_gradient(r, h));
    }
    for (size_t bi = 0; bi < boundary->count(); ++bi) {
      const Boundary& b = boundary->at(bi);
      auto rr = b.get_neighbors(id, RequestMode::Normal);
      for (const size_t* it = rr.first; it != rr.second; ++it) {
        V3 r = fluid.position[id] - b.position(*it);
        accu -= dt * b.volume(*it) * dot(vp[id] - b.velocity(*it), kernel_gradient(r, h));
      }
    }
    iisph.s_f[id] = accu;
  }
  });
}

// iisph.rs:175-251 (with_pred_positions = false in every production call)
void System::set_source_term_vp() {
  const size_t n = fluid.len();
  const double h = params.kernel_support_radius, dt = params.time_increment;
  const auto& vp = fluid.solver_velocity_slots[0];
parallel_for((size_t)(n), [&](size_t b__, size_t e__) {
  for (long long ii = (long long)b__; ii < (long long)e__; ++ii) {
    size_t id = (size_t)ii;
    double accu = 1. - params.rest_volume / fluid.volume[id];
    for (const size_t* it = fluid_nl.begin(id); it != fluid_nl.end(id); ++it) {
      size_t j = *it;
      V3 r = fluid.position[id] - fluid.position[j];
      accu -= dt * fluid.volume[j] * dot(vp[id] - vp[j], kernel_gradient(r, h));
    }
    for (size_t bi = 0; bi < boundary->count(); ++bi) {
      const Boundary& b = boundary->at(bi);
      auto rr = b.get_neighbors(id, RequestMode::Normal);
      for (const size_t* it = rr.first; it != rr.second; ++it) {
        V3 r = fluid.position[id] - b.position(*it);
        accu -= dt * b.volume(*it) * dot(vp[id] - b.velocity(*it), kernel_gradient(r, h));
      }
    }
    iisph.s_f[id] = accu;
  }
  });
}

// iisph.rs:254-342
void System::set_diagonal_element() {
  const size_t n = fluid.len();
  const double h = params.kernel_support_radius, dt = params.time_increment;
  const double wgt = params.boundary_pressure_acceleration_weighting;
parallel_for((size_t)(n), [&](size_t b__, size_t e__) {
  for (long long ii = (long long)b__; ii < (long long)e__; ++ii) {
    size_t id = (size_t)ii;
    V3 sum_fluid{0, 0, 0};
    double sum_fluid2 = 0.;
    for (const size_t* it = fluid_nl.begin(id); it != fluid_nl.end(id); ++it) {
      size_t j = *it;
      V3 g = kernel_gradient(fluid.position[id] - fluid.position[j], h);
      sum_fluid += fluid.volume[j] * g;
      sum_fluid2 -= powi2(dt) * fluid.volume[id] * powi2(fluid.volume[j]) / fluid.mass[j] *
                    norm_squared(g);
    }
    V3 sum_boundary{0, 0, 0};
    for (size_t bi = 0; bi < boundary->count(); ++bi) {
      const Boundary& b = boundary->at(bi);
      auto rr = b.get_neighbors(id, RequestMode::Normal);
      for (const size_t* it = rr.first; it != rr.second; ++it)
        sum_boundary += b.volume(*it) * kernel_gradient(fluid.position[id] - b.position(*it), h);
    }
    V3 c_f = -fluid.volume[id] / fluid.mass[id] * (sum_fluid + 2. * wgt * sum_boundary);
    iisph.a_ff[id] = powi2(dt) * dot(c_f, sum_fluid + sum_boundary) + sum_fluid2;
  }
  });
}

// iisph.rs:344-376
void System::iisph_initialize(bool clamp) {
  const size_t n = fluid.len();
  const double eps = sp.min_diagonal_element, w = sp.relaxation_factor;
  for (size_t id = 0; id < n; ++id) {
    double a = iisph.a_ff[id];
    if (a > eps || a < -eps) {
      double p = w * iisph.s_f[id] / a;
      fluid.pressure[id] = clamp ? std::max(p, 0.) : p;
    } else {
      fluid.pressure[id] = 0.;
    }
  }
}

// iisph.rs:401-560 (Jacobi: the pressure accelerations of a sweep all use
// the previous sweep's pressures)
void System::resolve_pressure_globally(bool after_iteration, uint32_t n_after, double tde,
                                       bool clamp) {
  const size_t n = fluid.len();
  if (n == 0) return;
  set_diagonal_element();
  iisph_initialize(clamp);
  const double h = params.kernel_support_radius, dt = params.time_increment;
  const double eps = sp.min_diagonal_element, w = sp.relaxation_factor;
  uint32_t it_count = 0;
  double err = std::numeric_limits<double>::infinity();
  auto converged = [&]() {  // :378-393
    if (after_iteration) return it_count > n_after;
    return (it_count > 2 && err < tde) || it_count >= sp.iteration_cap;
  };
  std::vector<double> e(n);
  while (!converged()) {
    add_pressure_acceleration(&iisph.pressure_acc_f, false, true, false);
    const auto& ap = iisph.pressure_acc_f;
parallel_for((size_t)(n), [&](size_t b__, size_t e__) {
    for (long long ii = (long long)b__; ii < (long long)e__; ++ii) {
      size_t id = (size_t)ii;
      double adp = 0.;
      for (const size_t* it = fluid_nl.begin(id); it != fluid_nl.end(id); ++it) {
        size_t j = *it;
        adp += powi2(dt) * fluid.volume[j] *
               dot(ap[id] - ap[j], kernel_gradient(fluid.position[id] - fluid.position[j], h));
      }
      for (size_t bi = 0; bi < boundary->count(); ++bi) {
        const Boundary& b = boundary->at(bi);
        auto rr = b.get_neighbors(id, RequestMode::Normal);
        for (const size_t* it = rr.first; it != rr.second; ++it)
          adp += powi2(dt) * b.volume(*it) *
                 dot(ap[id], kernel_gradient(fluid.position[id] - b.position(*it), h));
      }
      double a = iisph.a_ff[id], s = iisph.s_f[id];
      if (a < -eps) {
        double p = fluid.pressure[id] + w * (s - adp) / a;
        fluid.pressure[id] = clamp ? std::max(p, 0.) : p;
      }
      if ((s < 0. && clamp) || (!clamp && a < -eps)) e[id] = std::fabs(adp - s);
      else e[id] = 0.;
    }
  });
    double total = 0;
    for (size_t i = 0; i < n; ++i) total += e[i];
    err = total / (double)n * 100.0;
    it_count += 1;
  }
  iisph.last_solver_iterations = it_count;
  iisph.predicted_density_error = err;
}

// iisph.rs:55-96
void System::iisph_solve() {
  const size_t n = fluid.len();
  iisph.s_f.assign(n, 0.0); iisph.a_ff.assign(n, 0.0);
  iisph.pressure_acc_f.assign(n, V3{});
  set_pred_vel_by_applying_acc(false);
  set_source_term_vp();
  resolve_pressure_globally(false, 0, sp.target_density_error, true);
  add_pressure_acceleration(nullptr, false, false, true);
}

// iisph_optimized_source_term.rs:53-217
void System::iisph_w_ost() {
  const size_t n = fluid.len();
  iisph.s_f.assign(n, 0.0); iisph.a_ff.assign(n, 0.0);
  iisph.pressure_acc_f.assign(n, V3{});
  const double dt = params.time_increment;
  set_pred_vel_by_applying_acc(false);
  set_source_term_vde();
  resolve_pressure_globally(true, 3, 0.0, true);
  add_pressure_acceleration(nullptr, false, true, true);
  set_pred_vel_by_applying_acc(true);
  auto& xp = fluid.solver_position_slots[0];
  auto& vp = fluid.solver_velocity_slots[0];
  for (size_t i = 0; i < n; ++i) xp[i] = fluid.position[i] + dt * vp[i];
  set_source_term_vp();
  resolve_pressure_globally(false, 0, sp.target_density_error, true);
  add_pressure_acceleration(nullptr, false, true, true);
  // The velocity Jacobian of :155-183 is computed by the reference but never
  // used; only the DFSPH-style update below reaches the state.
  for (size_t i = 0; i < n; ++i) {
    V3 new_pos = xp[i] + powi2(dt) * fluid.acceleration[i];
    iisph.pressure_acc_f[i] = vp[i] + dt * fluid.acceleration[i];
    xp[i] = new_pos;
  }
  for (size_t i = 0; i < n; ++i) vp[i] = iisph.pressure_acc_f[i];
  std::swap(fluid.integrator_position_slots[0], fluid.solver_position_slots[0]);
  std::swap(fluid.integrator_velocity_slots[0], fluid.solver_velocity_slots[0]);
}


// ---------------------------------------------------------------------------
// Surface reconstruction (fluid.rs:212-347; splashsurf_lib 0.14.1 restated)
// ---------------------------------------------------------------------------
namespace {

constexpr double kIsoSurfaceThreshold = 0.6;  // fluid.rs:265

// Cube corners c = bx + 2 by + 4 bz; local edge e = 4 * dir + rank of its
// lower corner among the corners whose bit `dir` is 0.
int corner_bit(int c, int d) { return (c >> d) & 1; }
int edge_of(int a, int b) {
  const int x = a ^ b;
  const int d = x == 1 ? 0 : (x == 2 ? 1 : 2);
  const int lo = a < b ? a : b;
  int rank = 0;
  for (int c = 0; c < lo; ++c)
    if (!corner_bit(c, d)) ++rank;
  return 4 * d + rank;
}
int edge_lower_corner(int e) {
  const int d = e / 4;
  int rank = e % 4;
  for (int c = 0; c < 8; ++c)
    if (!corner_bit(c, d) && rank-- == 0) return c;
  return -1;
}

// The six faces as corner cycles, counter-clockwise seen from outside.
struct FaceCycles {
  int c[6][4];
  FaceCycles() {
    int f = 0;
    for (int a = 0; a < 3; ++a)
      for (int s = 0; s < 2; ++s, ++f) {
        const int u = (a + 1) % 3, v = (a + 2) % 3;
        const int uv[4][2] = {{0, 0}, {1, 0}, {1, 1}, {0, 1}};
        int cyc[4];
        for (int k = 0; k < 4; ++k) cyc[k] = (s << a) | (uv[k][0] << u) | (uv[k][1] << v);
        // (p1 - p0) x (p2 - p1) is +e_a for this u, v order; outward is (2s - 1) e_a
        const bool ccw = s == 1;
        for (int k = 0; k < 4; ++k) c[f][k] = ccw ? cyc[k] : cyc[3 - k];
      }
  }
};
const FaceCycles kFaces;

// Polygons of one cell (lists of local edges) for the corners' inside flags:
// on every face each run of inside corners gives a segment from the edge
// where the cycle enters the run to the edge where it leaves it (so a face
// with two diagonal inside corners keeps them apart), and the segments chain
// into closed loops through the edges they share.
std::vector<std::vector<int>> cell_polygons(const bool inside[8]) {
  int next[12];
  bool has[12] = {false};
  for (int f = 0; f < 6; ++f) {
    int cross[4], type[4], nc = 0;  // type 1 entering, 0 leaving
    for (int k = 0; k < 4; ++k) {
      const int a = kFaces.c[f][k], b = kFaces.c[f][(k + 1) % 4];
      if (inside[a] != inside[b]) {
        cross[nc] = edge_of(a, b);
        type[nc] = inside[b] ? 1 : 0;
        ++nc;
      }
    }
    for (int k = 0; k < nc; ++k)
      if (type[k] == 1) {
        const int x = cross[(k + 1) % nc];
        next[cross[k]] = x;
        has[cross[k]] = true;
      }
  }
  std::vector<std::vector<int>> loops;
  bool used[12] = {false};
  for (int e = 0; e < 12; ++e) {
    if (!has[e] || used[e]) continue;
    std::vector<int> loop;
    int cur = e;
    while (!used[cur]) {
      used[cur] = true;
      loop.push_back(cur);
      cur = next[cur];
    }
    loops.push_back(loop);
  }
  return loops;
}

}  // namespace

SurfaceGrid surface_grid(const std::vector<V3>& positions, double h, double cube) {
  SurfaceGrid g;
  g.cube = cube;
  V3 lo{std::numeric_limits<double>::infinity(), std::numeric_limits<double>::infinity(),
        std::numeric_limits<double>::infinity()};
  V3 hi{-lo.x, -lo.y, -lo.z};
  for (const V3& p : positions) {
    lo = V3{std::min(lo.x, p.x), std::min(lo.y, p.y), std::min(lo.z, p.z)};
    hi = V3{std::max(hi.x, p.x), std::max(hi.y, p.y), std::max(hi.z, p.z)};
  }
  const double l[3] = {lo.x, lo.y, lo.z}, u[3] = {hi.x, hi.y, hi.z};
  for (int d = 0; d < 3; ++d) {
    const int64_t a = (int64_t)std::floor((l[d] - h) / cube) - 1;
    const int64_t b = (int64_t)std::floor((u[d] + h) / cube) + 1;
    g.k0[d] = a;
    g.n[d] = b - a + 1;
  }
  return g;
}

std::vector<SurfaceMesh> reconstruct_surfaces(const Fluid& fluid, double spacing, double rest_volume, double h) {
  std::vector<SurfaceMesh> out;
  // groups by fluid id in ascending order, each with its first particle's mass
  std::vector<uint32_t> ids;
  for (size_t i = 0; i < fluid.len(); ++i) ids.push_back(fluid.fluid_id[i]);
  std::sort(ids.begin(), ids.end());
  ids.erase(std::unique(ids.begin(), ids.end()), ids.end());
  const double r = 0.5 * spacing, cube = 0.75 * r;
  for (uint32_t id : ids) {
    std::vector<V3> pos;
    double mass0 = 0.0;
    for (size_t i = 0; i < fluid.len(); ++i)
      if (fluid.fluid_id[i] == id) {
        if (pos.empty()) mass0 = fluid.mass[i];
        pos.push_back(fluid.position[i]);
      }
    const double rest_density = mass0 / rest_volume;
    const double m = rest_density * (4.0 / 3.0 * PI * (r * r * r));
    // particle densities
    SpatialHashing ns(h);
    NeighborList nl;
    ns.find_samples(h, pos, pos, nl);
    std::vector<double> vol(pos.size());
    for (size_t i = 0; i < pos.size(); ++i) {
      double rho = 0.0;
      for (const size_t* it = nl.begin(i); it != nl.end(i); ++it) rho += m * kernel_function(pos[i] - pos[*it], h);
      vol[i] = m / rho;
    }
    // level set on the grid points
    const SurfaceGrid g = surface_grid(pos, h, cube);
    const int64_t nx = g.n[0], ny = g.n[1], nz = g.n[2];
    std::vector<V3> pts((size_t)(nx * ny * nz));
    for (int64_t k = 0; k < nz; ++k)
      for (int64_t j = 0; j < ny; ++j)
        for (int64_t i = 0; i < nx; ++i)
          pts[(size_t)(i + nx * (j + ny * k))] = V3{g.coord(0, i), g.coord(1, j), g.coord(2, k)};
    NeighborList gl;
    SpatialHashing gs(h);
    gs.find_samples(h, pts, pos, gl);
    std::vector<double> phi(pts.size());
    for (size_t q = 0; q < pts.size(); ++q) {
      double s = 0.0;
      for (const size_t* it = gl.begin(q); it != gl.end(q); ++it) s += vol[*it] * kernel_function(pts[q] - pos[*it], h);
      phi[q] = s;
    }
    auto inside = [&](size_t q) { return phi[q] > kIsoSurfaceThreshold; };
    // vertices: crossing lattice edges, in order of (point, direction)
    SurfaceMesh mesh;
    mesh.fluid_id = id;
    std::unordered_map<uint64_t, uint32_t> vid;
    const int64_t step[3] = {1, nx, nx * ny};
    for (int64_t k = 0; k < nz; ++k)
      for (int64_t j = 0; j < ny; ++j)
        for (int64_t i = 0; i < nx; ++i) {
          const int64_t q = i + nx * (j + ny * k);
          const int64_t idx[3] = {i, j, k};
          for (int d = 0; d < 3; ++d) {
            if (idx[d] + 1 >= g.n[d]) continue;
            const int64_t q2 = q + step[d];
            if (inside((size_t)q) == inside((size_t)q2)) continue;
            const double t = (kIsoSurfaceThreshold - phi[(size_t)q]) / (phi[(size_t)q2] - phi[(size_t)q]);
            V3 a = pts[(size_t)q], b = pts[(size_t)q2];
            vid[(uint64_t)q * 3 + (uint64_t)d] = (uint32_t)mesh.position.size();
            mesh.position.push_back(a + t * (b - a));
          }
        }
    // triangles: cells in order, each cell's polygons fanned from their first vertex
    for (int64_t k = 0; k + 1 < nz; ++k)
      for (int64_t j = 0; j + 1 < ny; ++j)
        for (int64_t i = 0; i + 1 < nx; ++i) {
          bool in[8];
          int64_t corner_q[8];
          int cnt = 0;
          for (int c = 0; c < 8; ++c) {
            corner_q[c] = (i + corner_bit(c, 0)) + nx * ((j + corner_bit(c, 1)) + ny * (k + corner_bit(c, 2)));
            in[c] = inside((size_t)corner_q[c]);
            cnt += in[c];
          }
          if (cnt == 0 || cnt == 8) continue;
          for (const auto& loop : cell_polygons(in)) {
            std::vector<uint32_t> v;
            for (int e : loop) {
              const int lo = edge_lower_corner(e);
              v.push_back(vid.at((uint64_t)corner_q[lo] * 3 + (uint64_t)(e / 4)));
            }
            for (size_t t = 1; t + 1 < v.size(); ++t) {
              mesh.indices.push_back(v[0]);
              mesh.indices.push_back(v[t]);
              mesh.indices.push_back(v[t + 1]);
            }
          }
        }
    if (mesh.indices.empty()) continue;
    // fluid.rs:296-323: area-weighted vertex normals
    mesh.normal.assign(mesh.position.size(), V3{0, 0, 0});
    for (size_t t = 0; t < mesh.indices.size(); t += 3) {
      const V3 v0 = mesh.position[mesh.indices[t]], v1 = mesh.position[mesh.indices[t + 1]],
               v2 = mesh.position[mesh.indices[t + 2]];
      const V3 fn = cross(v1 - v0, v2 - v0);
      for (int c = 0; c < 3; ++c) mesh.normal[mesh.indices[t + c]] += fn;
    }
    for (V3& n : mesh.normal) {
      const double len = std::sqrt(n.x * n.x + n.y * n.y + n.z * n.z);
      if (len > 1e-10) n = V3{n.x / len, n.y / len, n.z / len};
    }
    out.push_back(std::move(mesh));
  }
  return out;
}

}  // namespace oracle
