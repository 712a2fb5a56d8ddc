// C entry points of the SPH oracle for the test harness (ctypes).
// TEST INFRASTRUCTURE ONLY: loaded by tests/, smoke() and bench.py's CPU
// baseline leg; never by the engine.
#include <cstring>
#include <stdexcept>

#include "sph_oracle.hpp"

using namespace oracle;

extern "C" {

// Same field meaning as `sph_config` of the engine's C ABI; kept separate so
// the oracle has no dependency on the product.
typedef struct oracle_config {
  int integration_scheme;  // 0 EulerCromer, 1 TakePredicted
  int pressure_solver;     // 0 SESPH, 1 SESPHwSplitting, 2 IISPH, 3 IISPHwOST
  int boundary_handling;   // 0 StaticSampleBoundary, 1 VolumeMapBoundary
  int cfl_time_step;
  double rest_density_grid_spacing, kernel_support_radius, disable_particles_below;
  double fluid_viscosity, boundary_viscosity;
  double boundary_pressure_acceleration_weighting, boundary_rest_volume_weighting;
  double stiffness, target_density_error, relaxation_factor, min_diagonal_element;
  double time_increment, max_time_increment, cfl_number;
  int gravity_mode;
  double gravity_center[3];
  unsigned max_solver_iterations;  // 0 = unbounded (reference semantics)
  unsigned contact_fixed_sweeps;   // 0 = the reference's merit test
} oracle_config;

struct OracleHandle {
  System sys;
  double rest_volume_weighting = 1.0;
};

static void read_rigid(const double* r, RigidBodyMotion& out) {
  // layout: mass, inertia_body[9] (row-major), inertia_inv_body[9], com[3],
  //         quat (w,i,j,k)[4], lin_vel[3], ang_vel[3]  -> 32 doubles
  M3 ib, iib;
  for (int i = 0; i < 9; ++i) { ib.m[i / 3][i % 3] = r[1 + i]; iib.m[i / 3][i % 3] = r[10 + i]; }
  V3 com{r[19], r[20], r[21]};
  Quat q{r[22], r[23], r[24], r[25]};
  V3 lv{r[26], r[27], r[28]}, av{r[29], r[30], r[31]};
  out = RigidBodyMotion(r[0], ib, iib, com, q, lv, av);
}

void* oracle_system_create(const oracle_config* c) {
  auto* h = new OracleHandle();
  System& s = h->sys;
  s.integrator = (Integrator)c->integration_scheme;
  s.solver = (Solver)c->pressure_solver;
  if (c->boundary_handling == 0) {
    s.boundary = std::make_unique<StaticSampleBoundary>();
  } else {
    auto vmb = std::make_unique<VolumeMapBoundary>();
    vmb->contact_fixed_sweeps = c->contact_fixed_sweeps;
    s.boundary = std::move(vmb);
  }
  SystemParameters& p = s.params;
  p.cfl = c->cfl_time_step != 0;
  p.time_increment = p.cfl ? 0.0 : c->time_increment;
  p.max_time_increment = c->max_time_increment;
  p.cfl_number = c->cfl_number;
  p.kernel_support_radius = c->kernel_support_radius;
  p.disable_particles_below = c->disable_particles_below;
  p.rest_density_grid_spacing = c->rest_density_grid_spacing;
  p.rest_volume = c->rest_density_grid_spacing * c->rest_density_grid_spacing *
                  c->rest_density_grid_spacing;
  p.fluid_viscosity = c->fluid_viscosity;
  p.boundary_viscosity = c->boundary_viscosity;
  p.boundary_pressure_acceleration_weighting = c->boundary_pressure_acceleration_weighting;
  p.gravity = c->gravity_mode == 1 ? Gravity::Radial : Gravity::Uniform;
  p.gravity_center = {c->gravity_center[0], c->gravity_center[1], c->gravity_center[2]};
  s.sp.stiffness = c->stiffness;
  s.sp.target_density_error = c->target_density_error;
  s.sp.relaxation_factor = c->relaxation_factor;
  s.sp.min_diagonal_element = c->min_diagonal_element;
  s.sp.iteration_cap = c->max_solver_iterations ? c->max_solver_iterations : 0xffffffffu;
  h->rest_volume_weighting = c->boundary_rest_volume_weighting;
  return h;
}

void oracle_destroy(void* h) { delete (OracleHandle*)h; }
void* oracle_clone(void* h) { return new OracleHandle(*(OracleHandle*)h); }

int oracle_upload_fluid(void* hh, size_t n, const double* pos, const double* vel,
                        const double* mass, const unsigned* fid) {
  Fluid& f = ((OracleHandle*)hh)->sys.fluid;
  f = Fluid();
  f.num_active = n;
  f.position.resize(n); f.velocity.resize(n); f.acceleration.assign(n, V3{});
  f.mass.resize(n); f.volume.assign(n, 0.); f.pressure.assign(n, 0.);
  f.fluid_id.resize(n); f.origin.resize(n);
  for (size_t i = 0; i < n; ++i) {
    f.position[i] = {pos[3 * i], pos[3 * i + 1], pos[3 * i + 2]};
    f.velocity[i] = vel ? V3{vel[3 * i], vel[3 * i + 1], vel[3 * i + 2]} : V3{};
    f.mass[i] = mass[i];
    f.fluid_id[i] = fid ? fid[i] : 0u;
    f.origin[i] = (uint32_t)i;
  }
  return 0;
}

int oracle_add_sample_boundary(void* hh, size_t nb, const double* pos, const double* rigid) {
  auto* sb = dynamic_cast<StaticSampleBoundary*>(((OracleHandle*)hh)->sys.boundary.get());
  if (!sb) return 1;
  SampleBoundary b;
  b.dynamic = rigid != nullptr;
  std::vector<V3> p(nb);
  for (size_t i = 0; i < nb; ++i) p[i] = {pos[3 * i], pos[3 * i + 1], pos[3 * i + 2]};
  if (b.dynamic) {
    b.xb_body = p;
    b.xb.assign(nb, V3{});
    read_rigid(rigid, b.state);
  } else {
    b.xb = p;
  }
  b.vb.assign(nb, V3{});
  b.vol.assign(nb, 0.);
  sb->boundaries.push_back(std::move(b));
  return 0;
}

static void read_field(const double* desc, const long long* n, const double* nodes,
                       Serendipity& s) {
  s.x_min = {desc[0], desc[1], desc[2]};
  s.x_max = {desc[3], desc[4], desc[5]};
  s.dx = desc[6];
  for (int d = 0; d < 3; ++d) s.n[d] = n[d];
  size_t cnt = (size_t)(s.NX() * s.NY() * s.NZ());
  s.nodes.assign(nodes, nodes + cnt);
}

int oracle_add_volume_map_boundary(void* hh, const double* sdf_desc, const long long* sdf_n,
                                   const double* sdf_nodes, const double* vm_desc,
                                   const long long* vm_n, const double* vm_nodes,
                                   const double* rigid) {
  auto* vb = dynamic_cast<VolumeMapBoundary*>(((OracleHandle*)hh)->sys.boundary.get());
  if (!vb) return 1;
  VMBoundary b;
  read_field(sdf_desc, sdf_n, sdf_nodes, b.sdf);
  read_field(vm_desc, vm_n, vm_nodes, b.vm);
  b.dynamic = rigid != nullptr;
  if (b.dynamic) read_rigid(rigid, b.state);
  vb->boundaries.push_back(std::move(b));
  return 0;
}

// Mesh bounding box (body frame) of volume-map boundary `bi`, which makes it
// take part in rigid-rigid contact.
int oracle_set_vm_aabb(void* hh, size_t bi, const double* center, const double* half) {
  auto* vb = dynamic_cast<VolumeMapBoundary*>(((OracleHandle*)hh)->sys.boundary.get());
  if (!vb || bi >= vb->boundaries.size()) return 1;
  VMBoundary& b = vb->boundaries[bi];
  b.has_aabb = true;
  b.aabb_center = V3{center[0], center[1], center[2]};
  b.aabb_half = V3{half[0], half[1], half[2]};
  return 0;
}

// One contact solve on the current state without applying it: per-boundary
// force and torque (3 doubles each), the number of contact cells and sweeps.
int oracle_contact_probe(void* hh, double dt, double* force, double* torque, size_t* cells,
                         unsigned* iterations) {
  auto* vb = dynamic_cast<VolumeMapBoundary*>(((OracleHandle*)hh)->sys.boundary.get());
  if (!vb) return 1;
  ContactResult r = vb->solve_contacts(dt, false);
  for (size_t b = 0; b < r.force.size(); ++b) {
    force[3 * b] = r.force[b].x; force[3 * b + 1] = r.force[b].y; force[3 * b + 2] = r.force[b].z;
    torque[3 * b] = r.torque[b].x; torque[3 * b + 1] = r.torque[b].y; torque[3 * b + 2] = r.torque[b].z;
  }
  *cells = r.cells;
  *iterations = r.iterations;
  return 0;
}

// A System around given fluid arrays for the solver-level probes below (the
// shape of the reference's solver unit tests): fluid neighbors from the
// spatial hashing, or none (with_nl = 0); the nb boundary samples
// (positions, volumes) form one sample boundary, dynamic (unit mass and
// inertia) with its center of mass at body_com when that is given.
static void probe_system(System& s, double h, double spacing, size_t n, const double* pos, const double* vel,
                         const double* mass, const double* vol, const double* acc, int with_nl, size_t nb,
                         const double* bpos, const double* bvol, const double* body_com) {
  SystemParameters& P = s.params;
  P.kernel_support_radius = h;
  P.rest_density_grid_spacing = spacing;
  P.rest_volume = spacing * spacing * spacing;
  auto sb = std::make_unique<StaticSampleBoundary>();
  sb->cell_size = h;
  if (nb) {
    SampleBoundary b;
    for (size_t k = 0; k < nb; ++k) {
      b.xb.push_back(V3{bpos[3 * k], bpos[3 * k + 1], bpos[3 * k + 2]});
      b.vb.push_back(V3{0, 0, 0});
      b.vol.push_back(bvol[k]);
    }
    b.dynamic = body_com != nullptr;
    if (b.dynamic) {
      M3 eye;
      eye.m[0][0] = eye.m[1][1] = eye.m[2][2] = 1.0;
      b.state = RigidBodyMotion(1.0, eye, eye, V3{body_com[0], body_com[1], body_com[2]}, Quat{}, V3{}, V3{});
    }
    sb->boundaries.push_back(std::move(b));
  }
  s.boundary = std::move(sb);
  Fluid& f = s.fluid;
  f.num_active = n;
  f.fluid_id.assign(n, 0);
  f.origin.assign(n, 0);
  f.position.resize(n);
  f.velocity.resize(n);
  f.acceleration.resize(n);
  f.mass.assign(mass, mass + n);
  f.volume.assign(vol, vol + n);
  f.pressure.assign(n, 0.0);
  for (size_t i = 0; i < n; ++i) {
    f.position[i] = V3{pos[3 * i], pos[3 * i + 1], pos[3 * i + 2]};
    f.velocity[i] = vel ? V3{vel[3 * i], vel[3 * i + 1], vel[3 * i + 2]} : V3{0, 0, 0};
    f.acceleration[i] = V3{acc[3 * i], acc[3 * i + 1], acc[3 * i + 2]};
  }
  f.resize_slots(0, 0, 0, 0);
  if (with_nl) {
    s.ns = SpatialHashing(h);
    s.ns.find_samples(h, f.position, f.position, s.fluid_nl);
  } else {
    s.fluid_nl.indices.clear();
    s.fluid_nl.offsets.assign(n + 1, 0);
  }
  s.boundary->find_boundary_samples(h, f.position, spacing);
}

static void probe_outputs(System& s, size_t nb, const double* body_com, double* acc_out, double* body_ft) {
  const Fluid& f = s.fluid;
  for (size_t i = 0; i < f.len(); ++i) {
    acc_out[3 * i] = f.acceleration[i].x;
    acc_out[3 * i + 1] = f.acceleration[i].y;
    acc_out[3 * i + 2] = f.acceleration[i].z;
  }
  for (int k = 0; k < 6; ++k) body_ft[k] = 0.0;
  if (nb && body_com) {
    const RigidBodyMotion& m = static_cast<StaticSampleBoundary&>(*s.boundary).boundaries[0].state;
    const V3 v[2] = {m.force, m.torque};
    for (int k = 0; k < 2; ++k) {
      body_ft[3 * k] = v[k].x;
      body_ft[3 * k + 1] = v[k].y;
      body_ft[3 * k + 2] = v[k].z;
    }
  }
}

// SESPH::solve_and_add_acceleration (sesph.rs:31-67) on given fluid volumes
// (tests/sph/pressure_solver/sesph.rs:309-633). prm = {h, spacing,
// stiffness, boundary pressure weighting}.
int oracle_sesph_probe(const double* prm, size_t n, const double* pos, const double* mass, const double* vol,
                       const double* acc, int with_fluid_neighbors, size_t nb, const double* bpos,
                       const double* bvol, const double* body_com, double* p_out, double* acc_out,
                       double* body_force_torque) {
  System s;
  s.solver = Solver::SESPH;
  probe_system(s, prm[0], prm[1], n, pos, nullptr, mass, vol, acc, with_fluid_neighbors, nb, bpos, bvol, body_com);
  s.sp.stiffness = prm[2];
  s.params.boundary_pressure_acceleration_weighting = prm[3];
  s.sesph();
  for (size_t i = 0; i < n; ++i) p_out[i] = s.fluid.pressure[i];
  probe_outputs(s, nb, body_com, acc_out, body_force_torque);
  return 0;
}

// add_gravity_acceleration and add_viscosity_acceleration
// (non_pressure_accelerations.rs:64-185) on given fluid arrays
// (non_pressure_accelerations.rs:473-964 tests). prm = {h, spacing, fluid
// viscosity, boundary viscosity, gravity mode (0 uniform, 1 radial), center
// x, y, z}; which: bit 0 gravity, bit 1 viscosity.
int oracle_nonpressure_probe(const double* prm, int which, size_t n, const double* pos, const double* vel,
                             const double* mass, const double* vol, const double* acc, int with_fluid_neighbors,
                             size_t nb, const double* bpos, const double* bvol, const double* body_com,
                             double* acc_out, double* body_force_torque) {
  System s;
  probe_system(s, prm[0], prm[1], n, pos, vel, mass, vol, acc, with_fluid_neighbors, nb, bpos, bvol, body_com);
  s.params.fluid_viscosity = prm[2];
  s.params.boundary_viscosity = prm[3];
  s.params.gravity = prm[4] != 0.0 ? Gravity::Radial : Gravity::Uniform;
  s.params.gravity_center = V3{prm[5], prm[6], prm[7]};
  if (which & 1) s.add_gravity_acceleration();
  if (which & 2) s.add_viscosity_acceleration();
  probe_outputs(s, nb, body_com, acc_out, body_force_torque);
  return 0;
}

// SESPHwSplitting::solve_and_add_acceleration (sesph_with_splitting.rs:
// 33-152) on given fluid arrays (sesph_with_splitting.rs:428-660 tests).
// prm = {h, spacing, dt, stiffness, boundary pressure weighting}. Writes the
// predicted densities, pressures, accelerations and the body's force and
// torque.
int oracle_splitting_probe(const double* prm, size_t n, const double* pos, const double* vel, const double* mass,
                           const double* vol, const double* acc, int with_fluid_neighbors, size_t nb,
                           const double* bpos, const double* bvol, const double* body_com, double* rho_out,
                           double* p_out, double* acc_out, double* body_force_torque) {
  System s;
  s.solver = Solver::SESPHwSplitting;
  probe_system(s, prm[0], prm[1], n, pos, vel, mass, vol, acc, with_fluid_neighbors, nb, bpos, bvol, body_com);
  s.params.time_increment = prm[2];
  s.sp.stiffness = prm[3];
  s.params.boundary_pressure_acceleration_weighting = prm[4];
  s.fluid.resize_slots(0, 0, 0, 1);
  s.sesph_w_splitting();
  for (size_t i = 0; i < n; ++i) {
    rho_out[i] = s.density_pred[i];
    p_out[i] = s.fluid.pressure[i];
  }
  probe_outputs(s, nb, body_com, acc_out, body_force_torque);
  return 0;
}

// IISPH's source terms and diagonal element (iisph.rs:117-342) on given
// fluid arrays, vel being the solver's predicted velocities
// (iisph.rs:714-1017 tests). prm = {h, spacing, dt, boundary pressure
// weighting}; which: 1 set_source_term_vde, 2 set_source_term_vp, 4
// set_diagonal_element.
int oracle_iisph_terms_probe(const double* prm, int which, size_t n, const double* pos, const double* vel,
                             const double* mass, const double* vol, int with_fluid_neighbors, size_t nb,
                             const double* bpos, const double* bvol, double* s_out, double* a_out) {
  System s;
  std::vector<double> acc(3 * n, 0.0);
  probe_system(s, prm[0], prm[1], n, pos, nullptr, mass, vol, acc.data(), with_fluid_neighbors, nb, bpos, bvol,
               nullptr);
  s.params.time_increment = prm[2];
  s.params.boundary_pressure_acceleration_weighting = prm[3];
  s.fluid.resize_slots(0, 0, 1, 1);
  for (size_t i = 0; i < n; ++i) s.fluid.solver_velocity_slots[0][i] = V3{vel[3 * i], vel[3 * i + 1], vel[3 * i + 2]};
  s.iisph.s_f.assign(n, 0.0);
  s.iisph.a_ff.assign(n, 0.0);
  if (which & 1) s.set_source_term_vde();
  if (which & 2) s.set_source_term_vp();
  if (which & 4) s.set_diagonal_element();
  for (size_t i = 0; i < n; ++i) {
    s_out[i] = s.iisph.s_f[i];
    a_out[i] = s.iisph.a_ff[i];
  }
  return 0;
}

// IISPH::initialize (iisph.rs:344-376) on given source terms and diagonals.
int oracle_iisph_initialize_probe(size_t n, const double* s_f, const double* a_ff, double omega, double eps,
                                  int clamp, double* p_out) {
  System s;
  s.fluid.num_active = n;
  s.fluid.pressure.assign(n, 0.0);
  s.iisph.s_f.assign(s_f, s_f + n);
  s.iisph.a_ff.assign(a_ff, a_ff + n);
  s.sp.relaxation_factor = omega;
  s.sp.min_diagonal_element = eps;
  s.iisph_initialize(clamp != 0);
  for (size_t i = 0; i < n; ++i) p_out[i] = s.fluid.pressure[i];
  return 0;
}

// Fluid::reconstruct_surfaces (fluid.rs:212-347) on n particles given as
// positions (3n), fluid ids and masses; returns an owned mesh list.
void* oracle_surfaces_from(size_t n, const double* pos, const uint32_t* ids, const double* mass, double spacing,
                           double rest_volume, double h) {
  Fluid f;
  f.num_active = n;
  f.position.resize(n);
  for (size_t i = 0; i < n; ++i) f.position[i] = V3{pos[3 * i], pos[3 * i + 1], pos[3 * i + 2]};
  f.fluid_id.assign(ids, ids + n);
  f.mass.assign(mass, mass + n);
  return new std::vector<SurfaceMesh>(reconstruct_surfaces(f, spacing, rest_volume, h));
}
// The same on an oracle system's current fluid.
void* oracle_surfaces(void* hh) {
  System& s = ((OracleHandle*)hh)->sys;
  return new std::vector<SurfaceMesh>(reconstruct_surfaces(s.fluid, s.params.rest_density_grid_spacing,
                                                           s.params.rest_volume, s.params.kernel_support_radius));
}
size_t oracle_surfaces_count(void* m) { return ((std::vector<SurfaceMesh>*)m)->size(); }
void oracle_surface_sizes(void* m, size_t k, uint32_t* id, size_t* nv, size_t* ni) {
  const SurfaceMesh& s = (*(std::vector<SurfaceMesh>*)m)[k];
  *id = s.fluid_id;
  *nv = s.position.size();
  *ni = s.indices.size();
}
void oracle_surface_copy(void* m, size_t k, double* pos, double* nrm, uint32_t* idx) {
  const SurfaceMesh& s = (*(std::vector<SurfaceMesh>*)m)[k];
  for (size_t v = 0; v < s.position.size(); ++v) {
    pos[3 * v] = s.position[v].x; pos[3 * v + 1] = s.position[v].y; pos[3 * v + 2] = s.position[v].z;
    nrm[3 * v] = s.normal[v].x; nrm[3 * v + 1] = s.normal[v].y; nrm[3 * v + 2] = s.normal[v].z;
  }
  for (size_t t = 0; t < s.indices.size(); ++t) idx[t] = s.indices[t];
}
void oracle_surfaces_free(void* m) { delete (std::vector<SurfaceMesh>*)m; }
// The marching-cubes lattice of a point set: k0[3], n[3], cube.
void oracle_surface_grid(size_t n, const double* pos, double h, double cube, long long* k0, long long* np) {
  std::vector<V3> p(n);
  for (size_t i = 0; i < n; ++i) p[i] = V3{pos[3 * i], pos[3 * i + 1], pos[3 * i + 2]};
  SurfaceGrid g = surface_grid(p, h, cube);
  for (int d = 0; d < 3; ++d) {
    k0[d] = g.k0[d];
    np[d] = g.n[d];
  }
}

// Fluid bookkeeping (fluid.rs:113-128, 159-204) driven the way its unit
// tests drive it: n particles (positions, masses, fluid ids; the rest zero),
// resize_slots(slots[0..4]) when `slots` is given, disable(id) for each of
// `ids` in order, drop_inactive when `drop`. Writes the first total_len
// positions, masses and ids, the active and total lengths, and the four slot
// pool counts and their length. Returns 1 where the reference's
// `id < num_active` assertion fails (at the failing disable).
int oracle_fluid_probe(size_t n, const double* pos, const double* mass, const uint32_t* fid,
                       const long long* slots, size_t nd, const long long* ids, int drop,
                       double* out_pos, double* out_mass, uint32_t* out_fid, size_t* out_len) {
  Fluid f;
  f.position.resize(n);
  for (size_t i = 0; i < n; ++i) f.position[i] = {pos[3 * i], pos[3 * i + 1], pos[3 * i + 2]};
  f.velocity.assign(n, V3{});
  f.acceleration.assign(n, V3{});
  f.mass.assign(mass, mass + n);
  f.volume.assign(n, 0.0);
  f.pressure.assign(n, 0.0);
  f.fluid_id.assign(fid, fid + n);
  f.origin.resize(n);
  for (size_t i = 0; i < n; ++i) f.origin[i] = (uint32_t)i;
  f.num_active = n;
  if (slots) f.resize_slots((size_t)slots[0], (size_t)slots[1], (size_t)slots[2], (size_t)slots[3]);
  for (size_t k = 0; k < nd; ++k) {
    if (ids[k] < 0) return 1;
    try {
      f.disable((size_t)ids[k]);
    } catch (const std::out_of_range&) {
      return 1;
    }
  }
  if (drop) f.drop_inactive();
  const size_t total = f.position.size();
  for (size_t i = 0; i < total; ++i) {
    out_pos[3 * i] = f.position[i].x; out_pos[3 * i + 1] = f.position[i].y;
    out_pos[3 * i + 2] = f.position[i].z;
    out_mass[i] = f.mass[i];
    out_fid[i] = f.fluid_id[i];
  }
  out_len[0] = f.len();
  out_len[1] = total;
  out_len[2] = f.integrator_position_slots.size();
  out_len[3] = f.integrator_velocity_slots.size();
  out_len[4] = f.solver_position_slots.size();
  out_len[5] = f.solver_velocity_slots.size();
  size_t slot_len = 0;
  for (auto* pool : {&f.integrator_position_slots, &f.integrator_velocity_slots,
                     &f.solver_position_slots, &f.solver_velocity_slots})
    for (auto& sl : *pool) slot_len = std::max(slot_len, sl.size());
  out_len[6] = slot_len;
  return 0;
}

// A StaticSampleBoundary driven on its own, the way the reference's unit
// tests drive it (static_sample_boundary.rs:142-168, 354-412, 544-552):
// boundaries of given samples (body frame for a dynamic one, world frame for
// a static one), initialize, find_boundary_samples, add_force_onto_boundary
// and step_forward_in_time, with the samples, volumes, neighbors and rigid
// state read back.
void* oracle_ssb_create() { return new StaticSampleBoundary(); }
void oracle_ssb_free(void* b) { delete (StaticSampleBoundary*)b; }
size_t oracle_ssb_count(void* b) { return ((StaticSampleBoundary*)b)->count(); }
size_t oracle_ssb_len(void* b, size_t bi) { return ((StaticSampleBoundary*)b)->boundaries[bi].xb.size(); }
int oracle_ssb_add(void* b, size_t nb, const double* pos, const double* rigid) {
  auto* sb = (StaticSampleBoundary*)b;
  SampleBoundary sbb;
  sbb.dynamic = rigid != nullptr;
  std::vector<V3> p(nb);
  for (size_t i = 0; i < nb; ++i) p[i] = {pos[3 * i], pos[3 * i + 1], pos[3 * i + 2]};
  if (sbb.dynamic) {
    sbb.xb_body = p;
    sbb.xb.assign(nb, V3{});
    read_rigid(rigid, sbb.state);
  } else {
    sbb.xb = p;
  }
  sbb.vb.assign(nb, V3{});
  sbb.vol.assign(nb, 0.);
  sb->boundaries.push_back(std::move(sbb));
  return 0;
}
void oracle_ssb_initialize(void* b, double h, double gamma) {
  ((StaticSampleBoundary*)b)->initialize(h, gamma);
}
void oracle_ssb_find(void* b, double range, size_t n, const double* pos, double spacing) {
  std::vector<V3> p(n);
  for (size_t i = 0; i < n; ++i) p[i] = {pos[3 * i], pos[3 * i + 1], pos[3 * i + 2]};
  ((StaticSampleBoundary*)b)->find_boundary_samples(range, p, spacing);
}
size_t oracle_ssb_neighbor_count(void* b, size_t bi, size_t id) {
  return ((StaticSampleBoundary*)b)->boundaries[bi].nl.count(id);
}
void oracle_ssb_add_force(void* b, size_t id, const double* f, const double* loc) {
  ((StaticSampleBoundary*)b)->add_force_onto_boundary(id, {f[0], f[1], f[2]},
                                                      {loc[0], loc[1], loc[2]});
}
void oracle_ssb_step(void* b, double dt) { ((StaticSampleBoundary*)b)->step_forward_in_time(dt); }
// positions, velocities (3 per sample) and volumes of boundary bi; returns
// whether it is dynamic and, if so, writes its center of mass.
int oracle_ssb_samples(void* b, size_t bi, double* pos, double* vel, double* vol, double* com) {
  const SampleBoundary& s = ((StaticSampleBoundary*)b)->boundaries[bi];
  for (size_t i = 0; i < s.xb.size(); ++i) {
    pos[3 * i] = s.xb[i].x; pos[3 * i + 1] = s.xb[i].y; pos[3 * i + 2] = s.xb[i].z;
    vel[3 * i] = s.vb[i].x; vel[3 * i + 1] = s.vb[i].y; vel[3 * i + 2] = s.vb[i].z;
    vol[i] = s.vol[i];
  }
  if (!s.dynamic) return 0;
  com[0] = s.state.center_of_mass.x; com[1] = s.state.center_of_mass.y;
  com[2] = s.state.center_of_mass.z;
  return 1;
}

// IntegrationScheme::integrate on given particle arrays, in place (3n
// doubles each): scheme 0 EulerCromer (slot pointers unused, may be null),
// 1 TakePredicted (one position and one velocity slot).
int oracle_integrate_probe(int scheme, size_t n, double* pos, double* vel, double* acc,
                           double* slot_pos, double* slot_vel, double dt) {
  if (scheme != 0 && scheme != 1) return 1;
  if (scheme == 1 && (!slot_pos || !slot_vel)) return 2;
  Fluid f;
  auto load = [n](const double* a) {
    std::vector<V3> v(n);
    for (size_t i = 0; i < n; ++i) v[i] = {a[3 * i], a[3 * i + 1], a[3 * i + 2]};
    return v;
  };
  auto store = [n](const std::vector<V3>& v, double* a) {
    for (size_t i = 0; i < n; ++i) { a[3 * i] = v[i].x; a[3 * i + 1] = v[i].y; a[3 * i + 2] = v[i].z; }
  };
  f.position = load(pos);
  f.velocity = load(vel);
  f.acceleration = load(acc);
  if (scheme == 1) {
    f.integrator_position_slots.push_back(load(slot_pos));
    f.integrator_velocity_slots.push_back(load(slot_vel));
  }
  f.num_active = n;
  integrate((Integrator)scheme, f, n, dt);
  store(f.position, pos);
  store(f.velocity, vel);
  store(f.acceleration, acc);
  if (scheme == 1) {
    store(f.integrator_position_slots[0], slot_pos);
    store(f.integrator_velocity_slots[0], slot_vel);
  }
  return 0;
}

// RigidBodyMotion (rigid_body_motion.rs:38-222) driven the way its unit
// tests drive it: built from the 32-double init (see read_rigid), then
// restore_from_checkpoint when `restore` is given (19 doubles: center of
// mass, orientation w,i,j,k, linear velocity, angular momentum, force,
// torque), add_force for each (force, location), reset_forces when `reset`,
// `n_steps` steps of `dt`. Then op 0 velocity_at_point(in), 1
// world_to_local(in), 2 local_to_world(in), 3 local_to_world_vector(in)
// (3 values), or 4 the checkpoint's 19 values followed by the angular
// velocity (22 values).
int oracle_rigid_probe(const double* init32, const double* restore, int n_forces,
                       const double* force, const double* location, int reset, double dt,
                       int n_steps, int op, const double* in, double* out) {
  RigidBodyMotion m;
  read_rigid(init32, m);
  auto v3 = [](const double* p) { return V3{p[0], p[1], p[2]}; };
  if (restore)
    m.restore_from_checkpoint(v3(restore), Quat{restore[3], restore[4], restore[5], restore[6]},
                              v3(restore + 7), v3(restore + 10), v3(restore + 13),
                              v3(restore + 16));
  for (int k = 0; k < n_forces; ++k) m.add_force(v3(force + 3 * k), v3(location + 3 * k));
  if (reset) m.reset_forces();
  for (int s = 0; s < n_steps; ++s) m.step_forward_in_time(dt);
  const V3 p = v3(in);
  V3 r;
  switch (op) {
    case 0: r = m.velocity_at_point(p); break;
    case 1: r = m.world_to_local(p); break;
    case 2: r = m.local_to_world(p); break;
    case 3: r = m.local_to_world_vector(p); break;
    case 4: {
      const double v[22] = {m.center_of_mass.x, m.center_of_mass.y, m.center_of_mass.z,
                            m.orientation.w, m.orientation.x, m.orientation.y, m.orientation.z,
                            m.linear_velocity.x, m.linear_velocity.y, m.linear_velocity.z,
                            m.angular_momentum.x, m.angular_momentum.y, m.angular_momentum.z,
                            m.force.x, m.force.y, m.force.z, m.torque.x, m.torque.y, m.torque.z,
                            m.angular_velocity.x, m.angular_velocity.y, m.angular_velocity.z};
      std::memcpy(out, v, sizeof v);
      return 0;
    }
    default: return 1;
  }
  out[0] = r.x; out[1] = r.y; out[2] = r.z;
  return 0;
}

int oracle_initialize(void* hh) {
  auto* h = (OracleHandle*)hh;
  try {
    h->sys.boundary->initialize(h->sys.params.kernel_support_radius, h->rest_volume_weighting);
    h->sys.new_boxed();
  } catch (...) {
    return 1;
  }
  return 0;
}

int oracle_step(void* hh, int n) {
  auto* h = (OracleHandle*)hh;
  for (int i = 0; i < n; ++i) h->sys.step_forward_in_time();
  return 0;
}

size_t oracle_num_particles(void* hh) { return ((OracleHandle*)hh)->sys.fluid.len(); }

// 16 doubles in Measurement order (solver_iterations as double)
void oracle_measure(void* hh, double* out) {
  Measurement m = ((OracleHandle*)hh)->sys.take_measurement();
  double v[16] = {m.time, m.density, m.density_error, m.kinetic_energy, m.stiffness,
                  m.fluid_viscosity, m.boundary_viscosity, m.fluid_depth,
                  m.rest_density_grid_spacing, m.kernel_support_radius, m.time_step_size,
                  m.target_density_error, (double)m.solver_iterations, m.relaxation_factor,
                  m.time_step_wall_clock_time, m.predicted_density_error};
  std::memcpy(out, v, sizeof v);
}

double oracle_time(void* hh) { return ((OracleHandle*)hh)->sys.time(); }
unsigned long long oracle_steps(void* hh) { return ((OracleHandle*)hh)->sys.time_steps_propagated; }
size_t oracle_hash_duplicates(void* hh) { return ((OracleHandle*)hh)->sys.hash_duplicates; }

// ScalarQuantity at n positions (3n floats) into out (n floats); 0 on
// success, 1 for an unknown quantity code.
int oracle_quantity_at_positions(void* hh, int quantity, size_t n, const float* pos, float* out) {
  System& s = ((OracleHandle*)hh)->sys;
  if (quantity < 0 || quantity > 5) return 1;
  std::vector<V3> eval(n);
  for (size_t i = 0; i < n; ++i) eval[i] = V3{(double)pos[3 * i], (double)pos[3 * i + 1], (double)pos[3 * i + 2]};
  std::vector<float> q = s.quantity_at_positions(quantity, eval);
  for (size_t i = 0; i < n; ++i) out[i] = q[i];
  return 0;
}

// field ids: 0 position, 1 velocity, 2 acceleration, 3 mass, 4 volume,
// 5 pressure, 6 fluid_id, 7 origin, 8 s_f, 9 a_ff, 10 solver velocity slot 0,
// 11 integrator position slot 0, 12 integrator velocity slot 0
int oracle_download(void* hh, int field, double* dst) {
  System& s = ((OracleHandle*)hh)->sys;
  Fluid& f = s.fluid;
  size_t n = f.len();
  auto vec3 = [&](const std::vector<V3>& v) {
    if (v.size() < n) return 1;
    for (size_t i = 0; i < n; ++i) { dst[3 * i] = v[i].x; dst[3 * i + 1] = v[i].y; dst[3 * i + 2] = v[i].z; }
    return 0;
  };
  auto sc = [&](const std::vector<double>& v) {
    if (v.size() < n) return 1;
    for (size_t i = 0; i < n; ++i) dst[i] = v[i];
    return 0;
  };
  switch (field) {
    case 0: return vec3(f.position);
    case 1: return vec3(f.velocity);
    case 2: return vec3(f.acceleration);
    case 3: return sc(f.mass);
    case 4: return sc(f.volume);
    case 5: return sc(f.pressure);
    case 6: for (size_t i = 0; i < n; ++i) dst[i] = f.fluid_id[i]; return 0;
    case 7: for (size_t i = 0; i < n; ++i) dst[i] = f.origin[i]; return 0;
    case 8: return sc(s.iisph.s_f);
    case 9: return sc(s.iisph.a_ff);
    case 10: return f.solver_velocity_slots.empty() ? 1 : vec3(f.solver_velocity_slots[0]);
    case 11: return f.integrator_position_slots.empty() ? 1 : vec3(f.integrator_position_slots[0]);
    case 12: return f.integrator_velocity_slots.empty() ? 1 : vec3(f.integrator_velocity_slots[0]);
  }
  return 1;
}

// Fluid neighbor list (in the oracle's current index space).
size_t oracle_fluid_neighbor_total(void* hh) { return ((OracleHandle*)hh)->sys.fluid_nl.indices.size(); }
void oracle_fluid_neighbors(void* hh, unsigned long long* offsets, unsigned long long* indices) {
  const NeighborList& nl = ((OracleHandle*)hh)->sys.fluid_nl;
  for (size_t i = 0; i < nl.offsets.size(); ++i) offsets[i] = nl.offsets[i];
  for (size_t i = 0; i < nl.indices.size(); ++i) indices[i] = nl.indices[i];
}
// Sample-boundary neighbor list of boundary `bi`.
size_t oracle_boundary_neighbor_total(void* hh, size_t bi) {
  auto* sb = dynamic_cast<StaticSampleBoundary*>(((OracleHandle*)hh)->sys.boundary.get());
  return sb && bi < sb->boundaries.size() ? sb->boundaries[bi].nl.indices.size() : 0;
}
void oracle_boundary_neighbors(void* hh, size_t bi, unsigned long long* offsets,
                               unsigned long long* indices) {
  auto* sb = dynamic_cast<StaticSampleBoundary*>(((OracleHandle*)hh)->sys.boundary.get());
  const NeighborList& nl = sb->boundaries[bi].nl;
  for (size_t i = 0; i < nl.offsets.size(); ++i) offsets[i] = nl.offsets[i];
  for (size_t i = 0; i < nl.indices.size(); ++i) indices[i] = nl.indices[i];
}
// Pseudo volumes of sample boundary `bi`.
int oracle_boundary_volumes(void* hh, size_t bi, double* dst) {
  auto* sb = dynamic_cast<StaticSampleBoundary*>(((OracleHandle*)hh)->sys.boundary.get());
  if (!sb || bi >= sb->boundaries.size()) return 1;
  std::memcpy(dst, sb->boundaries[bi].vol.data(), sb->boundaries[bi].vol.size() * sizeof(double));
  return 0;
}
// Volume-map boundary samples of boundary `bi` for every particle:
// has[n], xb[3n], vb[3n], vol[n] (zeros where absent).
int oracle_vm_samples(void* hh, size_t bi, unsigned char* has, double* xb, double* vb, double* vol) {
  auto* vb_ = dynamic_cast<VolumeMapBoundary*>(((OracleHandle*)hh)->sys.boundary.get());
  if (!vb_ || bi >= vb_->boundaries.size()) return 1;
  const VMBoundary& b = vb_->boundaries[bi];
  size_t n = b.nl_normal.num_samples();
  for (size_t i = 0; i < n; ++i) {
    size_t c = b.nl_normal.count(i);
    has[i] = c ? 1 : 0;
    if (c) {
      size_t k = *b.nl_normal.begin(i);
      xb[3 * i] = b.spos[k].x; xb[3 * i + 1] = b.spos[k].y; xb[3 * i + 2] = b.spos[k].z;
      vb[3 * i] = b.svel[k].x; vb[3 * i + 1] = b.svel[k].y; vb[3 * i + 2] = b.svel[k].z;
      vol[i] = b.svol[k];
    } else {
      for (int d = 0; d < 3; ++d) { xb[3 * i + d] = 0; vb[3 * i + d] = 0; }
      vol[i] = 0;
    }
  }
  return 0;
}
// Rigid body state of boundary `bi`: com[3], quat[4] (w,i,j,k), lin_vel[3],
// ang_mom[3], force[3], torque[3] -> 19 doubles. Returns 1 for static ones.
int oracle_rigid_state(void* hh, size_t bi, double* out) {
  BoundaryHandling* b = ((OracleHandle*)hh)->sys.boundary.get();
  if (bi >= b->count()) return 1;
  RigidBodyMotion* m = b->at(bi).motion();
  if (!m) return 1;
  double v[19] = {m->center_of_mass.x, m->center_of_mass.y, m->center_of_mass.z,
                  m->orientation.w, m->orientation.x, m->orientation.y, m->orientation.z,
                  m->linear_velocity.x, m->linear_velocity.y, m->linear_velocity.z,
                  m->angular_momentum.x, m->angular_momentum.y, m->angular_momentum.z,
                  m->force.x, m->force.y, m->force.z, m->torque.x, m->torque.y, m->torque.z};
  std::memcpy(out, v, sizeof v);
  return 0;
}

// ---- free functions ---------------------------------------------------------
double oracle_kernel_w(double q) { return kernel_w(q); }
double oracle_kernel_dqw(double q) { return kernel_dqw(q); }
double oracle_kernel_function(const double* r, double h) { return kernel_function({r[0], r[1], r[2]}, h); }
void oracle_kernel_gradient(const double* r, double h, double* out) {
  V3 g = kernel_gradient({r[0], r[1], r[2]}, h);
  out[0] = g.x; out[1] = g.y; out[2] = g.z;
}
unsigned long long oracle_map_int_to_uint(int k) { return SpatialHashing::map_int_to_uint(k); }
unsigned long long oracle_hash(int k, int l, int m) { return SpatialHashing::hash(k, l, m); }
void oracle_get_cell(const double* p, double cs, int* out) {
  int32_t c[3];
  SpatialHashing::get_cell({p[0], p[1], p[2]}, cs, c);
  out[0] = c[0]; out[1] = c[1]; out[2] = c[2];
}

struct NLHandle { NeighborList nl; size_t dups; };
void* oracle_find_samples(double range, double cell_size, size_t n, const double* pos, size_t ns,
                          const double* samples) {
  std::vector<V3> p(n), s(ns);
  for (size_t i = 0; i < n; ++i) p[i] = {pos[3 * i], pos[3 * i + 1], pos[3 * i + 2]};
  for (size_t i = 0; i < ns; ++i) s[i] = {samples[3 * i], samples[3 * i + 1], samples[3 * i + 2]};
  auto* h = new NLHandle();
  SpatialHashing sh(cell_size);
  sh.find_samples(range, p, s, h->nl);
  h->dups = sh.last_duplicates;
  return h;
}
size_t oracle_nl_total(void* h) { return ((NLHandle*)h)->nl.indices.size(); }
size_t oracle_nl_duplicates(void* h) { return ((NLHandle*)h)->dups; }
void oracle_nl_copy(void* hh, unsigned long long* offsets, unsigned long long* indices) {
  const NeighborList& nl = ((NLHandle*)hh)->nl;
  for (size_t i = 0; i < nl.offsets.size(); ++i) offsets[i] = nl.offsets[i];
  for (size_t i = 0; i < nl.indices.size(); ++i) indices[i] = nl.indices[i];
}
void oracle_nl_free(void* h) { delete (NLHandle*)h; }

int oracle_gauss_legendre(int deg, double* x, double* w) {
  std::vector<double> xs, ws;
  gauss_legendre(deg, xs, ws);
  std::memcpy(x, xs.data(), deg * sizeof(double));
  std::memcpy(w, ws.data(), deg * sizeof(double));
  return 0;
}

static TriMeshD make_mesh(const double* verts, size_t nv, const unsigned* faces, size_t nf) {
  TriMeshD m;
  m.v.resize(nv);
  for (size_t i = 0; i < nv; ++i) m.v[i] = {verts[3 * i], verts[3 * i + 1], verts[3 * i + 2]};
  m.f.assign(faces, faces + 3 * nf);
  return m;
}
double oracle_mesh_signed_distance(const double* verts, size_t nv, const unsigned* faces,
                                   size_t nf, const double* p) {
  return mesh_signed_distance(make_mesh(verts, nv, faces, nf), {p[0], p[1], p[2]});
}

struct FieldHandle { Serendipity sdf, vm; };
void* oracle_build_fields(const double* verts, size_t nv, const unsigned* faces, size_t nf,
                          double dx, double r, int degree) {
  TriMeshD m = make_mesh(verts, nv, faces, nf);
  auto* h = new FieldHandle();
  build_sdf_field(m, dx, r, h->sdf);
  build_volume_map_field(m, h->sdf, dx, r, degree, h->vm);
  return h;
}
// Builds only the SDF; the volume map is built from `sdf_nodes` supplied later.
void* oracle_build_sdf_only(const double* verts, size_t nv, const unsigned* faces, size_t nf,
                            double dx, double r) {
  TriMeshD m = make_mesh(verts, nv, faces, nf);
  auto* h = new FieldHandle();
  build_sdf_field(m, dx, r, h->sdf);
  return h;
}
void oracle_fields_free(void* h) { delete (FieldHandle*)h; }
// which: 0 sdf, 1 vm. desc[7] = x_min, x_max, dx; n[3]
void oracle_field_desc(void* hh, int which, double* desc, long long* n) {
  const Serendipity& s = which ? ((FieldHandle*)hh)->vm : ((FieldHandle*)hh)->sdf;
  desc[0] = s.x_min.x; desc[1] = s.x_min.y; desc[2] = s.x_min.z;
  desc[3] = s.x_max.x; desc[4] = s.x_max.y; desc[5] = s.x_max.z; desc[6] = s.dx;
  for (int d = 0; d < 3; ++d) n[d] = s.n[d];
}
void oracle_field_nodes(void* hh, int which, double* dst) {
  const Serendipity& s = which ? ((FieldHandle*)hh)->vm : ((FieldHandle*)hh)->sdf;
  std::memcpy(dst, s.nodes.data(), s.nodes.size() * sizeof(double));
}
// Evaluate a field given as raw arrays: returns 0 ok, 1 error.
int oracle_serendipity_function(const double* desc, const long long* n, const double* nodes,
                                const double* p, double* out) {
  Serendipity s;
  s.x_min = {desc[0], desc[1], desc[2]}; s.x_max = {desc[3], desc[4], desc[5]}; s.dx = desc[6];
  for (int d = 0; d < 3; ++d) s.n[d] = n[d];
  s.nodes.assign(nodes, nodes + (size_t)(s.NX() * s.NY() * s.NZ()));
  return s.function({p[0], p[1], p[2]}, *out) ? 0 : 1;
}
int oracle_serendipity_gradient(const double* desc, const long long* n, const double* nodes,
                                const double* p, double* out) {
  Serendipity s;
  s.x_min = {desc[0], desc[1], desc[2]}; s.x_max = {desc[3], desc[4], desc[5]}; s.dx = desc[6];
  for (int d = 0; d < 3; ++d) s.n[d] = n[d];
  s.nodes.assign(nodes, nodes + (size_t)(s.NX() * s.NY() * s.NZ()));
  V3 g;
  if (!s.gradient({p[0], p[1], p[2]}, g)) return 1;
  out[0] = g.x; out[1] = g.y; out[2] = g.z;
  return 0;
}
// One ball-volume evaluation (SDFnWrapper::volume) on a raw SDF field.
int oracle_volume_at(const double* desc, const long long* n, const double* nodes, const double* p,
                     double r, int degree, double* out) {
  Serendipity s;
  s.x_min = {desc[0], desc[1], desc[2]}; s.x_max = {desc[3], desc[4], desc[5]}; s.dx = desc[6];
  for (int d = 0; d < 3; ++d) s.n[d] = n[d];
  s.nodes.assign(nodes, nodes + (size_t)(s.NX() * s.NY() * s.NZ()));
  bool ok;
  *out = volume_at(s, {p[0], p[1], p[2]}, r, degree, ok);
  return ok ? 0 : 1;
}

// Rigid body: one step from a 32-double init (see read_rigid) with an applied
// force/torque; writes the 19-double state of oracle_rigid_state.
int oracle_rigid_body_step(const double* init, const double* force, const double* location,
                           int n_forces, double dt, int n_steps, double* out) {
  RigidBodyMotion m;
  read_rigid(init, m);
  for (int s = 0; s < n_steps; ++s) {
    for (int k = 0; k < n_forces; ++k)
      m.add_force({force[3 * k], force[3 * k + 1], force[3 * k + 2]},
                  {location[3 * k], location[3 * k + 1], location[3 * k + 2]});
    m.step_forward_in_time(dt);
  }
  double v[19] = {m.center_of_mass.x, m.center_of_mass.y, m.center_of_mass.z,
                  m.orientation.w, m.orientation.x, m.orientation.y, m.orientation.z,
                  m.linear_velocity.x, m.linear_velocity.y, m.linear_velocity.z,
                  m.angular_momentum.x, m.angular_momentum.y, m.angular_momentum.z,
                  m.force.x, m.force.y, m.force.z, m.torque.x, m.torque.y, m.torque.z};
  std::memcpy(out, v, sizeof v);
  return 0;
}

int oracle_num_threads() { return num_threads(); }
void oracle_set_num_threads(int n) { set_num_threads(n); }

}  // extern "C"

extern "C" {
// IISPH::solve_and_add_acceleration (iisph.rs:55-96) for one fluid particle
// with a pre-existing acceleration and at most one boundary sample that is its
// Normal neighbor; `com` non-null makes that boundary a dynamic body with the
// given center of mass (the reference's MockBoundary tests,
// simulation_lib/tests/sph/pressure_solver/iisph.rs:495-592). out: pressure,
// acceleration (3), sweeps, predicted density error, the force and torque the
// body received (6).
int oracle_iisph_solve_probe(const double* pos, const double* vel, double mass, double volume,
                             const double* acc0, double dt, double h, double spacing,
                             double gamma_p, double omega, double eps, double tde,
                             const double* bpos, double bvol, const double* com, double* out) {
  System s;
  s.params.time_increment = dt;
  s.params.kernel_support_radius = h;
  s.params.rest_density_grid_spacing = spacing;
  s.params.rest_volume = spacing * spacing * spacing;
  s.params.boundary_pressure_acceleration_weighting = gamma_p;
  s.sp.relaxation_factor = omega;
  s.sp.min_diagonal_element = eps;
  s.sp.target_density_error = tde;
  auto sb = std::make_unique<StaticSampleBoundary>();
  if (bpos) {
    SampleBoundary b;
    b.xb = {V3{bpos[0], bpos[1], bpos[2]}};
    b.vb = {V3{}};
    b.vol = {bvol};
    b.nl.indices = {0};
    b.nl.offsets = {0, 1};
    if (com) {
      b.dynamic = true;
      b.xb_body = b.xb;
      b.state.center_of_mass = V3{com[0], com[1], com[2]};
    }
    sb->boundaries.push_back(std::move(b));
  }
  s.boundary = std::move(sb);
  Fluid& f = s.fluid;
  f.num_active = 1;
  f.position = {V3{pos[0], pos[1], pos[2]}};
  f.velocity = {V3{vel[0], vel[1], vel[2]}};
  f.acceleration = {V3{acc0[0], acc0[1], acc0[2]}};
  f.mass = {mass};
  f.volume = {volume};
  f.pressure = {0.0};
  f.fluid_id = {0};
  f.origin = {0};
  f.resize_slots(0, 0, 1, 1);
  s.fluid_nl.indices.clear();
  s.fluid_nl.offsets = {0, 0};
  s.iisph_solve();
  out[0] = f.pressure[0];
  out[1] = f.acceleration[0].x; out[2] = f.acceleration[0].y; out[3] = f.acceleration[0].z;
  out[4] = s.iisph.last_solver_iterations;
  out[5] = s.iisph.predicted_density_error;
  V3 F{}, T{};
  if (bpos && com) {
    RigidBodyMotion* m = s.boundary->at(0).motion();
    F = m->force;
    T = m->torque;
  }
  out[6] = F.x; out[7] = F.y; out[8] = F.z;
  out[9] = T.x; out[10] = T.y; out[11] = T.z;
  return 0;
}

// Single fluid particle with one static boundary sample of given volume
// (the reference's IISPH MockBoundary tests, simulation_lib/tests/sph/
// pressure_solver/iisph.rs:158-490): runs set_pred_vel, the volume-preserving
// source term and resolve_pressure_globally with AfterIteration(after) (after
// < 0: only the initial guess). out: pressure, a_ff, s_f, sweeps.
int oracle_iisph_probe(const double* pos, const double* vel, double mass, double volume, double dt,
                       double h, double spacing, double gamma_p, double omega, double eps,
                       const double* bpos, double bvol, int after, double* out) {
  System s;
  s.params.time_increment = dt;
  s.params.kernel_support_radius = h;
  s.params.rest_density_grid_spacing = spacing;
  s.params.rest_volume = spacing * spacing * spacing;
  s.params.boundary_pressure_acceleration_weighting = gamma_p;
  s.sp.relaxation_factor = omega;
  s.sp.min_diagonal_element = eps;
  auto sb = std::make_unique<StaticSampleBoundary>();
  if (bpos) {
    SampleBoundary b;
    b.xb = {V3{bpos[0], bpos[1], bpos[2]}};
    b.vb = {V3{}};
    b.vol = {bvol};
    b.nl.indices = {0};
    b.nl.offsets = {0, 1};
    sb->boundaries.push_back(std::move(b));
  }
  s.boundary = std::move(sb);
  Fluid& f = s.fluid;
  f.num_active = 1;
  f.position = {V3{pos[0], pos[1], pos[2]}};
  f.velocity = {V3{vel[0], vel[1], vel[2]}};
  f.acceleration = {V3{}};
  f.mass = {mass};
  f.volume = {volume};
  f.pressure = {0.0};
  f.fluid_id = {0};
  f.origin = {0};
  f.resize_slots(0, 0, 1, 1);
  s.fluid_nl.indices.clear();
  s.fluid_nl.offsets = {0, 0};
  s.iisph.s_f.assign(1, 0.0);
  s.iisph.a_ff.assign(1, 0.0);
  s.iisph.pressure_acc_f.assign(1, V3{});
  s.set_pred_vel_by_applying_acc(false);
  s.set_source_term_vp();
  if (after < 0) {
    s.set_diagonal_element();
    s.iisph_initialize(true);
    s.iisph.last_solver_iterations = 0;
  } else {
    s.resolve_pressure_globally(true, (uint32_t)after, 0.0, true);
  }
  out[0] = f.pressure[0];
  out[1] = s.iisph.a_ff[0];
  out[2] = s.iisph.s_f[0];
  out[3] = s.iisph.last_solver_iterations;
  return 0;
}
}
