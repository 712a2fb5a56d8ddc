// SPH oracle — TEST INFRASTRUCTURE ONLY.
//
// A CPU, f64 restatement of the reference's SPH time-step path
// (SammyMcFly/fluid-simulation, crate `simulation_lib`). The GPU engine is
// compared against it: only `tests/`, `__graft_entry__.smoke()` and
// the `cpu_baseline` / `--impl reference` legs of `bench.py` load it. Nothing in
// the product (`fluid-simulation_b200/`, `include/`) links or calls it.
//
// Parity pinning: the reference is pure Rust and cannot be compiled here (no
// cargo/rustc, no vendored crates). This restatement is pinned to the
// reference's own known-answer tests (kernel constants and values, hash values,
// strict-range neighbor semantics, volume / viscosity / pressure formulas,
// the one-sweep IISPH pressure, the Euler-Cromer recurrence, rigid-body
// quaternion steps), which `tests/test_oracle_known_answers.py` restates.
// Where a reference test disagrees with its code (the IISPH iteration-count
// tests), this file follows the code.
//
// Every function cites the reference file:line it follows. Path prefixes:
//   SL/ = simulation_lib/src/
#pragma once

#include <cmath>
#include <functional>
#include <thread>
#include <cstddef>
#include <cstdint>
#include <limits>
#include <memory>
#include <unordered_map>
#include <vector>

namespace oracle {

// Static-chunked parallel loop over [0, n) on the host's hardware threads
// (the build has no OpenMP runtime). Each index runs exactly once; chunk
// boundaries depend only on n and the thread count.
int num_threads();
void set_num_threads(int n);
void parallel_for(size_t n, const std::function<void(size_t, size_t)>& body);

// ---------------------------------------------------------------------------
// Vector arithmetic with nalgebra's evaluation order: 3-vector dot products and
// squared norms sum as (x*x + y*y) + z*z with no FMA (built with
// -ffp-contract=off).
// ---------------------------------------------------------------------------
struct V3 {
  double x = 0, y = 0, z = 0;
};
inline V3 operator+(V3 a, V3 b) { return {a.x + b.x, a.y + b.y, a.z + b.z}; }
inline V3 operator-(V3 a, V3 b) { return {a.x - b.x, a.y - b.y, a.z - b.z}; }
inline V3 operator-(V3 a) { return {-a.x, -a.y, -a.z}; }
inline V3 operator*(double s, V3 a) { return {s * a.x, s * a.y, s * a.z}; }
inline V3 operator*(V3 a, double s) { return {a.x * s, a.y * s, a.z * s}; }
inline V3 operator/(V3 a, double s) { return {a.x / s, a.y / s, a.z / s}; }
inline V3& operator+=(V3& a, V3 b) { a = a + b; return a; }
inline V3& operator-=(V3& a, V3 b) { a = a - b; return a; }
inline double dot(V3 a, V3 b) { return (a.x * b.x + a.y * b.y) + a.z * b.z; }
inline double norm_squared(V3 a) { return dot(a, a); }
inline double norm(V3 a) { return std::sqrt(norm_squared(a)); }
inline V3 cross(V3 a, V3 b) {
  return {a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x};
}

struct M3 {  // row-major
  double m[3][3] = {{0, 0, 0}, {0, 0, 0}, {0, 0, 0}};
};
M3 mul(const M3& a, const M3& b);
V3 mul(const M3& a, V3 v);
M3 transpose(const M3& a);

struct Quat {  // w + i x + j y + k z
  double w = 1, x = 0, y = 0, z = 0;
};
Quat qmul(Quat a, Quat b);
V3 qrotate(Quat q, V3 v);
M3 qto_matrix(Quat q);
Quat qfrom_scaled_axis(V3 v);

// ---------------------------------------------------------------------------
// Kernel: CubicBSpline3D (SL/sph/kernel/mod.rs:17-46, cubic_spline.rs:7-17)
// ---------------------------------------------------------------------------
double kernel_w(double q);
double kernel_dqw(double q);
double kernel_function(V3 r, double h);
V3 kernel_gradient(V3 r, double h);

// ---------------------------------------------------------------------------
// NeighborList (SL/neighbor_search/mod.rs:49-161): CSR of usize indices,
// duplicates kept verbatim.
// ---------------------------------------------------------------------------
struct NeighborList {
  std::vector<size_t> indices;
  std::vector<size_t> offsets{0};
  size_t num_samples() const { return offsets.size() - 1; }
  size_t count(size_t id) const { return offsets[id + 1] - offsets[id]; }
  const size_t* begin(size_t id) const { return indices.data() + offsets[id]; }
  const size_t* end(size_t id) const { return indices.data() + offsets[id + 1]; }
};

// ---------------------------------------------------------------------------
// SpatialHashing (SL/neighbor_search/spatial_hashing.rs:20-159)
// ---------------------------------------------------------------------------
struct SpatialHashing {
  double cell_size;
  std::unordered_map<uint64_t, std::vector<size_t>> cells;
  explicit SpatialHashing(double search_range) : cell_size(search_range) {}

  static int32_t saturating_i32(double v);
  static void get_cell(V3 p, double cell_size, int32_t out[3]);
  static uint64_t map_int_to_uint(int32_t k);
  static uint64_t hash(int32_t k, int32_t l, int32_t m);
  void populate(const std::vector<V3>& samples);
  void find_samples(double search_range, const std::vector<V3>& positions,
                    const std::vector<V3>& samples, NeighborList& nl);
  // Number of duplicate entries the XOR-prime hash produced in the last
  // find_samples call (two stencil cells sharing a hash bucket).
  size_t last_duplicates = 0;
};

// ---------------------------------------------------------------------------
// Parameters (SL/sph/mod.rs:753-830, SL/sph/setup/input.rs Parameters)
// ---------------------------------------------------------------------------
enum class Gravity { Uniform = 0, Radial = 1 };
struct SystemParameters {
  double time_increment = 0;
  bool cfl = false;
  double max_time_increment = 0, cfl_number = 0;
  double current_time = 0;  // cfl mode
  double time_offset = 0;   // fixed mode
  uint64_t time_offset_steps = 0;
  double kernel_support_radius = 0;
  double disable_particles_below = -1e300;
  double rest_volume = 0;
  double rest_density_grid_spacing = 0;
  double fluid_viscosity = 0, boundary_viscosity = 0;
  double boundary_pressure_acceleration_weighting = 0;
  Gravity gravity = Gravity::Uniform;
  V3 gravity_center;
};

// ---------------------------------------------------------------------------
// Fluid SoA (SL/sph/fluid.rs:26-210)
// ---------------------------------------------------------------------------
struct Fluid {
  std::vector<uint32_t> fluid_id;
  std::vector<V3> position, velocity, acceleration;
  std::vector<double> mass, volume, pressure;
  std::vector<std::vector<V3>> integrator_position_slots, integrator_velocity_slots;
  std::vector<std::vector<V3>> solver_position_slots, solver_velocity_slots;
  // Original upload index of each particle (test bookkeeping, not physics).
  std::vector<uint32_t> origin;
  size_t num_active = 0;
  size_t len() const { return num_active; }
  void resize_slots(size_t ip, size_t iv, size_t sp, size_t sv);
  void disable(size_t id);
  void swap(size_t a, size_t b);
  void drop_inactive();
};

// ---------------------------------------------------------------------------
// Rigid-body motion (SL/sph/boundary_handling/rigid_body_motion.rs:22-223)
// ---------------------------------------------------------------------------
struct RigidBodyMotion {
  double mass = 1;
  M3 inertia_tensor_inv_body;
  V3 center_of_mass;
  Quat orientation;
  V3 linear_velocity, angular_momentum, force, torque;
  M3 inertia_tensor_inv_world;
  V3 angular_velocity;

  RigidBodyMotion() = default;
  RigidBodyMotion(double mass, const M3& inertia_body, const M3& inertia_inv_body, V3 com,
                  Quat orientation, V3 lin_vel, V3 ang_vel);
  void update_derived_variables();
  V3 local_to_world(V3 p) const;
  V3 world_to_local(V3 p) const;
  V3 local_to_world_vector(V3 v) const;
  V3 velocity_at_point(V3 p) const;
  void add_force(V3 f, V3 location);
  void reset_forces();
  void step_forward_in_time(double dt);
  void restore_from_checkpoint(V3 com, Quat q, V3 lin_vel, V3 ang_momentum, V3 f, V3 t);
};

// ---------------------------------------------------------------------------
// Boundary seam (SL/sph/boundary_handling/mod.rs:39-126)
// ---------------------------------------------------------------------------
enum class RequestMode { Normal, ViscosityAcceleration };

struct Boundary {
  virtual ~Boundary() = default;
  virtual std::pair<const size_t*, const size_t*> get_neighbors(size_t id,
                                                                RequestMode mode) const = 0;
  virtual V3 position(size_t id) const = 0;
  virtual V3 velocity(size_t id) const = 0;
  virtual double volume(size_t id) const = 0;
  virtual bool is_dynamic() const = 0;
  virtual RigidBodyMotion* motion() = 0;
};

struct BoundaryHandling {
  virtual ~BoundaryHandling() = default;
  virtual void initialize(double kernel_support_radius, double rest_volume_weighting) = 0;
  virtual void find_boundary_samples(double search_range, const std::vector<V3>& positions,
                                     double rest_density_grid_spacing) = 0;
  virtual size_t count() const = 0;
  virtual Boundary& at(size_t i) = 0;
  virtual const Boundary& at(size_t i) const = 0;
  virtual void step_forward_in_time(double dt) = 0;
  virtual std::unique_ptr<BoundaryHandling> clone() const = 0;
  void add_force_onto_boundary(size_t id, V3 force, V3 location);
};

// StaticSampleBoundary (SL/sph/boundary_handling/static_sample_boundary.rs)
struct SampleBoundary : Boundary {
  bool dynamic = false;
  std::vector<V3> xb_body, xb, vb;
  std::vector<double> vol;
  RigidBodyMotion state;
  NeighborList nl;
  std::pair<const size_t*, const size_t*> get_neighbors(size_t id, RequestMode) const override {
    return {nl.begin(id), nl.end(id)};
  }
  V3 position(size_t id) const override { return xb[id]; }
  V3 velocity(size_t id) const override { return vb[id]; }
  double volume(size_t id) const override { return vol[id]; }
  bool is_dynamic() const override { return dynamic; }
  RigidBodyMotion* motion() override { return dynamic ? &state : nullptr; }
  void update_positions_and_velocities();
};

struct StaticSampleBoundary : BoundaryHandling {
  std::vector<SampleBoundary> boundaries;
  double cell_size = 0;
  void initialize(double kernel_support_radius, double rest_volume_weighting) override;
  void find_boundary_samples(double search_range, const std::vector<V3>& positions,
                             double spacing) override;
  size_t count() const override { return boundaries.size(); }
  Boundary& at(size_t i) override { return boundaries[i]; }
  const Boundary& at(size_t i) const override { return boundaries[i]; }
  void step_forward_in_time(double dt) override;
  std::unique_ptr<BoundaryHandling> clone() const override {
    return std::make_unique<StaticSampleBoundary>(*this);
  }
};

// CubicSerendipityDiscretization evaluation (SL/utilities/discretization.rs:81-557),
// stored as a dense node lattice of (3n+1)^3 values with NaN marking absent nodes.
struct Serendipity {
  V3 x_min, x_max;
  double dx = 1;
  int64_t n[3] = {0, 0, 0};
  std::vector<double> nodes;  // index ((kz*NY)+ky)*NX+kx, NX=3n0+1...
  int64_t NX() const { return 3 * n[0] + 1; }
  int64_t NY() const { return 3 * n[1] + 1; }
  int64_t NZ() const { return 3 * n[2] + 1; }
  // Returns false on OutOfBounds / PrunedCell.
  bool function(V3 p, double& out) const;
  bool gradient(V3 p, V3& out) const;
};

// VolumeMapBoundary per-step sampling (volume_map_boundary.rs:1259-1424) and
// rigid-rigid contact (volume_map_boundary.rs:55-1102, solve_contacts below).
struct VMBoundary : Boundary {
  bool dynamic = false;
  Serendipity sdf, vm;
  RigidBodyMotion state;
  // Mesh bounding box in the body frame (trimesh.local_aabb(),
  // volume_map_boundary.rs:1137-1150); boundaries without one take no part
  // in rigid-rigid contact.
  bool has_aabb = false;
  V3 aabb_center, aabb_half;
  // flattened samples: Normal entries [0, n_normal), viscosity after
  std::vector<V3> spos, svel;
  std::vector<double> svol;
  NeighborList nl_normal, nl_visc;
  std::pair<const size_t*, const size_t*> get_neighbors(size_t id,
                                                        RequestMode mode) const override {
    const NeighborList& l = mode == RequestMode::Normal ? nl_normal : nl_visc;
    return {l.begin(id), l.end(id)};
  }
  V3 position(size_t id) const override { return spos[id]; }
  V3 velocity(size_t id) const override { return svel[id]; }
  double volume(size_t id) const override { return svol[id]; }
  bool is_dynamic() const override { return dynamic; }
  RigidBodyMotion* motion() override { return dynamic ? &state : nullptr; }
  bool signed_distance(V3 p, double& out) const;
  bool signed_distance_gradient(V3 p, V3& out) const;
  bool volume_map_value(V3 p, double& out) const;
  V3 velocity_at_point_on_boundary(V3 p) const;
};

// Result of one rigid-rigid contact solve (volume_map_boundary.rs:186-645).
struct ContactResult {
  size_t cells = 0;
  uint32_t iterations = 0;
  std::vector<V3> force, torque;  // per boundary, added to the dynamic ones
};

struct VolumeMapBoundary : BoundaryHandling {
  std::vector<VMBoundary> boundaries;
  double kernel_support_radius = 0;
  // Sweep cap of the contact solve; the reference loops until converged.
  uint32_t contact_iteration_cap = 100000;
  // > 0: exactly this many sweeps after the first (no merit test), so that
  // solvers that sum in other orders can be compared on the same iterate.
  uint32_t contact_fixed_sweeps = 0;
  void initialize(double ksr, double) override { kernel_support_radius = ksr; }
  // Contact cells, NNCG-accelerated projected Jacobi for the contact
  // pressures and frictions, and the resulting forces and torques; with
  // `commit` they are added to the bodies.
  ContactResult solve_contacts(double dt, bool commit);
  void find_boundary_samples(double search_range, const std::vector<V3>& positions,
                             double spacing) override;
  size_t count() const override { return boundaries.size(); }
  Boundary& at(size_t i) override { return boundaries[i]; }
  const Boundary& at(size_t i) const override { return boundaries[i]; }
  void step_forward_in_time(double dt) override;
  std::unique_ptr<BoundaryHandling> clone() const override {
    return std::make_unique<VolumeMapBoundary>(*this);
  }
};

// Volume-map field construction (volume_map_boundary.rs:1547-1741,
// discretization.rs:33-245).
struct TriMeshD {
  std::vector<V3> v;
  std::vector<uint32_t> f;  // 3 per triangle
};
double mesh_signed_distance(const TriMeshD& mesh, V3 p);
bool gauss_legendre(int degree, std::vector<double>& x, std::vector<double>& w);
void build_sdf_field(const TriMeshD& mesh, double dx, double kernel_support_radius,
                     Serendipity& out);
void build_volume_map_field(const TriMeshD& mesh, const Serendipity& sdf, double dx,
                            double kernel_support_radius, int quadrature_degree,
                            Serendipity& out);
double volume_at(const Serendipity& sdf, V3 p, double r, int degree, bool& ok);

// ---------------------------------------------------------------------------
// Pressure solvers and integrators (SL/sph/pressure_solver/*, integration_schemes/*)
// ---------------------------------------------------------------------------
enum class Solver { SESPH = 0, SESPHwSplitting = 1, IISPH = 2, IISPHwOST = 3 };
enum class Integrator { EulerCromer = 0, TakePredicted = 1 };
// IntegrationScheme::integrate of the first n particles (euler_cromer.rs:12-25,
// take_predicted.rs:14-27); TakePredicted swaps whole slot 0 with the state.
void integrate(Integrator scheme, Fluid& fluid, size_t n, double dt);

struct SolverParams {
  double stiffness = 1000;
  double target_density_error = 0.1;
  double relaxation_factor = 0.5;
  double min_diagonal_element = 1e-10;
  uint32_t iteration_cap = 0xffffffffu;  // sweeps; the reference has none (u32::MAX)
};

struct IISPHState {
  std::vector<double> s_f, a_ff;
  std::vector<V3> pressure_acc_f;
  uint32_t last_solver_iterations = 0;
  double predicted_density_error = 0;
};

struct Measurement {  // SL/measurement.rs:59-78
  double time, density, density_error, kinetic_energy, stiffness, fluid_viscosity,
      boundary_viscosity, fluid_depth, rest_density_grid_spacing, kernel_support_radius,
      time_step_size, target_density_error;
  uint32_t solver_iterations;
  double relaxation_factor, time_step_wall_clock_time, predicted_density_error;
};

// ---------------------------------------------------------------------------
// Fluid surface reconstruction for render frames (Fluid::reconstruct_surfaces,
// SL/sph/fluid.rs:212-347), whose core is the third-party splashsurf_lib
// 0.14.1 `reconstruct_surface` (absent from the reference tree). Restated
// from its published method: particle densities with the cubic spline of the
// compact support radius and particle mass rest_density * 4/3 pi r^3, the
// level set phi(x) = sum_i (m / rho_i) W(x - x_i) on a grid of cube_size
// aligned to multiples of the cube size, marching cubes at the iso value
// (0.6) with vertices interpolated linearly on crossing edges, then the
// area-weighted vertex normals of fluid.rs:296-323.
// ---------------------------------------------------------------------------
struct SurfaceMesh {
  uint32_t fluid_id = 0;
  std::vector<V3> position, normal;
  std::vector<uint32_t> indices;
};
struct SurfaceGrid {  // the marching-cubes lattice of one group: point k at cube * (k0 + k)
  int64_t k0[3] = {0, 0, 0};
  double cube = 0;
  int64_t n[3] = {0, 0, 0};  // points per axis
  double coord(int d, int64_t k) const { return cube * (double)(k0[d] + k); }
};
SurfaceGrid surface_grid(const std::vector<V3>& positions, double h, double cube);
std::vector<SurfaceMesh> reconstruct_surfaces(const Fluid& fluid, double spacing, double rest_volume, double h);

struct System {
  SystemParameters params;
  SolverParams sp;
  Solver solver = Solver::IISPH;
  Integrator integrator = Integrator::EulerCromer;
  Fluid fluid;
  NeighborList fluid_nl;
  std::unique_ptr<BoundaryHandling> boundary;
  SpatialHashing ns{1.0};
  IISPHState iisph;
  std::vector<double> density_pred;  // SESPHwSplitting scratch
  uint64_t time_steps_propagated = 0;
  double average_density = 0;
  double wall_clock = 0;
  size_t hash_duplicates = 0;

  System() = default;
  System(const System& o);

  double time() const;
  void new_boxed();  // slots + first update (SL/sph/mod.rs:389-421)
  void step_forward_in_time();
  void update();
  void calc_acceleration();
  double calc_max_speed() const;
  double calc_average_mass_density() const;
  double calc_average_mass_density_error() const;
  double calc_average_kinetic_energy() const;
  Measurement take_measurement() const;

  // pieces
  void get_volume();
  // ScalarQuantity at arbitrary positions (sensor planes), f32 in and out.
  std::vector<float> quantity_at_positions(int quantity, const std::vector<V3>& eval);
  void add_gravity_acceleration();
  void add_viscosity_acceleration();
  void set_pred_vel_by_applying_acc(bool to_pred_vel);
  void add_pressure_acceleration(std::vector<V3>* custom_target, bool with_pred_positions,
                                 bool overwrite, bool mirror);
  void sesph();
  void sesph_w_splitting();
  void iisph_solve();
  void iisph_w_ost();
  void set_source_term_vde();
  void set_source_term_vp();
  void set_diagonal_element();
  void iisph_initialize(bool clamp);
  void resolve_pressure_globally(bool after_iteration, uint32_t n_after, double tde,
                                 bool clamp);
};

}  // namespace oracle
