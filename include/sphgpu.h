/*
 * sphgpu.h — C ABI of the B200 SPH step engine.
 *
 * This is the boundary a host written in any language binds (the reference's
 * Rust workspace through an `extern "C"` FFI crate; Python through ctypes).
 * Plain pointers and sizes only. Every entry point returns an `int` status
 * (`SPH_OK` or an `SPH_ERR_*` / `SPH_NOT_CONVERGED` code) and never unwinds
 * across the boundary; `sph_last_error()` returns the calling thread's
 * message for the last failure.
 *
 * Reference interfaces (SammyMcFly/fluid-simulation, paths under
 * simulation_lib/src/) that each entry point replaces are cited beside it.
 * The production seam is the object-safe `SPHSystem` trait
 * (sph/mod.rs:40-69): a handle owns all particle state on the GPU and copies
 * it back only when asked (recording / render frames / checkpoints).
 *
 * Threading: a handle is driven by one host thread at a time; each handle
 * owns its CUDA stream.
 */
#ifndef SPHGPU_H
#define SPHGPU_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ---- status codes ------------------------------------------------------ */
enum sph_status {
  SPH_OK = 0,
  SPH_ERR_INVALID = 1,      /* bad argument or unsupported combination */
  SPH_ERR_OOM = 2,          /* device allocation failed */
  SPH_ERR_CUDA = 3,         /* CUDA runtime error (no device, launch failure) */
  SPH_NOT_CONVERGED = 4,    /* IISPH hit `max_solver_iterations` (step still completed) */
  SPH_ERR_STATE = 5,        /* call out of order (e.g. step before initialize) */
  SPH_ERR_CAPACITY = 6,     /* a caller buffer is too small; required size returned */
  SPH_PENDING = 7,          /* a served scene has not finished yet */
};

/* ---- procedure variants (sph/setup/input.rs:101-134 `Procedures`) ------ */
enum sph_kernel_fn { SPH_CUBIC_BSPLINE_3D = 0 };                 /* kernel/mod.rs:9-12 */
enum sph_integration_scheme {                                      /* integration_schemes/mod.rs:15-21 */
  SPH_EULER_CROMER = 0,
  SPH_TAKE_PREDICTED = 1,
};
enum sph_pressure_solver {                                         /* pressure_solver/mod.rs:29-35 */
  SPH_SESPH = 0,
  SPH_SESPH_W_SPLITTING = 1,
  SPH_IISPH = 2,
  SPH_IISPH_W_OST = 3,
};
enum sph_neighbor_search { SPH_SPATIAL_HASHING = 0 };             /* neighbor_search/mod.rs:13-16 */
enum sph_boundary_handling {                                       /* boundary_handling/mod.rs:33-37 */
  SPH_STATIC_SAMPLE_BOUNDARY = 0,
  SPH_VOLUME_MAP_BOUNDARY = 1,
};
enum sph_precision { SPH_F32 = 0, SPH_F64 = 1 };
enum sph_gravity_mode { SPH_GRAVITY_UNIFORM = 0, SPH_GRAVITY_RADIAL = 1 };

/* ---- configuration: `Parameters` (sph/setup/input.rs:56-260) + procedures */
typedef struct sph_config {
  int kernel_fn;                /* enum sph_kernel_fn */
  int integration_scheme;       /* enum sph_integration_scheme */
  int pressure_solver;          /* enum sph_pressure_solver */
  int neighbor_search;          /* enum sph_neighbor_search */
  int boundary_handling;        /* enum sph_boundary_handling */
  int precision;                /* enum sph_precision: state and bulk arithmetic */
  int cfl_time_step;            /* 0: fixed time_increment; 1: CFL (feature `cfl_time_step`) */
  int gravity_mode;             /* enum sph_gravity_mode */
  double rest_density_grid_spacing;
  double kernel_support_radius;
  double disable_particles_below;
  double fluid_viscosity;
  double boundary_viscosity;
  double boundary_pressure_acceleration_weighting;  /* gamma_p */
  double boundary_rest_volume_weighting;            /* gamma_V */
  double stiffness;                                 /* SESPH k */
  double target_density_error;                      /* IISPH, in percent */
  double relaxation_factor;                         /* IISPH omega */
  double min_diagonal_element;                      /* IISPH epsilon */
  double time_increment;                            /* fixed dt */
  double max_time_increment;                        /* CFL dt cap */
  double cfl_number;
  double gravity_center[3];                         /* radial gravity */
  uint32_t max_solver_iterations; /* 0 = unbounded like the reference; else a cap
                                     that ends the solve with SPH_NOT_CONVERGED */
  uint32_t neighbor_capacity;     /* fluid neighbors stored per particle (16-bit entries);
                                     0 = 128; grows when a step needs more */
  int device;                     /* CUDA device ordinal */
} sph_config;

/* Fills `cfg` with the reference's defaults for the numeric fields
 * (params.toml semantics) and CubicBSpline3D / EulerCromer / IISPH /
 * SpatialHashing / VolumeMapBoundary, f32. */
void sph_config_default(sph_config* cfg);

/* Rigid-body initial state for a dynamic boundary
 * (rigid_body_motion.rs:39-65 `RigidBodyMotion::new`). */
typedef struct sph_rigid_init {
  double mass;
  double inertia_body[9];       /* row-major, body frame */
  double inertia_inv_body[9];   /* row-major, body frame */
  double center_of_mass[3];     /* world */
  double orientation[4];        /* quaternion w, i, j, k */
  double linear_velocity[3];
  double angular_velocity[3];
} sph_rigid_init;

/* Dense cubic-serendipity node lattice of a volume-map field
 * (utilities/discretization.rs:81-94): n cells per axis, 3n+1 nodes per
 * axis, node (kx,ky,kz) at nodes[(kz*(3n_y+1)+ky)*(3n_x+1)+kx] and position
 * x_min + k*dx/3. NaN marks an absent (pruned) node. */
typedef struct sph_grid_desc {
  double x_min[3];
  double x_max[3];
  double dx;
  int64_t n[3];
} sph_grid_desc;

/* Measurement row (measurement.rs:59-78). */
typedef struct sph_measurement {
  double time;
  double density;
  double density_error;
  double kinetic_energy;
  double stiffness;
  double fluid_viscosity;
  double boundary_viscosity;
  double fluid_depth;
  double rest_density_grid_spacing;
  double kernel_support_radius;
  double time_step_size;
  double target_density_error;
  uint32_t solver_iterations;
  double relaxation_factor;
  double time_step_wall_clock_time;
  double predicted_density_error;
} sph_measurement;

/* Per-particle fields for sph_download (reference index order). */
enum sph_field {
  SPH_FIELD_POSITION = 0,        /* 3 doubles per particle */
  SPH_FIELD_VELOCITY = 1,        /* 3 */
  SPH_FIELD_ACCELERATION = 2,    /* 3 */
  SPH_FIELD_MASS = 3,            /* 1 */
  SPH_FIELD_VOLUME = 4,          /* 1 */
  SPH_FIELD_PRESSURE = 5,        /* 1 */
  SPH_FIELD_FLUID_ID = 6,        /* 1 (as double) */
  SPH_FIELD_SOURCE_TERM = 8,     /* 1, IISPH s_f (iisph.rs:31) */
  SPH_FIELD_DIAGONAL = 9,        /* 1, IISPH a_ff (iisph.rs:32) */
  SPH_FIELD_PREDICTED_VELOCITY = 10, /* 3, solver velocity slot 0 */
  SPH_FIELD_INTEGRATOR_POSITION = 11,/* 3, integrator position slot 0 */
  SPH_FIELD_INTEGRATOR_VELOCITY = 12,/* 3, integrator velocity slot 0 */
};

/* Scalar quantities of render_info.rs `ScalarQuantity` (sph/mod.rs:202-239). */
enum sph_quantity {
  SPH_Q_SPEED = 0, SPH_Q_VOLUME = 1, SPH_Q_DENSITY = 2, SPH_Q_DENSITY_ERROR = 3,
  SPH_Q_PRESSURE = 4, SPH_Q_KINETIC_ENERGY = 5,
};

typedef struct sph_system sph_system_t;

/* ---- lifetime (SPHSystem, sph/mod.rs:40-71; System::new_boxed :389-421) -- */
/* Creates an empty system on cfg->device. Rejects the pairings the reference
 * rejects in SystemConstructor::new (sph/setup/mod.rs:229-244). */
int sph_create(const sph_config* cfg, sph_system_t** out);
void sph_destroy(sph_system_t* h);
/* Deep copy of all device state (SPHSystem: DynClone, sci-phi-backend/src/lib.rs:111). */
int sph_clone(const sph_system_t* h, sph_system_t** out);

/* Fluid samples (Fluid::add_samples fluid.rs:79-104 / the `--state` restore
 * path sph/setup/mod.rs:142-153): positions/velocities 3*n doubles, masses n
 * doubles, fluid ids n (may be NULL = 0). */
int sph_upload_fluid(sph_system_t* h, size_t n, const double* position, const double* velocity,
                     const double* mass, const uint32_t* fluid_id);

/* StaticSampleBoundary::add_static_boundary / add_dynamic_boundary
 * (static_sample_boundary.rs:48-140): surface samples (3*nb doubles), world
 * frame for static boundaries (rigid == NULL), body frame (centered on the
 * center of mass) for dynamic ones. Writes the boundary index. */
int sph_add_sample_boundary(sph_system_t* h, size_t nb, const double* positions,
                            const sph_rigid_init* rigid, int* boundary_index);

/* VolumeMapBoundary::add_static_boundary / add_dynamic_boundary
 * (volume_map_boundary.rs:1113-1249) with prebuilt fields. */
int sph_add_volume_map_boundary(sph_system_t* h, const sph_grid_desc* sdf, const double* sdf_nodes,
                                const sph_grid_desc* vm, const double* vm_nodes,
                                const sph_rigid_init* rigid, int* boundary_index);

/* The mesh's bounding box in the body frame (center, half extents) of
 * volume-map boundary `bi`, as VolumeMapBoundary keeps it
 * (volume_map_boundary.rs:1137-1150, 1209-1222). Boundaries with a box take
 * part in rigid-rigid contact: before each body step, every pair of
 * overlapping boxes with a dynamic body is cut into contact cells and the
 * contact pressures and frictions are solved (volume_map_boundary.rs:55-1102,
 * 1440-1453). Without boxes there is no contact. Call before initialize. */
int sph_set_volume_map_aabb(sph_system_t* h, int bi, const double* center, const double* half_extents);
/* Contact cells, solver sweeps, whether sub-cells were dropped for capacity,
 * and whether the sweep cap (10000) stopped the solve, for the last step. */
int sph_get_contact_stats(sph_system_t* h, uint32_t* out4);
/* Contact solve stopping rule. 0 (default): the reference's test, stop once
 * the mean Fischer-Burmeister merits of pressure and friction pass their
 * tolerances (volume_map_boundary.rs:163-176). n > 0: exactly n sweeps after
 * the first, like IISPH's AfterIteration, so that two solvers summing in
 * different orders can be compared on the same iterate. Re-captures the step
 * graphs. */
int sph_set_contact_sweeps(sph_system_t* h, uint32_t fixed_sweeps);

/* BoundaryHandling::initialize (boundary_handling/mod.rs:62-67) followed by
 * the first update() of System::new_boxed (sph/mod.rs:418-419). */
int sph_initialize(sph_system_t* h);

/* ---- stepping (sph/mod.rs:125-144, 674-731) ----------------------------- */
/* Advances n_steps time steps. Returns SPH_NOT_CONVERGED (after finishing
 * all steps) if an IISPH solve hit the configured iteration cap. */
int sph_step(sph_system_t* h, uint32_t n_steps);
/* The plugin-style step on host buffers: overwrites the fluid's positions and
 * velocities from host arrays (reference index order, 3n doubles each; either
 * may be NULL to keep the device state), advances n_steps, and copies the new
 * positions and velocities back (either output may be NULL). Host-to-device
 * and device-to-host copies are part of the call; pinned buffers make them
 * fastest. */
int sph_step_host(sph_system_t* h, uint32_t n_steps, const double* position_in,
                  const double* velocity_in, double* position_out, double* velocity_out);
/* The CUDA stream (cudaStream_t) every kernel of this handle runs on, for
 * callers that time or order work against it. */
int sph_get_stream(const sph_system_t* h, void** stream);
int sph_time(const sph_system_t* h, double* out);                         /* :107-116 */
int sph_time_steps_propagated(const sph_system_t* h, uint64_t* out);     /* :118-120 */
int sph_take_measurement(sph_system_t* h, sph_measurement* out);          /* :147-184 */
int sph_num_particles(const sph_system_t* h, size_t* out);

/* ---- readback ----------------------------------------------------------- */
int sph_get_fluid_ids(sph_system_t* h, uint32_t* out);                    /* :186-188 */
int sph_get_fluid_pos(sph_system_t* h, float* out);                       /* :190-196 */
int sph_get_quantity_of_fluid_samples(sph_system_t* h, int quantity, float* out); /* :202-239 */
/* SPHSystem::get_quantity_at_positions (sph/mod.rs:241-341, sums of
 * sph/quantities.rs:14-330): `quantity` (sph_quantity) at n positions
 * (3n floats, e.g. a sensor plane) into out[n], from the state of the last
 * update. Speed and volume include the boundary samples of each position.
 * Unlike the reference, which searches the boundary samples of the
 * positions in place of the fluid's until the next update, the system's
 * state is left unchanged. n == 0 is a no-op. Rejects an unknown quantity
 * (SPH_ERR_INVALID) and a call while a chunk of graph steps is in flight
 * (SPH_ERR_STATE). */
int sph_get_quantity_at_positions(sph_system_t* h, int quantity, size_t n, const float* positions,
                                  float* out);
int sph_download(sph_system_t* h, int field, double* out);
/* Fluid neighbor lists in reference index space, self included, each row
 * sorted ascending (NeighborList, neighbor_search/mod.rs:49-161).
 * offsets: n+1 entries. If `capacity` < total, returns SPH_ERR_CAPACITY and
 * writes the required total. */
int sph_get_fluid_neighbors(sph_system_t* h, uint64_t* offsets, uint32_t* indices,
                            size_t capacity, size_t* total);
/* Sample-boundary neighbors of boundary `bi` (indices into its samples). */
int sph_get_boundary_neighbors(sph_system_t* h, int bi, uint64_t* offsets, uint32_t* indices,
                               size_t capacity, size_t* total);
/* Pseudo volumes of the samples of sample boundary `bi` (upload order). */
int sph_get_boundary_volumes(sph_system_t* h, int bi, double* out);
/* World positions (3 doubles each) of the samples of sample boundary `bi`
 * at the last update, upload order (Boundary::positions,
 * static_sample_boundary.rs:311-321). */
int sph_get_boundary_positions(sph_system_t* h, int bi, double* out);
/* Volume-map samples of boundary `bi` per particle: has[n] (0/1),
 * x_b[3n], v_b[3n], vol[n] (volume_map_boundary.rs:1287-1342). */
int sph_get_volume_map_samples(sph_system_t* h, int bi, uint8_t* has, double* xb, double* vb,
                               double* vol);
/* Rigid-body state of boundary `bi`: com[3], q[4] (w,i,j,k), v[3], L[3],
 * F[3], T[3] (RigidBodyMotionCheckpoint, rigid_body_motion.rs:230-245). */
int sph_get_rigid_state(sph_system_t* h, int bi, double* out19);
int sph_set_rigid_state(sph_system_t* h, int bi, const double* in19);
/* Number of XOR-prime hash collisions between cells of one 3x3x3 stencil
 * among occupied cells at the last update (spatial_hashing.rs:49-71). */
int sph_hash_collisions(sph_system_t* h, uint64_t* out);

/* ---- checkpoints (sph/mod.rs:833-915, continue_from_checkpoint :362-378) - */
/* Restores fluid state (reference order) and the step counter / time, zeroes
 * solver slots, then runs update(). */
int sph_continue_from_checkpoint(sph_system_t* h, uint64_t time_steps_propagated,
                                 double current_time, size_t n, const double* position,
                                 const double* velocity, const double* mass,
                                 const uint32_t* fluid_id, const double* integrator_position,
                                 const double* integrator_velocity);

/* ---- per-trait shims (upload -> kernel -> download), for per-trait parity - */
/* NeighborSearch::find_samples with SpatialHashing (neighbor_search/mod.rs:18-28,
 * spatial_hashing.rs:130-158): neighbors of each of the n positions among the
 * ns samples (cell size = search range), rows in stencil order x->y->z then
 * ascending sample index. */
int sph_spatial_hashing_find_samples(double search_range, size_t n, const double* positions,
                                     size_t ns, const double* samples, uint64_t* offsets,
                                     uint32_t* indices, size_t capacity, size_t* total, int device);
/* Allocation-free variant of sph_spatial_hashing_find_samples. No counterpart
 * in the reference: it exists for callers that cannot allocate device memory
 * (a host whose allocator belongs to another runtime or memory pool, a loop
 * that forbids allocation). Inputs and outputs are DEVICE pointers owned by
 * the caller (positions 3n doubles, samples 3ns doubles, offsets n+1, indices
 * `capacity`); `total` is a host pointer. Every temporary lives in one static
 * device array of about 15 MB that each GPU loading the library holds until
 * the process exits; at most 1,048,576 samples and 1,048,576 positions
 * (larger inputs return SPH_ERR_INVALID). The first call on a device resolves
 * that array's address and should come before any stream capture. The work
 * runs on the legacy default stream of `device`: a caller that writes the
 * inputs on a non-blocking stream must finish that work (synchronize the
 * stream or the device) before the call. All calls share the array, so calls
 * that overlap on the GPU race; the call synchronizes the device before it
 * returns. Results equal those of sph_spatial_hashing_find_samples, rows in
 * the same order. */
int sph_spatial_hashing_find_samples_noalloc(double search_range, size_t n, const double* d_positions,
                                             size_t ns, const double* d_samples, uint64_t* d_offsets,
                                             uint32_t* d_indices, size_t capacity, size_t* total,
                                             int device);
/* KernelFn (kernel/mod.rs:17-46) for CubicBSpline3D on n vectors (3n doubles). */
int sph_kernel_function(size_t n, const double* r, double h, double* out_w, int precision,
                        int device);
int sph_kernel_gradient(size_t n, const double* r, double h, double* out_grad, int precision,
                        int device);

/* ---- volume-map field construction (volume_map_boundary.rs:1547-1741) --- */
/* Grids of a closed triangle mesh's fields: the signed-distance field over the
 * mesh AABB padded by 3.1 r, the volume map padded by 2 r + dx/6, with n =
 * round(extent / dx) cells per axis (discretization.rs:99-113). */
int sph_volume_map_grids(const double* verts, size_t nv, double dx, double kernel_support_radius,
                         sph_grid_desc* sdf_grid, sph_grid_desc* vm_grid);
/* Signed-distance node values of the mesh (3*nv vertex coordinates, 3*nf
 * vertex indices; the side the face winding points to is positive), pruned to
 * the band |sd| <= 3.1 r (NaN elsewhere). nodes_out: (3n_x+1)(3n_y+1)(3n_z+1). */
int sph_build_sdf_field(const double* verts, size_t nv, const uint32_t* faces, size_t nf,
                        const sph_grid_desc* grid, double kernel_support_radius, double* nodes_out,
                        int device);
/* Volume-map node values: the Gauss-Legendre ball integral (degree
 * `quadrature_degree`, the reference uses 30) of the cubic extension function
 * of the discretized signed distance, clamped to [0, 4/3 pi r^3]. */
int sph_build_volume_map_field(const sph_grid_desc* sdf_grid, const double* sdf_nodes,
                               const sph_grid_desc* vm_grid, double kernel_support_radius,
                               int quadrature_degree, double* nodes_out, int device);

/* ---- graph-captured stepping -------------------------------------------- */
/* With chunk_steps > 0, sph_step captures one time step (with its IISPH
 * Jacobi loop as a conditional while-node) into a CUDA graph and advances in
 * chunks of up to chunk_steps graph launches with one host check per chunk
 * instead of one per step. Results are the same as the per-step path: a
 * chunk in which a step needed host work (neighbor capacity growth, disabled
 * particles, a solve still unconverged after 10000 sweeps without a cap) is
 * put back from a device snapshot and replayed per step. 0 (the default)
 * selects the per-step path. Profiling (sph_set_profiling) uses the per-step
 * path. */
int sph_set_step_graphs(sph_system_t* h, uint32_t chunk_steps);
/* Chunks replayed on the per-step path since creation. */
int sph_graph_replays(const sph_system_t* h, uint64_t* out);

/* ---- launch tuning -------------------------------------------------------- */
/* Launch parameters of the neighbor passes that leave every result bit for bit
 * unchanged (the reference has no counterpart; its passes run on the CPU):
 * the number of neighbors a thread gathers per batch (4 or 8; it applies to
 * the passes that test the neighbor count per slot, i.e. SESPHwSplitting's
 * predicted density; the others walk whole groups of four) and the halo
 * records a block copies to shared memory before its neighbor loop (blocks
 * with larger halos, and every block at 0, gather from global memory). The
 * records must fit one block's shared memory. Setting them re-captures the
 * step graphs; clones inherit them. */
typedef struct sph_tuning {
  uint32_t gather_batch;
  uint32_t halo_stage;
  uint32_t sweep_stage;  /* halo records the IISPH sweep passes stage (their
                          * records are 16 and 24 bytes in f32, 32 and 48 in f64) */
} sph_tuning;
int sph_get_tuning(const sph_system_t* h, sph_tuning* out);
int sph_set_tuning(sph_system_t* h, const sph_tuning* tuning);
/* Autotuner: it times candidate tunings on clones of the system (one warm-up
 * step, then `steps` steps on the clone's stream with CUDA events): first the
 * gather batch (4, 8) times three staging capacities per precision, then,
 * with the best of those, three sweep staging capacities. It applies the
 * fastest to `h` and returns it with its time per step in milliseconds
 * (best_ms_per_step may be NULL). The system's own state does not advance. */
int sph_autotune(sph_system_t* h, uint32_t steps, sph_tuning* best, double* best_ms_per_step);

/* ---- diagnostics -------------------------------------------------------- */
/* Scalars of the last completed update, read from the host copy the step
 * already made (no device work). */
typedef struct sph_step_stats {
  uint64_t particles;           /* active particles after the update */
  uint32_t solver_iterations;   /* IISPH sweeps of the (last) pressure solve */
  uint32_t solver_iterations_first; /* IISPHwOST: sweeps of the first solve */
  uint32_t max_neighbors;       /* largest fluid neighbor count (self excluded) */
  uint32_t max_boundary_neighbors;
  double predicted_density_error;
  double time_increment;        /* dt the next step integrates with */
  double average_density;
  int not_converged;            /* 1 if the solve stopped at max_solver_iterations */
} sph_step_stats;
int sph_get_step_stats(const sph_system_t* h, sph_step_stats* out);

const char* sph_last_error(void);
/* Kernel launches issued by this handle since creation (all of its CUDA
 * kernels, every step). */
int sph_launch_count(const sph_system_t* h, uint64_t* out);
/* Event-timed duration (ms) and launch count of the named kernel class,
 * summed over every launch timed while profiling was enabled with
 * sph_set_profiling ("*": all classes). With profiling on, an IISPH solve
 * runs one sweep per host check, so every timed sweep launch does a sweep's
 * work; the results are the same as without profiling. */
int sph_set_profiling(sph_system_t* h, int enabled);
int sph_kernel_time(sph_system_t* h, const char* kernel, double* ms, uint64_t* launches);
/* Device-resident bytes held by the handle. */
int sph_device_bytes(const sph_system_t* h, size_t* out);

/* ---- scene server: continuous batching of scene solves on one GPU -------- */
/* The reference runs one scene per backend worker (sci-phi-backend/src/lib.rs:
 * 190-210 steps a Box<dyn SPHSystem> in a loop). The server is the request
 * loop form of that worker: scenes are submitted at any time, admitted while
 * the device has slots and memory for them (an estimate of each scene's
 * device bytes against a budget), advanced concurrently (each on its own
 * stream, in chunks of graph-captured steps issued by one scheduler thread)
 * and retired at their step count. A scene's result does not depend on what
 * else runs beside it. */
typedef struct sph_server sph_server_t;

typedef struct sph_server_config {
  int device;                   /* CUDA device ordinal */
  uint64_t memory_budget_bytes; /* 0: 90 % of the device memory free at creation */
  uint32_t max_active;          /* scenes on the device at once; 0: 64 */
  uint32_t chunk_steps;         /* graph launches per host check; 0: 25 */
} sph_server_config;

typedef struct sph_sample_set {   /* one sph_add_sample_boundary call */
  size_t count;
  const double* positions;        /* 3*count */
  const sph_rigid_init* rigid;    /* NULL: static */
} sph_sample_set;

typedef struct sph_volume_map_set {  /* one sph_add_volume_map_boundary call */
  const sph_grid_desc* sdf;
  const double* sdf_nodes;
  const sph_grid_desc* vm;
  const double* vm_nodes;
  const sph_rigid_init* rigid;
} sph_volume_map_set;

typedef struct sph_scene_request {
  sph_config config;
  size_t n;                       /* fluid particles */
  const double* position;         /* 3n */
  const double* velocity;         /* 3n or NULL */
  const double* mass;             /* n */
  const uint32_t* fluid_id;       /* n or NULL */
  size_t num_sample_sets;
  const sph_sample_set* sample_sets;
  size_t num_volume_maps;
  const sph_volume_map_set* volume_maps;
  uint32_t steps;                 /* time steps to run */
  int keep_state;                 /* 1: keep the final positions/velocities */
} sph_scene_request;

typedef struct sph_scene_result {
  int status;                     /* SPH_OK, SPH_NOT_CONVERGED or an error code */
  uint64_t steps;                 /* steps run */
  double time;                    /* simulated time */
  uint64_t particles;             /* active particles at the end */
  sph_measurement measurement;    /* take_measurement at the end */
  double submit_s, start_s, finish_s;  /* seconds since server creation */
  uint64_t device_bytes_reserved; /* admission estimate */
  uint64_t graph_replays;         /* chunks redone on the per-step path */
  uint64_t kernel_launches;
} sph_scene_result;

typedef struct sph_server_stats {
  uint64_t submitted, completed, queued, active, peak_active;
  uint64_t budget_bytes, reserved_bytes, peak_reserved_bytes;
  uint64_t graph_replays, kernel_launches;
} sph_server_stats;

int sph_server_create(const sph_server_config* cfg, sph_server_t** out);
/* Copies the request (the caller may free its arrays on return). Fails with
 * SPH_ERR_CAPACITY when the scene alone exceeds the memory budget. */
int sph_server_submit(sph_server_t* s, const sph_scene_request* req, uint64_t* ticket);
/* SPH_OK and the result once the scene finished, else SPH_PENDING. */
int sph_server_poll(sph_server_t* s, uint64_t ticket, sph_scene_result* out);
/* Blocks up to timeout_s seconds (< 0: no limit); SPH_PENDING on timeout. */
int sph_server_wait(sph_server_t* s, uint64_t ticket, double timeout_s, sph_scene_result* out);
/* Final positions and velocities (3*particles doubles each, reference index
 * order) of a finished scene submitted with keep_state = 1. */
int sph_server_fetch_state(sph_server_t* s, uint64_t ticket, double* position, double* velocity);
/* Drops a finished scene's result. */
int sph_server_release(sph_server_t* s, uint64_t ticket);
int sph_server_get_stats(sph_server_t* s, sph_server_stats* out);
/* Cancels queued scenes, stops running ones after their current chunk and
 * frees everything. */
void sph_server_destroy(sph_server_t* s);

/* ---- checkpoint and recording formats ----------------------------------- */
/* The readback formats either side of the step: the system checkpoint
 * (SerSystemCheckpoint, sph/mod.rs:883-915) that sci-phi-backend writes as
 * RON (recording.rs:37-61) and the `--state` path reads back
 * (sph/setup/mod.rs:142-153), also in its bincode form (its Encode/Decode
 * derive), and the recording frame (TimeStepInfo, render_info.rs:71-106) in
 * bincode's standard configuration, each record of a recording file being a
 * little-endian u64 length and these bytes (recording.rs:146-210). */
enum sph_format { SPH_FORMAT_RON = 0, SPH_FORMAT_BINCODE = 1 };

/* An owned byte string; `data` stays valid until sph_bytes_free. */
typedef struct sph_bytes sph_bytes_t;
int sph_bytes_get(const sph_bytes_t* b, const uint8_t** data, size_t* len);
void sph_bytes_free(sph_bytes_t* b);

/* SystemCheckpoint as plain arrays (fluid.rs:351-421, reference index order;
 * boundary_handling/mod.rs:135-170, one entry per boundary in add order). */
typedef struct sph_checkpoint_view {
  uint64_t time_steps_propagated;
  double current_time;
  size_t n;                          /* fluid samples */
  const uint32_t* fluid_id;          /* n */
  const double* position;            /* 3n */
  const double* velocity;            /* 3n */
  const double* mass;                /* n */
  size_t integrator_position_slots;  /* slots of 3n doubles each, back to back */
  const double* integrator_position;
  size_t integrator_velocity_slots;
  const double* integrator_velocity;
  size_t num_boundaries;
  const uint8_t* dynamic;            /* per boundary: 1 = rigid state present */
  const double* rigid_state;         /* 19 per boundary, sph_get_rigid_state layout */
} sph_checkpoint_view;

/* An owned checkpoint. */
typedef struct sph_checkpoint sph_checkpoint_t;
int sph_checkpoint_from_view(const sph_checkpoint_view* view, sph_checkpoint_t** out);
/* Fills `view` with pointers into `c` (valid until sph_checkpoint_free). */
int sph_checkpoint_view_of(const sph_checkpoint_t* c, sph_checkpoint_view* view);
void sph_checkpoint_free(sph_checkpoint_t* c);
/* SerSystemCheckpoint -> RON text (ron::to_string) or bincode bytes. */
int sph_checkpoint_encode(const sph_checkpoint_t* c, int format, sph_bytes_t** out);
/* RON text (any whitespace, comments, struct names, field order) or bincode
 * bytes -> checkpoint; SPH_ERR_INVALID with the position of a syntax error. */
int sph_checkpoint_decode(const uint8_t* data, size_t len, int format, sph_checkpoint_t** out);
/* SystemCheckpoint::from_sph_system (sph/mod.rs:849-856). */
int sph_get_checkpoint(sph_system_t* h, sph_checkpoint_t** out);
/* SPHSystem::continue_from_checkpoint (sph/mod.rs:362-378): fluid, rigid
 * states, step counter and time, then update(). The boundaries must match
 * the system's in number and static/dynamic kind, and the integrator slots
 * its integration scheme (TakePredicted: 1 each, else none). */
int sph_restore_checkpoint(sph_system_t* h, const sph_checkpoint_t* c);

/* Recording frames: TimeStepInfo with FluidVisualization::TriangleMesh
 * (reconstructed surfaces), ::Samples or ::SensorPlane, and
 * BoundaryVisualization::Samples or ::TriangleMesh (the caller's render
 * meshes with the boundaries' current poses) (render_info.rs:110-245). */
enum sph_fluid_visualization {
  SPH_FLUID_TRIANGLE_MESH = 0, SPH_FLUID_SAMPLES = 1, SPH_FLUID_SENSOR_PLANE = 2
};

/* Fluid::reconstruct_surfaces (sph/fluid.rs:212-347): one triangle mesh per
 * fluid id (ascending), each vertex 6 doubles (position, area-weighted unit
 * normal), from the device state. The surface is the 0.6 level of
 * phi(x) = sum_i (m / rho_i) W(x - x_i) on a lattice of 0.75 r (r = half the
 * rest spacing), the method of the third-party splashsurf_lib 0.14.1 that
 * the reference calls, restated. */
typedef struct sph_meshes sph_meshes_t;
int sph_reconstruct_surfaces(sph_system_t* h, sph_meshes_t** out);
int sph_meshes_count(const sph_meshes_t* m, size_t* out);
int sph_meshes_get(const sph_meshes_t* m, size_t k, uint32_t* fluid_id, size_t* num_vertices,
                   const double** vertices, size_t* num_indices, const uint32_t** indices);
void sph_meshes_free(sph_meshes_t* m);
enum sph_sample_coloring { SPH_COLORING_UNIFORM = 0, SPH_COLORING_ID = 1, SPH_COLORING_QUANTITY = 2 };

/* BoundaryVisualization variants as this API selects them (the wire format
 * keeps the reference's variant order, TriangleMesh first). */
enum sph_boundary_visualization { SPH_BOUNDARY_SAMPLES = 0, SPH_BOUNDARY_TRIANGLE_MESH = 1 };
/* BoundaryMeshColoring (render_info.rs:259-264). */
enum sph_boundary_mesh_coloring {
  SPH_MESH_ORIGINAL = 0, SPH_MESH_UNIFORM = 1, SPH_MESH_BOUNDARY_ID = 2
};
/* RenderMesh (utilities/triangle_mesh.rs:61-64) of a boundary in its body
 * frame (world frame for a static boundary). */
typedef struct sph_render_mesh {
  const double* vertices;          /* 6 per vertex: position, normal */
  size_t num_vertices;
  const uint32_t* indices;
  size_t num_indices;
} sph_render_mesh;

typedef struct sph_sensor_plane {  /* SensorPlaneData (render_info.rs:196-202) */
  const float* positions;          /* 3 * rows * cols */
  const float* data;               /* rows * cols (frame views only) */
  size_t rows, cols;
} sph_sensor_plane;

/* What a frame shows (the selector TimeStepInfo::from_system takes). */
typedef struct sph_frame_selector {
  int fluid;                       /* sph_fluid_visualization */
  int fluid_coloring;              /* Samples: UNIFORM, ID (fluid id) or QUANTITY;
                                      TriangleMesh: UNIFORM or ID */
  int quantity;                    /* sph_quantity for QUANTITY and SENSOR_PLANE */
  size_t num_planes;
  const sph_sensor_plane* planes;  /* positions, rows, cols (data unused) */
  int boundary_coloring;           /* UNIFORM or ID (render mesh id) */
  const uint32_t* render_mesh_ids; /* per boundary; NULL = the boundary index */
  int boundary_visualization;      /* sph_boundary_visualization */
  int boundary_mesh_coloring;      /* TriangleMesh: sph_boundary_mesh_coloring */
  const sph_render_mesh* render_meshes; /* TriangleMesh: one per boundary */
} sph_frame_selector;

/* A frame's contents (TimeStepInfo itself). */
typedef struct sph_frame_view {
  uint64_t time_step_number;
  sph_measurement measurement;
  int fluid, fluid_coloring, quantity;
  size_t n;                        /* Samples */
  const float* fluid_positions;    /* 3n */
  const uint32_t* fluid_ids;       /* n, ID coloring */
  const float* fluid_data;         /* n, QUANTITY coloring */
  size_t num_planes;
  const sph_sensor_plane* planes;  /* SensorPlane, with data */
  int boundary_coloring;
  size_t num_boundary_samples;
  const float* boundary_positions; /* 3 * num_boundary_samples */
  const uint32_t* boundary_ids;    /* per sample, ID coloring */
  const sph_meshes_t* meshes;      /* TriangleMesh */
  uint32_t max_fluid_id;           /* TriangleMesh: the largest fluid id */
  int boundary_visualization;      /* sph_boundary_visualization */
  int boundary_mesh_coloring;      /* sph_boundary_mesh_coloring */
  size_t num_boundary_meshes;
  const sph_render_mesh* boundary_meshes;
  const float* boundary_poses;     /* 7 per mesh: translation, rotation (i, j, k, w) */
  size_t num_mesh_ids;             /* BOUNDARY_ID coloring: the ids and their count */
  const uint32_t* mesh_ids;
} sph_frame_view;

/* TimeStepInfo -> bincode bytes (render_info.rs:101-106). */
int sph_frame_encode(const sph_frame_view* frame, sph_bytes_t** out);
/* TimeStepInfo::from_system (render_info.rs:83-92) on the device state,
 * encoded; sensor planes are evaluated with sph_get_quantity_at_positions. */
int sph_encode_time_step_info(sph_system_t* h, const sph_frame_selector* sel, sph_bytes_t** out);

#ifdef __cplusplus
}
#endif
#endif /* SPHGPU_H */
