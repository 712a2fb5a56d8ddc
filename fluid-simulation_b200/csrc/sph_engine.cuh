// Device-side state layout and kernel launchers of the SPH step engine.
//
// Layout in HBM (one scene, capacity N, stride Np = N rounded up to 32):
//   pos   R4 {x,y,z,-}      integrated positions, permuted by the cell sort
//   vel   R4 {vx,vy,vz,m}   velocity with the particle mass in w
//   xv    R4 {x,y,z,V}      sorted positions with the current volume in w
//   acc   R4 {ax,ay,az,-}   total acceleration
//   ref   u32               reference-order index (the row a download writes)
//   fid   u32               fluid id
//   nbr   u16 [Np/32][K/4][32][4]  fluid neighbor lists as positions in the
//                           block's halo, warp-tiled: lane `i%32` of tile
//                           `i/32` keeps neighbors 4g..4g+3 in one 8-byte
//                           group; self is implicit, not stored
//   halo  u32 [blocks][hcap] particle indices of each block's halo (the union
//                           of its cells' stencil buckets), ascending
//   ncnt  u32 [N]           neighbor counts
//   bW, bG, bGu             per-particle boundary aggregates (see kernels)
//   IISPH scratch: vstar R4, s R, aii R, accp R4, p R
// Cell grid: a Morton key of floor(x / h) modulo 2^(3m) buckets; a counting
// sort orders particles by bucket and, inside a bucket, by reference index.
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

#include "sph_math.cuh"

namespace sph {

constexpr int kBlock = 256;
// List batches the Jacobi sweep passes keep in flight ahead of the one they consume.
#ifndef SPH_SWEEP_PREFETCH
#define SPH_SWEEP_PREFETCH 2
#endif
constexpr int kSweepPrefetch = SPH_SWEEP_PREFETCH;
constexpr int kMaxBodies = 32;

// Per-scene scalars that stay on the device so that a step needs no host
// round trip (time increment, active count, IISPH convergence state).
struct Scalars {
  double dt;                       // time increment used by this step
  unsigned long long max_speed;    // bits of the max |v| (non-negative double)
  int n;                           // particles entering this update
  int n_active;                    // particles after disabling
  int n_below;                     // particles disabled in this update
  int max_nbrs;                    // largest fluid neighbor count seen
  int iterations;                  // IISPH sweeps of the last solve
  int converged;                   // IISPH loop flag (1 = stop)
  double err;                      // IISPH average predicted density error (%)
  double avg_density;              // average mass density after the update
  unsigned int done_blocks;        // last-block-done counter for reductions
  int status;                      // 0 ok, 2 not converged within the cap
  int iterations_eqs1;             // IISPHwOST first solve sweeps
  int max_bnbrs;                   // largest boundary-sample neighbor count seen
  int max_halo;                    // largest block halo (particles) seen
  unsigned int vm_near;            // particles within the support radius of a volume map
  // graph-captured stepping (the host reads these once per chunk)
  double time_acc;                 // simulated time under CFL steps
  unsigned int trouble;            // bits: 1 neighbor overflow, 2 disabled particles, 4 unconverged
  int status_any;                  // 2 once any step of the chunk hit the sweep cap
  unsigned long long loop_sweeps;  // sweeps run by the graph's solver while-loops
  int chunk_max_nbrs;              // largest fluid neighbor count over the chunk
  int chunk_max_halo;              // largest block halo over the chunk
};

// Parameters that are constant over a step (passed by value).
template <class R>
struct StepParams {
  KernelConst<R> k;
  double range;          // kernel support radius (search range and cell size)
  R range2_lo, range2_hi;
  double spacing;        // rest density grid spacing
  R V0;                  // rest volume spacing^3
  R visc_f, visc_b;      // 10 * viscosity (= nu * 2 * (3 + 2))
  R eps_visc;            // 0.01 * spacing^2
  R gamma_p;             // boundary pressure weighting
  int gravity_mode;      // 0 uniform -z, 1 radial
  R gc[3];               // radial gravity center
  double disable_below;
  uint32_t mask;         // Morton coordinate mask (2^m - 1)
  uint32_t T;            // bucket count; bucket T holds disabled particles
  int K;                 // neighbor capacity per particle
  int Np;                // neighbor stride
  int cfl;               // 1: dt = min(dt_max, cfl * spacing / max|v|)
  double dt_fixed, dt_max, cfl_number;
  R stiffness;
  R omega, min_diag;
  double tde;            // IISPH target density error (%)
  int iteration_cap;     // 0 = unbounded (reference)
  int sorted_lists;      // 1: neighbor lists in ascending index order
};

// Rigid body state, f64 (rigid_body_motion.rs:22-36).
struct Body {
  double mass;
  double inv_inertia_body[9];
  double com[3];
  double q[4];  // w, i, j, k
  double v[3];
  double L[3];
  double F[3];
  double T[3];
  double inv_inertia_world[9];
  double omega[3];
  int dynamic;
  int pad;
};

// Dense serendipity node lattice (3n+1 per axis, NaN = absent node).
struct DevField {
  double xmin[3], xmax[3], dx;
  int n[3];
  long long NX, NY;
  const double* nodes;
};

struct VMDesc {
  DevField sdf, vm;
  int body;                     // index into the body table, -1 for static
  int has_aabb;                 // 1: takes part in rigid-rigid contact
  double aabb_c[3], aabb_h[3];  // mesh bounding box in the body frame
};

// Rigid-rigid contact of volume-map bodies (volume_map_boundary.rs:55-1102).
// A pair of overlapping world bounding boxes is cut into sub-cells (tasks);
// a task whose quadrature finds both bodies' solids becomes a contact cell.
constexpr int kContactQuad = 8;  // Gauss-Legendre points per axis (:57)
// Sweeps of one contact solve at most; the reference iterates until its
// merits converge (it only warns beyond 100 sweeps, :63, :163-176).
constexpr int kContactSweepCap = 10000;
struct ContactGL {
  double x[kContactQuad], w[kContactQuad];
};
struct ContactPair {
  int a, b;
  int n[3];       // sub-cells per axis
  int first;      // first task of the pair
  double min[3];  // overlap box corner
  double cs[3];   // sub-cell size
};
struct ContactCell {  // ContactCell after compute_diagonal (:678-697, 835-926)
  int valid, a, b, pad;
  double volume, center[3], f_a[3], tau_a[3], f_b[3], tau_b[3], tproj[9], acc_p, acc_f;
};
struct ContactState {  // per compacted cell, the solver's iterates
  double p, s_p, v_err, pj, gp;
  double lambda[3], s_l[3], v_tang[3], lj[3], gl[3];
};
struct ContactScalars {
  int npairs, ntasks, ncells, iterations;
  int overflow;  // tasks beyond the capacity were dropped
  int capped;    // the solve stopped at the sweep cap
};

// Sample-boundary grid (all sample boundaries of a scene in one sorted set).
template <class R>
struct SampleGrid {
  const R4<R>* xb;   // {x,y,z,V_b} sorted
  const R4<R>* vb;   // {vx,vy,vz,-}
  const uint32_t* bid;
  const uint32_t* orig;
  const uint32_t* start;  // bucket starts, T+2 entries
  uint32_t mask;
};

}  // namespace sph
