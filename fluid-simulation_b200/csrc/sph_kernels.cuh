// CUDA kernels of the SPH step engine (sm_100a). One thread per particle;
// neighbor lists are stored warp-tiled (see nbr_slot): the 32 particles of a
// warp own one contiguous block, and each lane reads four consecutive
// neighbors with one 128-bit load, so a warp streams its lists as 512-byte
// coalesced, page-local reads. Gathered neighbor state comes through L1/L2
// because the cell sort keeps spatial neighbors close in memory.
//
// Reference functions each kernel restates (paths under simulation_lib/src/):
//   k_integrate_key      integration_schemes/euler_cromer.rs:12-25,
//                        take_predicted.rs:14-27, sph/mod.rs:674-699 (disable,
//                        max speed), spatial_hashing.rs:27-46 (cells)
//   k_sort_*             spatial_hashing.rs:27-37 (populate) as a counting sort
//   k_neighbors_density  spatial_hashing.rs:75-158, neighbor_search/mod.rs:118-155,
//                        sph/quantities.rs:14-61 (get_volume)
//   k_sample_aggregate   boundary_handling/static_sample_boundary.rs:157-168
//   k_vm_sample          boundary_handling/volume_map_boundary.rs:1259-1424,
//                        utilities/discretization.rs:437-557
//   k_accel              sph/non_pressure_accelerations.rs:19-185,
//                        pressure_solver/mod.rs:90-195, sesph.rs:31-67
//   k_iisph_*            pressure_solver/iisph.rs:117-560,
//                        iisph_optimized_source_term.rs:53-217
//   k_body_*             boundary_handling/rigid_body_motion.rs:135-201
//   k_quantity_at        sph/mod.rs:241-341, sph/quantities.rs:14-330
#pragma once

#include <cfloat>
#include <cmath>

#include "sph_engine.cuh"

namespace sph {

// ---------------------------------------------------------------------------
// Reductions: fixed-order block reductions and last-block completion so the
// result does not depend on scheduling.
// ---------------------------------------------------------------------------
__device__ __forceinline__ double warp_sum(double v) {
  for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
  return v;
}
__device__ __forceinline__ double block_sum(double v, double* sh) {
  v = warp_sum(v);
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  if (lane == 0) sh[w] = v;
  __syncthreads();
  double t = 0;
  if (w == 0) {
    t = lane < (int)(blockDim.x >> 5) ? sh[lane] : 0.0;
    t = warp_sum(t);
  }
  __syncthreads();
  return t;  // valid in thread 0
}

// Sum of per-block partials in a fixed order, run by the last block to finish.
// Returns true in thread 0 of that block with *total set.
__device__ __forceinline__ bool last_block_total(double block_value, double* partials,
                                                 unsigned int* counter, double* total,
                                                 double* sh) {
  __shared__ bool is_last;
  if (threadIdx.x == 0) {
    partials[blockIdx.x] = block_value;
    __threadfence();
    unsigned t = atomicAdd(counter, 1u);
    is_last = (t == gridDim.x - 1);
  }
  __syncthreads();
  if (!is_last) return false;
  __threadfence();
  double s = 0;
  for (unsigned b = threadIdx.x; b < gridDim.x; b += blockDim.x) s += ((volatile double*)partials)[b];
  s = block_sum(s, sh);
  if (threadIdx.x == 0) {
    *total = s;
    *counter = 0;
  }
  return threadIdx.x == 0;
}

// ---------------------------------------------------------------------------
// Rigid-body helpers (f64), nalgebra semantics (rigid_body_motion.rs)
// ---------------------------------------------------------------------------
__device__ __forceinline__ void qrot(const double q[4], const double v[3], double out[3]) {
  // t = 2 (q.v x v); out = v + w t + q.v x t
  double tx = 2.0 * (q[2] * v[2] - q[3] * v[1]);
  double ty = 2.0 * (q[3] * v[0] - q[1] * v[2]);
  double tz = 2.0 * (q[1] * v[1] - q[2] * v[0]);
  double cx = q[2] * tz - q[3] * ty, cy = q[3] * tx - q[1] * tz, cz = q[1] * ty - q[2] * tx;
  out[0] = (tx * q[0] + cx) + v[0];
  out[1] = (ty * q[0] + cy) + v[1];
  out[2] = (tz * q[0] + cz) + v[2];
}
__device__ __forceinline__ void body_world_to_local(const Body& b, const double p[3], double out[3]) {
  double d[3] = {p[0] - b.com[0], p[1] - b.com[1], p[2] - b.com[2]};
  double qi[4] = {b.q[0], -b.q[1], -b.q[2], -b.q[3]};
  qrot(qi, d, out);
}
__device__ __forceinline__ void body_velocity_at(const Body& b, const double p[3], double out[3]) {
  double r[3] = {p[0] - b.com[0], p[1] - b.com[1], p[2] - b.com[2]};
  out[0] = b.v[0] + (b.omega[1] * r[2] - b.omega[2] * r[1]);
  out[1] = b.v[1] + (b.omega[2] * r[0] - b.omega[0] * r[2]);
  out[2] = b.v[2] + (b.omega[0] * r[1] - b.omega[1] * r[0]);
}

// ---------------------------------------------------------------------------
// 1. integrate + cell key + bucket histogram (+ disable test, max speed)
// ---------------------------------------------------------------------------
// mode: 0 EulerCromer, 1 TakePredicted, 2 no integration (initial update)
template <class R>
__global__ void __launch_bounds__(kBlock) k_integrate_key(
    Scalars* __restrict__ sc, R4<R>* __restrict__ pos, R4<R>* __restrict__ vel,
    const R4<R>* __restrict__ acc, const R4<R>* __restrict__ xint, const R4<R>* __restrict__ vint,
    int mode, uint32_t* __restrict__ key, uint32_t* __restrict__ slot,
    uint32_t* __restrict__ count, StepParams<R> P) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  const int n = sc->n;
  double speed = 0.0;
  if (i < n) {
    R4<R> x = pos[i], v = vel[i];
    if (mode == 0) {
      const R dt = (R)sc->dt;
      const R4<R> a = acc[i];
      v.x = v.x + dt * a.x; v.y = v.y + dt * a.y; v.z = v.z + dt * a.z;
      x.x = x.x + dt * v.x; x.y = x.y + dt * v.y; x.z = x.z + dt * v.z;
      pos[i] = x;
      vel[i] = v;
    } else if (mode == 1) {
      const R m = v.w;
      x = xint[i];
      v = vint[i];
      v.w = m;
      pos[i] = x;
      vel[i] = v;
    }
    uint32_t k;
    if ((double)x.z < P.disable_below) {
      k = P.T;
      atomicAdd(&sc->n_below, 1);
    } else {
      k = morton_key(cell_coord((double)x.x, P.range), cell_coord((double)x.y, P.range),
                     cell_coord((double)x.z, P.range), P.mask);
      const double vx = v.x, vy = v.y, vz = v.z;
      speed = sqrt((vx * vx + vy * vy) + vz * vz);
    }
    key[i] = k;
    slot[i] = atomicAdd(&count[k], 1u);
  }
  // block max of the speed (non-negative doubles order like their bit patterns)
  unsigned long long bits = (unsigned long long)__double_as_longlong(speed);
  for (int o = 16; o > 0; o >>= 1) {
    unsigned long long ob = __shfl_down_sync(0xffffffffu, bits, o);
    bits = ob > bits ? ob : bits;
  }
  __shared__ unsigned long long smax[kBlock / 32];
  if ((threadIdx.x & 31) == 0) smax[threadIdx.x >> 5] = bits;
  __syncthreads();
  if (threadIdx.x == 0) {
    unsigned long long m = 0;
    for (int w = 0; w < (int)(blockDim.x >> 5); ++w) m = smax[w] > m ? smax[w] : m;
    if (m) atomicMax(&sc->max_speed, m);
  }
}

// Step prologue: active count and the CFL time increment (sph/mod.rs:825-829).
template <class R>
__global__ void k_prologue(Scalars* sc, StepParams<R> P, int accumulate_time) {
  sc->n_active = sc->n - sc->n_below;
  // simulated time of a CFL step advances by the increment it integrated with
  // (the one chosen by the previous update); graph-captured steps keep it here
  if (accumulate_time) sc->time_acc += sc->dt;
  if (P.cfl) {
    const double ms = __longlong_as_double((long long)sc->max_speed);
    const double c = P.cfl_number * P.spacing / ms;  // +inf at rest
    sc->dt = fmin(P.dt_max, c);
  }
  sc->max_nbrs = 0;
  sc->max_bnbrs = 0;
  sc->max_halo = 0;
  sc->vm_near = 0;
  sc->iterations = 0;
  sc->iterations_eqs1 = 0;
  sc->converged = 0;
  sc->err = INFINITY;
  sc->status = 0;
}

// ---------------------------------------------------------------------------
// 2. exclusive scan of bucket counts (3 phases); clears the counts for reuse
// ---------------------------------------------------------------------------
constexpr int kScanItems = 8;
constexpr int kScanTile = kBlock * kScanItems;

__device__ __forceinline__ uint32_t block_excl_scan_u32(uint32_t v, uint32_t* sh, uint32_t* total) {
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  uint32_t x = v;
  for (int o = 1; o < 32; o <<= 1) {
    uint32_t y = __shfl_up_sync(0xffffffffu, x, o);
    if (lane >= o) x += y;
  }
  if (lane == 31) sh[w] = x;
  __syncthreads();
  if (w == 0) {
    uint32_t s = lane < (int)(blockDim.x >> 5) ? sh[lane] : 0;
    for (int o = 1; o < 32; o <<= 1) {
      uint32_t y = __shfl_up_sync(0xffffffffu, s, o);
      if (lane >= o) s += y;
    }
    sh[lane] = s;
  }
  __syncthreads();
  uint32_t base = w > 0 ? sh[w - 1] : 0;
  if (total) *total = sh[(blockDim.x >> 5) - 1];
  __syncthreads();
  return base + x - v;
}

// A thread's kScanItems consecutive counts: two 16-byte loads when they lie
// inside [0, m) (the arrays are 16-byte aligned and base is a multiple of 8).
static_assert(kScanItems == 8, "two uint4 per thread");
__device__ __forceinline__ void scan_load8(const uint32_t* __restrict__ in, int base, int m, uint32_t v[8]) {
  if (base + 8 <= m) {
    const uint4 a = __ldcs(reinterpret_cast<const uint4*>(in + base));
    const uint4 b = __ldcs(reinterpret_cast<const uint4*>(in + base) + 1);
    v[0] = a.x; v[1] = a.y; v[2] = a.z; v[3] = a.w; v[4] = b.x; v[5] = b.y; v[6] = b.z; v[7] = b.w;
  } else {
#pragma unroll
    for (int k = 0; k < 8; ++k) v[k] = base + k < m ? in[base + k] : 0u;
  }
}

__global__ void __launch_bounds__(kBlock) k_scan_tiles(const uint32_t* __restrict__ in, int m,
                                                      uint32_t* __restrict__ tile_sums) {
  __shared__ uint32_t sh[32];
  const int base = blockIdx.x * kScanTile + threadIdx.x * kScanItems;
  uint32_t v[kScanItems];
  scan_load8(in, base, m, v);
  uint32_t s = 0;
#pragma unroll
  for (int k = 0; k < kScanItems; ++k) s += v[k];
  uint32_t total;
  block_excl_scan_u32(s, sh, &total);
  if (threadIdx.x == 0) tile_sums[blockIdx.x] = total;
}

__global__ void __launch_bounds__(1024) k_scan_tile_sums(uint32_t* __restrict__ tile_sums, int ntiles) {
  __shared__ uint32_t sh[32];
  // each thread owns a contiguous run of tiles
  const int per = (ntiles + blockDim.x - 1) / blockDim.x;
  const int b = threadIdx.x * per;
  uint32_t s = 0;
  for (int k = 0; k < per; ++k) s += b + k < ntiles ? tile_sums[b + k] : 0u;
  uint32_t run = block_excl_scan_u32(s, sh, nullptr);
  for (int k = 0; k < per; ++k)
    if (b + k < ntiles) {
      uint32_t t = tile_sums[b + k];
      tile_sums[b + k] = run;
      run += t;
    }
}

__global__ void __launch_bounds__(kBlock) k_scan_apply(uint32_t* __restrict__ in, int m,
                                                      const uint32_t* __restrict__ tile_sums,
                                                      uint32_t* __restrict__ out) {
  __shared__ uint32_t sh[32];
  const int base = blockIdx.x * kScanTile + threadIdx.x * kScanItems;
  uint32_t v[kScanItems];
  scan_load8(in, base, m, v);
  uint32_t s = 0;
#pragma unroll
  for (int k = 0; k < kScanItems; ++k) s += v[k];
  uint32_t run = block_excl_scan_u32(s, sh, nullptr) + tile_sums[blockIdx.x];
  if (base + 8 <= m) {
    uint32_t o[8];
#pragma unroll
    for (int k = 0; k < 8; ++k) {
      o[k] = run;
      run += v[k];
    }
    uint4* po = reinterpret_cast<uint4*>(out + base);
    po[0] = make_uint4(o[0], o[1], o[2], o[3]);
    po[1] = make_uint4(o[4], o[5], o[6], o[7]);
    uint4* pz = reinterpret_cast<uint4*>(in + base);  // counts are rebuilt by the next histogram
    pz[0] = make_uint4(0u, 0u, 0u, 0u);
    pz[1] = make_uint4(0u, 0u, 0u, 0u);
  } else {
#pragma unroll
    for (int k = 0; k < kScanItems; ++k)
      if (base + k < m) {
        out[base + k] = run;
        run += v[k];
        in[base + k] = 0u;
      }
  }
}

// ---------------------------------------------------------------------------
// 3. scatter, in-bucket ordering by reference index, gather
// ---------------------------------------------------------------------------
__global__ void __launch_bounds__(kBlock) k_scatter(const int* __restrict__ n_ptr,
                                                   const uint32_t* __restrict__ key,
                                                   const uint32_t* __restrict__ slot,
                                                   const uint32_t* __restrict__ start,
                                                   uint32_t* __restrict__ perm) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= *n_ptr) return;
  perm[start[key[i]] + slot[i]] = (uint32_t)i;
}

// The first slot of every bucket orders the bucket's entries by `order`
// (the reference index), which makes the sorted order independent of the
// atomic slot assignment.
__global__ void __launch_bounds__(kBlock) k_bucket_order(const int* __restrict__ n_ptr,
                                                        const uint32_t* __restrict__ key,
                                                        const uint32_t* __restrict__ start,
                                                        const uint32_t* __restrict__ order,
                                                        uint32_t* __restrict__ perm) {
  const int d = blockIdx.x * blockDim.x + threadIdx.x;
  if (d >= *n_ptr) return;
  const uint32_t k = key[perm[d]];
  const uint32_t b = start[k];
  if ((uint32_t)d != b) return;
  const uint32_t e = start[k + 1];
  for (uint32_t a = b + 1; a < e; ++a) {
    const uint32_t pa = perm[a];
    const uint32_t oa = order[pa];
    uint32_t c = a;
    while (c > b) {
      const uint32_t pc = perm[c - 1];
      if (order[pc] <= oa) break;
      perm[c] = pc;
      --c;
    }
    perm[c] = pa;
  }
}

template <class R>
__global__ void __launch_bounds__(kBlock) k_gather_particles(
    const int* __restrict__ n_ptr, const uint32_t* __restrict__ perm,
    const R4<R>* __restrict__ pos, const R4<R>* __restrict__ vel, const uint32_t* __restrict__ ref,
    const uint32_t* __restrict__ fid, R4<R>* __restrict__ pos2, R4<R>* __restrict__ vel2,
    uint32_t* __restrict__ ref2, uint32_t* __restrict__ fid2) {
  const int d = blockIdx.x * blockDim.x + threadIdx.x;
  if (d >= *n_ptr) return;
  const uint32_t j = perm[d];
  pos2[d] = pos[j];
  vel2[d] = vel[j];
  ref2[d] = ref[j];
  fid2[d] = fid[j];
}

// boundary samples: key + histogram (no integration)
template <class R>
__global__ void __launch_bounds__(kBlock) k_sample_key(const int* __restrict__ n_ptr,
                                                      const R4<R>* __restrict__ xb,
                                                      uint32_t* __restrict__ key,
                                                      uint32_t* __restrict__ slot,
                                                      uint32_t* __restrict__ count, double range,
                                                      uint32_t mask) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= *n_ptr) return;
  const R4<R> x = xb[i];
  const uint32_t k = morton_key(cell_coord((double)x.x, range), cell_coord((double)x.y, range),
                                cell_coord((double)x.z, range), mask);
  key[i] = k;
  slot[i] = atomicAdd(&count[k], 1u);
}

template <class R>
__global__ void __launch_bounds__(kBlock) k_gather_samples(
    const int* __restrict__ n_ptr, const uint32_t* __restrict__ perm,
    const R4<R>* __restrict__ xb, const R4<R>* __restrict__ vb, const uint32_t* __restrict__ bid,
    const uint32_t* __restrict__ orig, R4<R>* __restrict__ xb2, R4<R>* __restrict__ vb2,
    uint32_t* __restrict__ bid2, uint32_t* __restrict__ orig2) {
  const int d = blockIdx.x * blockDim.x + threadIdx.x;
  if (d >= *n_ptr) return;
  const uint32_t j = perm[d];
  xb2[d] = xb[j];
  vb2[d] = vb[j];
  bid2[d] = bid[j];
  orig2[d] = orig[j];
}

// ---------------------------------------------------------------------------
// 4. fluid neighbor lists + volume (fused), block halos
//
// The particles of one block (kBlock consecutive particles in bucket order)
// find their neighbors in the union of the 27-bucket stencils of their
// cells: the block's halo. Because buckets are contiguous in memory and the
// halo is kept in ascending bucket key order, the halo is a short list of
// runs of consecutive particle indices (halo_idx, ascending). Neighbor lists
// hold 16-bit positions in the block's halo. The passes over neighbors copy
// the halo's records into shared memory once per launch (ordered loads of
// those runs) and gather from there; a block whose halo does not fit the
// shared-memory capacity gathers through halo_idx from global memory.
//
// Neighbor-list layout: particle i = 32*t + lane keeps its k-th neighbor at
//   ((t * K/4 + k/4) * 32 + lane) * 4 + k % 4      (K a multiple of 4)
// i.e. tile-major, then groups of four neighbors, then lane, so a warp reads
// the next four neighbors of all its lanes as one 256-byte coalesced load.
__device__ __forceinline__ size_t nbr_slot(int i, int k, int K) {
  const size_t t = (size_t)(i >> 5), lane = (size_t)(i & 31);
  return ((t * (size_t)(K >> 2) + (size_t)(k >> 2)) * 32 + lane) * 4 + (size_t)(k & 3);
}

constexpr int kHaloKeys = 8192;            // >= 27 * kBlock stencil keys, a power of two
static_assert(kHaloKeys >= 27 * kBlock, "the sort buffer must hold the stencil keys of a full block");
constexpr uint32_t kNoKey = 0xffffffffu;
constexpr size_t kSearchSmem = kHaloKeys * (sizeof(uint32_t) + sizeof(uint16_t));

// Neighbor lists of one step and the block halos they index.
struct NbrArgs {
  const uint16_t* nbr;   // halo positions, layout of nbr_slot
  const uint32_t* ncnt;  // neighbors per particle (self excluded)
  const uint32_t* hidx;  // [blocks][hcap] halo particle indices
  const uint32_t* hn;    // [blocks] halo sizes
  int K;                 // list capacity per particle
  int hcap;              // halo table capacity per block
  int hs;                // halo records a launch stages in shared memory
  int ahead = 0;         // sweep passes: blocks resident at once (L2 prefetch distance), 0 = none
};

// L2 prefetch for the block one wave ahead (block b + ahead runs on the slot
// this block frees, about one block lifetime later): its particles' records,
// the first list groups of its warps and its halo indices, so that its start
// reads from L2 instead of DRAM.
__device__ __forceinline__ void prefetch_l2(const void* p) {
  asm volatile("prefetch.global.L2 [%0];\n" ::"l"(p));
}
__device__ __forceinline__ void prefetch_lines(const void* p, size_t bytes) {
  const char* c = static_cast<const char*>(p);
  for (size_t o = (size_t)threadIdx.x * 128; o < bytes; o += (size_t)kBlock * 128) prefetch_l2(c + o);
}
constexpr int kPrefetchGroups = 10;     // list groups per warp (about 36 neighbors)
constexpr int kPrefetchHalo = 1408;     // halo indices (the typical halo of a block)
// (m: the block's particles; its warps beyond them hold no lists)
__device__ __forceinline__ void prefetch_block_lists(const NbrArgs& N, int b, int m) {
  const int G = min(N.K >> 2, kPrefetchGroups);
  const char* base = reinterpret_cast<const char*>(N.nbr + nbr_slot(b * kBlock, 0, N.K));
  const size_t warp_bytes = (size_t)(N.K >> 2) * 256;
  for (int q = threadIdx.x; q < ((m + 31) >> 5) * G * 2; q += kBlock)
    prefetch_l2(base + (size_t)(q / (2 * G)) * warp_bytes + (size_t)(q % (2 * G)) * 128);
  prefetch_lines(N.hidx + (size_t)b * N.hcap, (size_t)min(N.hcap, kPrefetchHalo) * sizeof(uint32_t));
}
// The prefetch of a neighbor pass: the per-particle streams it reads (and
// the neighbor counts) for block blockIdx.x + N.ahead, its lists and halo.
template <class... T>
__device__ __forceinline__ void prefetch_ahead(const NbrArgs& N, int n, const T*... streams) {
  if (N.ahead <= 0) return;
  const int b = blockIdx.x + N.ahead;
  if (b * kBlock >= n) return;
  const int i0 = b * kBlock, m = min(kBlock, n - i0);
  (prefetch_lines(streams + i0, (size_t)m * sizeof(T)), ...);
  prefetch_lines(N.ncnt + i0, (size_t)m * sizeof(uint32_t));
  prefetch_block_lists(N, b, m);
}

// The block's halo: its particle indices, its size and whether the launch
// copies its records to shared memory.
struct HaloView {
  const uint32_t* idx;
  int size;
  bool staged;
};
__device__ __forceinline__ HaloView halo_view(const NbrArgs& N) {
  HaloView h;
  h.idx = N.hidx + (size_t)blockIdx.x * (size_t)N.hcap;
  h.size = min((int)N.hn[blockIdx.x], N.hcap);
  h.staged = h.size <= N.hs;
  return h;
}

// Asynchronous global -> shared copies (cp.async): the records travel without
// passing through registers, so every copy a thread issues is in flight at
// once; stage_done() waits for this thread's copies and then for the block.
template <class T>
__device__ __forceinline__ void async_copy(T* smem_dst, const T* gsrc) {
  static_assert(sizeof(T) == 4 || sizeof(T) == 8 || sizeof(T) % 16 == 0, "cp.async moves 4, 8 or 16 bytes");
  const uint32_t d = (uint32_t)__cvta_generic_to_shared(smem_dst);
  if constexpr (sizeof(T) % 16 == 0) {
#pragma unroll
    for (int o = 0; o < (int)sizeof(T); o += 16)
      asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(d + o),
                   "l"(reinterpret_cast<const char*>(gsrc) + o) : "memory");
  } else {
    asm volatile("cp.async.ca.shared.global [%0], [%1], %2;\n" ::"r"(d), "l"(gsrc), "n"(sizeof(T)) : "memory");
  }
}
__device__ __forceinline__ void stage_done() {
  asm volatile("cp.async.wait_all;\n" ::: "memory");
  __syncthreads();
}

// Programmatic dependent launch: a kernel launched with programmatic stream
// serialization may start while the kernel before it finishes its last wave.
// grid_dep_wait() returns once that kernel has completed and its writes are
// visible; everything before it may read only data the earlier kernel does
// not write. grid_dep_release() lets the next kernel start launching (once
// every block of this grid has started). Both are no-ops in a plain launch.
__device__ __forceinline__ void grid_dep_wait() { asm volatile("griddepcontrol.wait;\n" ::: "memory"); }
__device__ __forceinline__ void grid_dep_release() { asm volatile("griddepcontrol.launch_dependents;\n" ::: "memory"); }

// Copies the block's halo records to shared memory: copy(l, g) moves the
// record of particle g to position l. Four halo indices per thread are read
// at a time, then their records are requested.
template <class F>
__device__ __forceinline__ void stage_halo(const HaloView& H, F&& copy) {
  for (int l0 = threadIdx.x; l0 < H.size; l0 += 4 * kBlock) {
    uint32_t g[4];
#pragma unroll
    for (int u = 0; u < 4; ++u) {
      const int l = l0 + u * kBlock;
      g[u] = l < H.size ? __ldg(H.idx + l) : 0u;
    }
#pragma unroll
    for (int u = 0; u < 4; ++u) {
      const int l = l0 + u * kBlock;
      if (l < H.size) copy(l, g[u]);
    }
  }
}
// stage_halo in two steps for the sweep passes: halo_first() reads the
// first batch of halo indices (fixed during a solve, so before the grid
// dependency wait), stage_halo_from() requests the records and the rest.
struct HaloFirst {
  uint32_t g[4];
};
__device__ __forceinline__ HaloFirst halo_first(const HaloView& H) {
  HaloFirst f;
#pragma unroll
  for (int u = 0; u < 4; ++u) {
    const int l = threadIdx.x + u * kBlock;
    f.g[u] = H.staged && l < H.size ? __ldg(H.idx + l) : 0u;
  }
  return f;
}
template <class F>
__device__ __forceinline__ void stage_halo_from(const HaloView& H, const HaloFirst& f, F&& copy) {
  if (!H.staged) return;
#pragma unroll
  for (int u = 0; u < 4; ++u) {
    const int l = threadIdx.x + u * kBlock;
    if (l < H.size) copy(l, f.g[u]);
  }
  for (int l0 = threadIdx.x + 4 * kBlock; l0 < H.size; l0 += 4 * kBlock) {
    uint32_t g[4];
#pragma unroll
    for (int u = 0; u < 4; ++u) {
      const int l = l0 + u * kBlock;
      g[u] = l < H.size ? __ldg(H.idx + l) : 0u;
    }
#pragma unroll
    for (int u = 0; u < 4; ++u) {
      const int l = l0 + u * kBlock;
      if (l < H.size) copy(l, g[u]);
    }
  }
}

template <class R>
__device__ __forceinline__ void kahan_add(R& s, R& c, R t) {
  const R y = t - c;
  const R u = s + y;
  c = (u - s) - y;
  s = u;
}

// The 27 stencil bucket keys of cell (cx,cy,cz), ascending (= memory order)
// when `sorted`, else in stencil order.
__device__ __forceinline__ void stencil_keys(int cx, int cy, int cz, uint32_t mask, int sorted, uint32_t keys[27]) {
#pragma unroll
  for (int q = 0; q < 27; ++q) keys[q] = morton_key(cx + (q % 3) - 1, cy + (q / 3) % 3 - 1, cz + q / 9 - 1, mask);
  if (sorted) {
#pragma unroll
    for (int pass = 0; pass < 27; ++pass) {
#pragma unroll
      for (int q = pass & 1; q + 1 < 27; q += 2) {
        const uint32_t a = keys[q], b = keys[q + 1];
        keys[q] = min(a, b);
        keys[q + 1] = max(a, b);
      }
    }
  }
}

constexpr int kHashSlots = 4096;   // halo bucket set of a block (hash path)
constexpr int kHashElems = 3072;   // stencil keys the hash path takes (27 per cell)
__device__ __forceinline__ uint32_t hash_slot(uint32_t k) { return (k * 0x9E3779B1u) >> 20; }  // 12 bits

// Writes a neighbor list in whole groups of four 16-bit halo positions (one
// 8-byte store per group instead of one 2-byte store per neighbor); the last
// group is completed with the particle's own position.
struct ListWriter {
  uint2* groups;  // this particle's group 0; group g sits 32 uint2 further
  int cap;        // list capacity (a multiple of four)
  uint32_t g0 = 0, g1 = 0;
  __device__ __forceinline__ void add(int cnt, uint32_t l) {
    const int q = cnt & 3;
    if (q < 2) g0 = q == 0 ? l : (g0 | (l << 16));
    else g1 = q == 2 ? l : (g1 | (l << 16));
    if (q == 3 && cnt < cap) groups[(size_t)(cnt >> 2) * 32] = make_uint2(g0, g1);
  }
  __device__ __forceinline__ void finish(int cnt, uint32_t self) {
    if (cnt >= cap || (cnt & 3) == 0) return;
    for (int k = cnt; (k & 3) != 0; ++k) add(k, self);
  }
};

template <class R>
__global__ void __launch_bounds__(kBlock) k_neighbors_density(
    Scalars* __restrict__ sc, const R4<R>* __restrict__ pos, const uint32_t* __restrict__ start,
    R4<R>* __restrict__ xv, uint16_t* __restrict__ nbr, uint32_t* __restrict__ ncnt,
    uint32_t* __restrict__ halo_idx, uint32_t* __restrict__ halo_n, const R* __restrict__ bW,
    int has_boundary, int hcap, StepParams<R> P) {
  extern __shared__ __align__(32) unsigned char dsm[];
  __shared__ int3 s_cell[kBlock];
  __shared__ int s_own[kBlock];      // per cell: own bucket's halo offset - its first particle
  __shared__ uint32_t s_scan[32];
  const int tid = threadIdx.x;
  const int i = blockIdx.x * kBlock + tid;
  const bool active = i < sc->n_active;
  R4<R> xi = R4<R>{R(0), R(0), R(0), R(0)};
  int cx = 0, cy = 0, cz = 0;
  if (active) {
    xi = pos[i];
    cx = cell_coord((double)xi.x, P.range);
    cy = cell_coord((double)xi.y, P.range);
    cz = cell_coord((double)xi.z, P.range);
  }
  s_cell[tid] = make_int3(cx, cy, cz);
  __syncthreads();
  // one head per run of particles in the same cell
  const int3 prev = tid > 0 ? s_cell[tid - 1] : make_int3(0, 0, 0);
  const bool head = active && (tid == 0 || prev.x != cx || prev.y != cy || prev.z != cz);
  uint32_t nheads = 0;
  const uint32_t rank = block_excl_scan_u32(head ? 1u : 0u, s_scan, &nheads);
  const int nk = 27 * (int)nheads;
  uint32_t* hidx = halo_idx + (size_t)blockIdx.x * (size_t)hcap;
  uint32_t H = 0;
  bool miss = false;
  // Per cell, the 27 stencil buckets as (halo offset << 16 | size) spans in
  // ascending key order, in `span_tab` (27 words per cell) when the cells fit,
  // else per particle in `span`.
  const bool hashed = nk <= kHashElems;
  uint32_t* span_tab = nullptr;
  uint32_t span[27];
  if (hashed) {
    // hash path: the set of the cells' stencil buckets in a shared hash table,
    // halo offsets in slot order
    uint32_t* hkey = reinterpret_cast<uint32_t*>(dsm);            // kHashSlots
    uint32_t* hval = hkey + kHashSlots;                            // kHashSlots: offset << 16 | size
    span_tab = hval + kHashSlots;                                  // kHashElems: keys, then spans
    for (int t = tid; t < kHashSlots; t += kBlock) hkey[t] = kNoKey;
    if (head) {
      uint32_t keys[27];
      stencil_keys(cx, cy, cz, P.mask, P.sorted_lists, keys);
#pragma unroll
      for (int q = 0; q < 27; ++q) span_tab[27 * rank + q] = keys[q];
    }
    __syncthreads();
    // Ordered linear probing: a slot keeps the smaller of its key and the
    // one being inserted, and the larger moves on. The table (and so the
    // halo layout) then does not depend on the order the threads insert in
    // (kNoKey, the empty mark, is the largest key).
    for (int e = tid; e < nk; e += kBlock) {
      uint32_t k = span_tab[e];
      uint32_t h = hash_slot(k);
      for (int probe = 0; probe < kHashSlots; ++probe, h = (h + 1) & (kHashSlots - 1)) {
        const uint32_t old = atomicMin(&hkey[h], k);
        if (old == kNoKey || old == k) break;
        if (old > k) k = old;
      }
    }
    __syncthreads();
    // sizes of the distinct buckets, offsets by a block scan over the slots
    constexpr int per = kHashSlots / kBlock;
    uint32_t len[per], tot = 0;
#pragma unroll
    for (int u = 0; u < per; ++u) {
      const uint32_t k = hkey[tid * per + u];
      len[u] = k != kNoKey ? start[k + 1] - start[k] : 0u;
      tot += len[u];
    }
    uint32_t run = block_excl_scan_u32(tot, s_scan, &H);
#pragma unroll
    for (int u = 0; u < per; ++u) {
      const uint32_t k = hkey[tid * per + u];
      miss |= len[u] > 0xffffu;
      hval[tid * per + u] = (min(run, 65535u) << 16) | min(len[u], 65535u);
      if (k != kNoKey) {
        const uint32_t b = start[k];
        for (uint32_t r = 0; r < len[u]; ++r)
          if (run + r < (uint32_t)hcap) hidx[run + r] = b + r;
      }
      run += len[u];
    }
    __syncthreads();
    // each cell's spans: look its keys up in the table
    for (int e = tid; e < nk; e += kBlock) {
      const uint32_t k = span_tab[e];
      uint32_t h = hash_slot(k), v = 0;
      bool found = false;
      for (int probe = 0; probe < kHashSlots; ++probe, h = (h + 1) & (kHashSlots - 1)) {
        const uint32_t kk = hkey[h];
        if (kk == k) { v = hval[h]; found = true; break; }
        if (kk == kNoKey) break;
      }
      miss |= !found;
      span_tab[e] = v;
    }
    if (head) {
      // own bucket: its offset minus its first particle gives the halo position of i
      const uint32_t own = morton_key(cx, cy, cz, P.mask);
      uint32_t h = hash_slot(own), v = 0;
      for (int probe = 0; probe < kHashSlots; ++probe, h = (h + 1) & (kHashSlots - 1)) {
        const uint32_t kk = hkey[h];
        if (kk == own) { v = hval[h]; break; }
        if (kk == kNoKey) break;
      }
      s_own[rank] = (int)(v >> 16) - (int)start[own];
    }
  } else {
    // general path: bitonic-sorted stencil keys, halo offsets in key order,
    // per-particle lookups by binary search
    uint32_t* skey = reinterpret_cast<uint32_t*>(dsm);                 // sorted stencil keys
    uint16_t* soff = reinterpret_cast<uint16_t*>(skey + kHaloKeys);    // halo offset of each first key
    int S = 32;
    while (S < nk) S <<= 1;
    if (head) {
      uint32_t keys[27];
      stencil_keys(cx, cy, cz, P.mask, 0, keys);
#pragma unroll
      for (int q = 0; q < 27; ++q) skey[27 * rank + q] = keys[q];
    }
    for (int t = nk + tid; t < S; t += kBlock) skey[t] = kNoKey;
    __syncthreads();
    for (int k = 2; k <= S; k <<= 1)
      for (int j = k >> 1; j > 0; j >>= 1) {
        for (int t = tid; t < (S >> 1); t += kBlock) {
          const int a = (t / j) * 2 * j + (t % j), b = a + j;
          const uint32_t ka = skey[a], kb = skey[b];
          if ((ka > kb) == ((a & k) == 0)) {
            skey[a] = kb;
            skey[b] = ka;
          }
        }
        __syncthreads();
      }
    const int per = S >= kBlock ? S / kBlock : 1;
    const int p0 = tid * per;
    uint32_t len = 0;
    for (int q = 0; q < per; ++q) {
      const int p = p0 + q;
      if (p >= S) break;
      const uint32_t k = skey[p];
      if (k != kNoKey && (p == 0 || skey[p - 1] != k)) len += start[k + 1] - start[k];
    }
    uint32_t run = block_excl_scan_u32(len, s_scan, &H);
    for (int q = 0; q < per; ++q) {
      const int p = p0 + q;
      if (p >= S) break;
      const uint32_t k = skey[p];
      if (k != kNoKey && (p == 0 || skey[p - 1] != k)) {
        const uint32_t b = start[k], e = start[k + 1];
        soff[p] = (uint16_t)min(run, 65535u);
        for (uint32_t j = b; j < e; ++j)
          if (run + (j - b) < (uint32_t)hcap) hidx[run + (j - b)] = j;
        run += e - b;
      }
    }
    __syncthreads();
    if (active) {
      uint32_t keys[27];
      stencil_keys(cx, cy, cz, P.mask, P.sorted_lists, keys);
      const uint32_t own = morton_key(cx, cy, cz, P.mask);
#pragma unroll 1
      for (int q = 0; q < 27; ++q) {
        const uint32_t k = keys[q];
        int lo = 0, hi = S;
        while (lo < hi) {
          const int mid = (lo + hi) >> 1;
          if (skey[mid] < k) lo = mid + 1;
          else hi = mid;
        }
        const bool found = lo < S && skey[lo] == k;
        const uint32_t b = start[k], len2 = start[k + 1] - b;
        miss |= !found || len2 > 0xffffu;
        const uint32_t off = found ? (uint32_t)soff[lo] : 0u;
        span[q] = found && len2 <= 0xffffu ? (off << 16) | len2 : 0u;
        if (k == own) s_own[tid] = (int)off - (int)b;
      }
    }
  }
  if (tid == 0) {
    halo_n[blockIdx.x] = H;
    atomicMax(&sc->max_halo, (int)min(H, 0x7fffffffu));
  }
  __syncthreads();  // spans, offsets and halo_idx are complete; the sort / hash buffers are free
  const uint32_t usable = min(H, (uint32_t)hcap);
  // The halo's positions move into the first 32 KB of shared memory when they
  // fit (the cells' span table lies beyond them).
  const bool staged = H <= usable && H <= (uint32_t)(2 * kHashSlots * sizeof(uint32_t) / sizeof(R4<R>));
  R4<R>* s_x = reinterpret_cast<R4<R>*>(dsm);
  if (staged)
    for (uint32_t l = tid; l < H; l += kBlock) s_x[l] = pos[hidx[l]];
  __syncthreads();
  int cnt = 0;
  if (active) {
    if (miss) atomicMax(&sc->max_halo, 0x7fffffff);  // cannot happen: every stencil bucket is in the halo
    const int hr = head ? (int)rank : (int)rank - 1;  // this cell's row of the span table
    const uint32_t* row = hashed ? span_tab + 27 * hr : nullptr;
    const uint32_t own_local = (uint32_t)((hashed ? s_own[hr] : s_own[tid]) + i);
    ListWriter lw;
    lw.groups = reinterpret_cast<uint2*>(nbr + nbr_slot(i, 0, P.K));
    lw.cap = P.K;
    R sum = P.k.cw * R(0.5);  // self: W(0) = alpha/h^3 * 1/2
    R comp = 0;
    if (staged) {
      // pass 1: the strict-range test over all candidates builds the list;
      // in stencil order, a bucket whose cell lies entirely beyond the
      // support radius (with a relative margin, so it only skips particles
      // the test would reject) is passed over
      const R h = (R)P.range;
      const R cut2 = (R)(P.range * P.range * (1.0 + 1e-3));
      const R lox = (R)cx * h, loy = (R)cy * h, loz = (R)cz * h;
#pragma unroll 1
      for (int q = 0; q < 27; ++q) {
        const uint32_t sp = hashed ? row[q] : span[q];
        const uint32_t off = sp >> 16;
        uint32_t len = sp & 0xffffu;
        if (!P.sorted_lists && len) {
          const int ox = q % 3 - 1, oy = (q / 3) % 3 - 1, oz = q / 9 - 1;
          const R ex = ox < 0 ? xi.x - lox : (ox > 0 ? lox + h - xi.x : R(0));
          const R ey = oy < 0 ? xi.y - loy : (oy > 0 ? loy + h - xi.y : R(0));
          const R ez = oz < 0 ? xi.z - loz : (oz > 0 ? loz + h - xi.z : R(0));
          const R dx = fmax(ex, R(0)), dy = fmax(ey, R(0)), dz = fmax(ez, R(0));
          if (dx * dx + dy * dy + dz * dz > cut2) len = 0;
        }
        for (uint32_t r = 0; r < len; ++r) {
          const uint32_t local = off + r;
          const R4<R> xj = s_x[local];
          if (local != own_local && in_range(xi, xj, P.range, P.range2_lo, P.range2_hi)) {
            lw.add(cnt, local);
            ++cnt;
          }
        }
      }
      lw.finish(cnt, own_local);
      // pass 2: the kernel sum over the neighbors, in list order
      const int stored = min(cnt, P.K);
      for (int k0 = 0; k0 < stored; k0 += 4) {
        const uint2 w = lw.groups[(size_t)(k0 >> 2) * 32];
        const uint32_t l[4] = {w.x & 0xffffu, w.x >> 16, w.y & 0xffffu, w.y >> 16};
#pragma unroll
        for (int u = 0; u < 4; ++u) {
          if (k0 + u >= stored) break;
          const R4<R> xj = s_x[l[u]];
          const R rx = xi.x - xj.x, ry = xi.y - xj.y, rz = xi.z - xj.z;
          kahan_add(sum, comp, kernel_w_r2(rx * rx + ry * ry + rz * rz, P.k));
        }
      }
    } else {
#pragma unroll 1
      for (int q = 0; q < 27; ++q) {
        const uint32_t sp = hashed ? row[q] : span[q];
        const uint32_t off = sp >> 16, len = sp & 0xffffu;
        const uint32_t b = len && off < usable ? hidx[off] : 0u;
        for (uint32_t r = 0; r < len; ++r) {
          const uint32_t j = b + r;
          if ((int)j == i) continue;
          const R4<R> xj = pos[j];
          if (!in_range(xi, xj, P.range, P.range2_lo, P.range2_hi)) continue;
          const uint32_t local = off + r;
          lw.add(cnt, local < usable ? local : 0u);
          ++cnt;
          const R rx = xi.x - xj.x, ry = xi.y - xj.y, rz = xi.z - xj.z;
          kahan_add(sum, comp, kernel_w_r2(rx * rx + ry * ry + rz * rz, P.k));
        }
      }
    }
    // The unused slots of the last group of four hold the particle's own halo
    // position: a sweep pass reads whole groups, and the self pair adds zero.
    if (!staged) lw.finish(cnt, own_local < usable ? own_local : 0u);
    R denom = P.V0 * sum;
    if (has_boundary) denom += bW[i];
    const R V = P.V0 / denom;
    xv[i] = R4<R>{xi.x, xi.y, xi.z, V};
    ncnt[i] = (uint32_t)cnt;
  }
  // block max of the neighbor count
  for (int o = 16; o > 0; o >>= 1) cnt = max(cnt, __shfl_down_sync(0xffffffffu, cnt, o));
  if ((threadIdx.x & 31) == 0 && cnt > 0) atomicMax(&sc->max_nbrs, cnt);
}

// Reorders each particle's neighbor list so that, at one list slot, the lanes
// of a warp tend to read different shared-memory banks in the neighbor
// passes: lane j's slot k takes an entry whose halo position is j + k modulo
// 8 when it has one left, else the next residue it has (cyclically). A 16-byte
// staged record at halo position l sits in bank group l mod 8, so the eight
// lanes of one 16-byte load phase then mostly hit eight different groups.
// The list stays the same multiset; its padding slots keep the particle's own
// position. Lists longer than KMAX keep their order.
// RES residues (8: 16-byte records, eight lanes per shared-memory phase; 16:
// also the 8-byte records of the second sweep pass, sixteen lanes per phase).
// Dynamic shared memory: order_lists_smem(KMAX, RES) bytes.
__host__ __device__ constexpr size_t order_lists_smem(int kmax, int res) {
  return (size_t)kmax * kBlock * sizeof(uint16_t) + 2 * (size_t)res * kBlock * sizeof(uint32_t);
}
constexpr int kOrderResidues = 8;
template <int KMAX, int RES>
__global__ void __launch_bounds__(kBlock) k_order_lists(const Scalars* __restrict__ sc, uint16_t* __restrict__ nbr,
                                                       const uint32_t* __restrict__ ncnt, int K) {
  static_assert(RES == 8 || RES == 16, "8 or 16 residues");
  extern __shared__ __align__(32) unsigned char dsm[];
  uint32_t* s_cur = reinterpret_cast<uint32_t*>(dsm);  // per residue r of thread t, at [r * kBlock + t]:
  uint32_t* s_end = s_cur + RES * kBlock;               //   the next slot to read and the end of its entries
  uint16_t* ent = reinterpret_cast<uint16_t*>(s_end + RES * kBlock);  // entry e of thread t at [e * kBlock + t]
  constexpr uint32_t M = RES - 1;
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  const int t = threadIdx.x;
  if (i >= sc->n_active) return;
  const int cnt = min((int)ncnt[i], K);
  if (cnt < 2 || cnt > KMAX) return;
  uint2* groups = reinterpret_cast<uint2*>(nbr + nbr_slot(i, 0, K));
  const int ng = (cnt + 3) >> 2;
#pragma unroll
  for (int r = 0; r < RES; ++r) s_end[r * kBlock + t] = 0;
  // entries per residue
  uint2 last = make_uint2(0u, 0u);
  for (int g = 0; g < ng; ++g) {
    const uint2 w = groups[(size_t)g * 32];
    last = w;
    const uint32_t e[4] = {w.x & 0xffffu, w.x >> 16, w.y & 0xffffu, w.y >> 16};
#pragma unroll
    for (int u = 0; u < 4; ++u)
      if (4 * g + u < cnt) ++s_end[(e[u] & M) * kBlock + t];
  }
  // the entries grouped by residue (list order inside a residue); s_end
  // advances from each residue's first slot to its end
  uint32_t avail = 0, run = 0;
#pragma unroll
  for (int r = 0; r < RES; ++r) {
    const uint32_t c = s_end[r * kBlock + t];
    s_cur[r * kBlock + t] = run;
    s_end[r * kBlock + t] = run;
    if (c) avail |= ((1u << RES) + 1u) << r;  // the mask twice: a rotation is one shift
    run += c;
  }
  for (int g = 0; g < ng; ++g) {
    const uint2 w = groups[(size_t)g * 32];
    const uint32_t e[4] = {w.x & 0xffffu, w.x >> 16, w.y & 0xffffu, w.y >> 16};
#pragma unroll
    for (int u = 0; u < 4; ++u)
      if (4 * g + u < cnt) {
        uint32_t& f = s_end[(e[u] & M) * kBlock + t];
        const uint32_t pos = f;
        ent[pos * kBlock + t] = (uint16_t)e[u];
        f = pos + 1;
      }
  }
  const uint32_t pad[4] = {last.x & 0xffffu, last.x >> 16, last.y & 0xffffu, last.y >> 16};
  uint32_t target = (uint32_t)i & M;  // lane j's slot k wants residue j + k (mod RES)
  for (int g = 0; g < ng; ++g) {
    uint32_t v[4];
#pragma unroll
    for (int u = 0; u < 4; ++u) {
      const int k = 4 * g + u;
      if (k >= cnt) {
        v[u] = pad[u];
        continue;
      }
      // the first residue at or after the target (cyclically) with entries left
      const uint32_t r = (target + (uint32_t)(__ffs(avail >> target) - 1)) & M;
      uint32_t& c = s_cur[r * kBlock + t];
      const uint32_t pos = c;
      v[u] = ent[pos * kBlock + t];
      c = pos + 1;
      if (pos + 1 == s_end[r * kBlock + t]) avail &= ~(((1u << RES) + 1u) << r);
      target = (target + 1) & M;
    }
    groups[(size_t)g * 32] = make_uint2(v[0] | (v[1] << 16), v[2] | (v[3] << 16));
  }
}

// ---------------------------------------------------------------------------
// 5. boundary samples: sample boundaries (sorted sample grid) and volume maps
// ---------------------------------------------------------------------------
// Aggregates over a particle's boundary neighbors b (all boundaries):
//   bW  = sum V_b W_ib                                  (volume)
//   bG  = {sum V_b gradW_ib, sum V_b (v_b . gradW_ib)}  (pressure, source, a_ii)
//   bGu = {sum gradW_ib, -}                             (SESPHwSplitting)
template <class R>
__global__ void __launch_bounds__(kBlock) k_sample_aggregate(
    Scalars* __restrict__ sc, const R4<R>* __restrict__ pos, SampleGrid<R> G,
    R* __restrict__ bW, R4<R>* __restrict__ bG, R4<R>* __restrict__ bGu, StepParams<R> P) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  int cnt = 0;
  if (i < sc->n_active) {
    const R4<R> xi = pos[i];
    const int cx = cell_coord((double)xi.x, P.range), cy = cell_coord((double)xi.y, P.range),
              cz = cell_coord((double)xi.z, P.range);
    R w = 0, wc = 0;
    R gx = 0, gy = 0, gz = 0, gv = 0, ux = 0, uy = 0, uz = 0;
    for (int dz = -1; dz <= 1; ++dz)
      for (int dy = -1; dy <= 1; ++dy)
        for (int dx = -1; dx <= 1; ++dx) {
          const uint32_t k = morton_key(cx + dx, cy + dy, cz + dz, G.mask);
          const uint32_t b = G.start[k], e = G.start[k + 1];
          for (uint32_t s = b; s < e; ++s) {
            const R4<R> xs = G.xb[s];
            if (!in_range(xi, xs, P.range, P.range2_lo, P.range2_hi)) continue;
            ++cnt;
            const R rx = xi.x - xs.x, ry = xi.y - xs.y, rz = xi.z - xs.z;
            R kw, f;
            kernel_w_and_grad(rx * rx + ry * ry + rz * rz, P.k, kw, f);
            kahan_add(w, wc, xs.w * kw);
            const R vf = xs.w * f;
            gx += vf * rx; gy += vf * ry; gz += vf * rz;
            const R4<R> vs = G.vb[s];
            gv += vf * (vs.x * rx + vs.y * ry + vs.z * rz);
            ux += f * rx; uy += f * ry; uz += f * rz;
          }
        }
    bW[i] = w;
    bG[i] = R4<R>{gx, gy, gz, gv};
    bGu[i] = R4<R>{ux, uy, uz, R(0)};
  }
  for (int o = 16; o > 0; o >>= 1) cnt = max(cnt, __shfl_down_sync(0xffffffffu, cnt, o));
  if ((threadIdx.x & 31) == 0 && cnt > 0) atomicMax(&sc->max_bnbrs, cnt);
}

// Serendipity reference nodes (discretization.rs:267-300): lattice offsets and
// node kind (0 corner, 1/2/3 edge along x/y/z) with reference coordinates.
__constant__ double c_ser_ref[32][3];
__constant__ int c_ser_off[32][3];
__constant__ int c_ser_kind[32];

// f64 arithmetic that the compiler may not contract into FMAs, so that the
// field evaluation rounds exactly like the reference's (discretization.rs:
// 437-557 is plain f64 without fused operations): threshold decisions such
// as sd < r, sd <= -r or 0.5 < |grad| < 2 then fall on the same side.
__device__ __forceinline__ double mul_(double a, double b) { return __dmul_rn(a, b); }
__device__ __forceinline__ double add_(double a, double b) { return __dadd_rn(a, b); }
__device__ __forceinline__ double sub_(double a, double b) { return __dsub_rn(a, b); }
__device__ __forceinline__ double div_(double a, double b) { return __ddiv_rn(a, b); }

__device__ bool ser_function(const DevField& F, double px, double py, double pz, double& out) {
  const double p[3] = {px, py, pz};
  long long c[3];
#pragma unroll
  for (int d = 0; d < 3; ++d) {
    const double fi = floor(div_(sub_(p[d], F.xmin[d]), F.dx));
    if (p[d] < F.xmin[d] || p[d] > F.xmax[d]) return false;
    long long idx = (long long)fi;
    c[d] = idx < (long long)F.n[d] - 1 ? idx : (long long)F.n[d] - 1;
  }
  const double o0 = add_(F.xmin[0], mul_((double)c[0], F.dx));
  const double o1 = add_(F.xmin[1], mul_((double)c[1], F.dx));
  const double o2 = add_(F.xmin[2], mul_((double)c[2], F.dx));
  const double xi = sub_(div_(mul_(2.0, sub_(p[0], o0)), F.dx), 1.0);
  const double eta = sub_(div_(mul_(2.0, sub_(p[1], o1)), F.dx), 1.0);
  const double zeta = sub_(div_(mul_(2.0, sub_(p[2], o2)), F.dx), 1.0);
  const double r2 = add_(add_(mul_(xi, xi), mul_(eta, eta)), mul_(zeta, zeta));
  const double e19 = sub_(mul_(9.0, r2), 19.0);
  const long long bx = 3 * c[0], by = 3 * c[1], bz = 3 * c[2];
  double s = 0.0;
  for (int a = 0; a < 32; ++a) {
    const long long idx =
        ((bz + c_ser_off[a][2]) * F.NY + (by + c_ser_off[a][1])) * F.NX + (bx + c_ser_off[a][0]);
    const double v = __ldg(F.nodes + idx);
    if (v != v) return false;  // pruned cell
    const double ax = c_ser_ref[a][0], ay = c_ser_ref[a][1], az = c_ser_ref[a][2];
    const double lx = add_(1.0, mul_(xi, ax)), ly = add_(1.0, mul_(eta, ay)), lz = add_(1.0, mul_(zeta, az));
    double N;
    switch (c_ser_kind[a]) {
      case 0:  // (1/64)(1+xi a)(1+eta b)(1+zeta c)(9 r^2 - 19)
        N = mul_(mul_(mul_(mul_(1.0 / 64.0, lx), ly), lz), e19);
        break;
      case 1:  // (9/64)(1-xi^2)(1+9 xi a)(1+eta b)(1+zeta c)
        N = mul_(mul_(mul_(mul_(9.0 / 64.0, sub_(1.0, mul_(xi, xi))), add_(1.0, mul_(mul_(9.0, xi), ax))), ly), lz);
        break;
      case 2:  // (9/64)(1-eta^2)(1+9 eta b)(1+xi a)(1+zeta c)
        N = mul_(mul_(mul_(mul_(9.0 / 64.0, sub_(1.0, mul_(eta, eta))), add_(1.0, mul_(mul_(9.0, eta), ay))), lx), lz);
        break;
      default:  // (9/64)(1-zeta^2)(1+9 zeta c)(1+xi a)(1+eta b)
        N = mul_(mul_(mul_(mul_(9.0 / 64.0, sub_(1.0, mul_(zeta, zeta))), add_(1.0, mul_(mul_(9.0, zeta), az))), lx), ly);
        break;
    }
    s = add_(s, mul_(v, N));
  }
  out = s;
  return true;
}

__device__ bool ser_gradient(const DevField& F, double px, double py, double pz, double g[3]) {
  const double h = div_(F.dx, 6.0);
  const double h2 = mul_(2.0, h);
  double fp, fm;
  if (!ser_function(F, add_(px, h), py, pz, fp) || !ser_function(F, sub_(px, h), py, pz, fm)) return false;
  g[0] = div_(sub_(fp, fm), h2);
  if (!ser_function(F, px, add_(py, h), pz, fp) || !ser_function(F, px, sub_(py, h), pz, fm)) return false;
  g[1] = div_(sub_(fp, fm), h2);
  if (!ser_function(F, px, py, add_(pz, h), fp) || !ser_function(F, px, py, sub_(pz, h), fm)) return false;
  g[2] = div_(sub_(fp, fm), h2);
  return true;
}

// One volume-map boundary sample per (particle, boundary): x_b = x - n d with
// vol = min(VM, 4/3 pi r^3); stored as vmx = {x_b, vol}, vmv = {v_b, kind}
// where kind 0 = none, 1 = tangent helper x-axis, 2 = helper y-axis.
// Volume-map samples in two kernels: k_vm_near evaluates every particle's
// signed distance (the cheap, light first test of find_boundary_samples) and
// lists the particles within the support radius of some boundary, writing
// the empty result for all others; k_vm_sample then does the full sampling
// for the listed particles only.
template <class R>
__global__ void __launch_bounds__(kBlock) k_vm_near(
    Scalars* __restrict__ sc, const R4<R>* __restrict__ pos, const VMDesc* __restrict__ vms, int nvm,
    const Body* __restrict__ bodies, uint32_t* __restrict__ near_list, R4<R>* __restrict__ vmx,
    R4<R>* __restrict__ vmv, R* __restrict__ bW, R4<R>* __restrict__ bG, R4<R>* __restrict__ bGu,
    StepParams<R> P) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= sc->n_active) return;
  const R4<R> xr = pos[i];
  const double p[3] = {(double)xr.x, (double)xr.y, (double)xr.z};
  bool near = false;
  for (int b = 0; b < nvm && !near; ++b) {
    const VMDesc& D = vms[b];
    double pl[3] = {p[0], p[1], p[2]};
    if (D.body >= 0) body_world_to_local(bodies[D.body], p, pl);
    double sd;
    near = ser_function(D.sdf, pl[0], pl[1], pl[2], sd) && sd < P.range;
  }
  if (near) {
    near_list[atomicAdd(&sc->vm_near, 1u)] = (uint32_t)i;
    return;
  }
  for (int b = 0; b < nvm; ++b) {
    const size_t o = (size_t)b * P.Np + i;
    vmx[o] = R4<R>{R(0), R(0), R(0), R(0)};
    vmv[o] = R4<R>{R(0), R(0), R(0), R(0)};
  }
  bW[i] = R(0);
  bG[i] = R4<R>{R(0), R(0), R(0), R(0)};
  bGu[i] = R4<R>{R(0), R(0), R(0), R(0)};
}

// Normal-mode sample of volume map D for the world-frame point p
// (volume_map_boundary.rs:1287-1330): the signed distance (in the body frame
// for a dynamic map) must be below the search range, the gradient norm inside
// (0.5, 2) and the volume-map value positive (then clamped to the volume of
// the support ball); the sample sits at max(sd + spacing/4, spacing) against
// the normalized gradient, moving with the body's velocity there. Returns
// false, leaving the outputs untouched, when the point has no sample.
__device__ __forceinline__ bool vm_normal_sample(const VMDesc& D, const Body* body, const double p[3],
                                                 double range, double ball, double spacing,
                                                 double xb[3], double vb[3], double& vol) {
  double pl[3] = {p[0], p[1], p[2]};
  if (body) body_world_to_local(*body, p, pl);
  double sd;
  if (!ser_function(D.sdf, pl[0], pl[1], pl[2], sd) || !(sd < range)) return false;
  double g[3];
  if (!ser_gradient(D.sdf, pl[0], pl[1], pl[2], g)) return false;
  if (body) {
    double gw[3];
    qrot(body->q, g, gw);
    g[0] = gw[0]; g[1] = gw[1]; g[2] = gw[2];
  }
  const double gn = __dsqrt_rn(add_(add_(mul_(g[0], g[0]), mul_(g[1], g[1])), mul_(g[2], g[2])));
  double vm;
  if (!(gn > 0.5 && gn < 2.0) || !ser_function(D.vm, pl[0], pl[1], pl[2], vm) || !(vm > 0.0)) return false;
  vol = vm < ball ? vm : ball;
  const double d = fmax(add_(sd, mul_(0.25, spacing)), spacing);
  for (int c = 0; c < 3; ++c) xb[c] = sub_(p[c], mul_(div_(g[c], gn), d));
  if (body) body_velocity_at(*body, xb, vb);
  return true;
}

template <class R>
__global__ void __launch_bounds__(kBlock) k_vm_sample(
    Scalars* __restrict__ sc, const uint32_t* __restrict__ near_list, const R4<R>* __restrict__ pos,
    const VMDesc* __restrict__ vms, int nvm, const Body* __restrict__ bodies, R4<R>* __restrict__ vmx,
    R4<R>* __restrict__ vmv, R* __restrict__ bW, R4<R>* __restrict__ bG, R4<R>* __restrict__ bGu,
    StepParams<R> P) {
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= (int)sc->vm_near) return;
  const int i = (int)near_list[t];
  const R4<R> xr = pos[i];
  const double p[3] = {(double)xr.x, (double)xr.y, (double)xr.z};
  const double range = P.range;
  const double ball = 4.0 / 3.0 * 3.14159265358979323846 * (range * range * range);
  R w = 0, gx = 0, gy = 0, gz = 0, gv = 0, ux = 0, uy = 0, uz = 0;
  for (int b = 0; b < nvm; ++b) {
    const VMDesc& D = vms[b];
    const Body* body = D.body >= 0 ? &bodies[D.body] : nullptr;
    int kind = 0;
    double xb[3] = {0, 0, 0}, vb[3] = {0, 0, 0}, vol = 0;
    if (vm_normal_sample(D, body, p, range, ball, P.spacing, xb, vb, vol)) {
      const double u[3] = {xb[0] - p[0], xb[1] - p[1], xb[2] - p[2]};
      const double un = sqrt((u[0] * u[0] + u[1] * u[1]) + u[2] * u[2]);
      kind = fabs(u[0] / un) > 0.9 ? 2 : 1;
      // aggregates in f64 from the exact sample position
      const double rx = p[0] - xb[0], ry = p[1] - xb[1], rz = p[2] - xb[2];
      const double r2 = (rx * rx + ry * ry) + rz * rz;
      const double rn = sqrt(r2), q = rn / range;
      const double a1 = q < 1.0 ? 1.0 - q : 0.0, a2 = q < 0.5 ? 0.5 - q : 0.0;
      const double alpha = 16.0 / 3.14159265358979323846;
      const double kw = alpha / (range * range * range) * (a1 * a1 * a1 - 4.0 * (a2 * a2 * a2));
      const double f = rn > 0.0 ? alpha / (range * range * range * range) *
                                      (-3.0 * a1 * a1 + 12.0 * a2 * a2) / rn
                                : 0.0;
      w += (R)(vol * kw);
      const double vf = vol * f;
      gx += (R)(vf * rx); gy += (R)(vf * ry); gz += (R)(vf * rz);
      gv += (R)(vf * (vb[0] * rx + vb[1] * ry + vb[2] * rz));
      ux += (R)(f * rx); uy += (R)(f * ry); uz += (R)(f * rz);
    }
    const size_t o = (size_t)b * P.Np + i;
    vmx[o] = R4<R>{(R)xb[0], (R)xb[1], (R)xb[2], (R)vol};
    vmv[o] = R4<R>{(R)vb[0], (R)vb[1], (R)vb[2], (R)kind};
  }
  bW[i] = w;
  bG[i] = R4<R>{gx, gy, gz, gv};
  bGu[i] = R4<R>{ux, uy, uz, R(0)};
}

// ScalarQuantity at evaluation positions (sph/mod.rs:241-341 with the sums
// of quantities.rs:14-330), for sensor planes: one thread per position walks
// the 27 buckets of the fluid grid of the last update (sorted positions and
// volumes `xv`, velocities and masses `vel`, pressures), keeps the
// reference's exact neighbor predicate and sums in f64 whatever the state
// precision. Speed and volume also take the position's boundary samples
// (RequestMode::Normal): the sorted sample grid, or one sample per volume
// map. Quantities: 0 speed |sum v V W|, 1 volume V0 / sum V0 W, 2 density
// sum m W, 3 density error 100 sum_{m < V0} (V0/m - 1) m W (the reference
// passes the masses where the sum takes volumes), 4 pressure sum p V W,
// 5 kinetic energy sum m |v|^2 V W / 2. The result is cast to f32.
template <class R>
__global__ void __launch_bounds__(kBlock) k_quantity_at(
    int quantity, int n_eval, const float* __restrict__ eval, float* __restrict__ out,
    const uint32_t* __restrict__ start, const R4<R>* __restrict__ xv, const R4<R>* __restrict__ vel,
    const R* __restrict__ press, SampleGrid<R> G, const VMDesc* __restrict__ vms, int nvm,
    const Body* __restrict__ bodies, KernelConst<double> kd, double V0, StepParams<R> P) {
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= n_eval) return;
  const double p[3] = {(double)eval[3 * t], (double)eval[3 * t + 1], (double)eval[3 * t + 2]};
  const double h = P.range;
  const int cx = cell_coord(p[0], h), cy = cell_coord(p[1], h), cz = cell_coord(p[2], h);
  double s = 0, sx = 0, sy = 0, sz = 0;
  if (start) {
    for (int dz = -1; dz <= 1; ++dz)
      for (int dy = -1; dy <= 1; ++dy)
        for (int dx = -1; dx <= 1; ++dx) {
          const uint32_t k = morton_key(cx + dx, cy + dy, cz + dz, P.mask);
          const uint32_t e = start[k + 1];
          for (uint32_t j = start[k]; j < e; ++j) {
            const R4<R> xj = xv[j];
            const double qx = (double)xj.x, qy = (double)xj.y, qz = (double)xj.z;
            if (!in_range_exact(p[0], p[1], p[2], qx, qy, qz, h)) continue;
            const double rx = p[0] - qx, ry = p[1] - qy, rz = p[2] - qz;
            const double w = kernel_w_r2<double>((rx * rx + ry * ry) + rz * rz, kd);
            const double V = (double)xj.w;
            if (quantity == 1) { s += V0 * w; continue; }
            const R4<R> vj = vel[j];
            const double vx = (double)vj.x, vy = (double)vj.y, vz = (double)vj.z, m = (double)vj.w;
            switch (quantity) {
              case 0: sx += vx * V * w; sy += vy * V * w; sz += vz * V * w; break;
              case 2: s += m * w; break;
              case 3: if (m < V0) s += (V0 / m - 1.0) * m * w; break;
              case 4: s += (double)press[j] * V * w; break;
              default: s += 0.5 * m * ((vx * vx + vy * vy) + vz * vz) * V * w; break;
            }
          }
        }
  }
  if (quantity <= 1) {
    if (G.start) {
      for (int dz = -1; dz <= 1; ++dz)
        for (int dy = -1; dy <= 1; ++dy)
          for (int dx = -1; dx <= 1; ++dx) {
            const uint32_t k = morton_key(cx + dx, cy + dy, cz + dz, G.mask);
            const uint32_t e = G.start[k + 1];
            for (uint32_t j = G.start[k]; j < e; ++j) {
              const R4<R> xs = G.xb[j];
              const double qx = (double)xs.x, qy = (double)xs.y, qz = (double)xs.z;
              if (!in_range_exact(p[0], p[1], p[2], qx, qy, qz, h)) continue;
              const double rx = p[0] - qx, ry = p[1] - qy, rz = p[2] - qz;
              const double vw = (double)xs.w * kernel_w_r2<double>((rx * rx + ry * ry) + rz * rz, kd);
              if (quantity == 1) {
                s += vw;
              } else {
                const R4<R> vs = G.vb[j];
                sx += (double)vs.x * vw; sy += (double)vs.y * vw; sz += (double)vs.z * vw;
              }
            }
          }
    }
    const double ball = 4.0 / 3.0 * 3.14159265358979323846 * (h * h * h);
    for (int b = 0; b < nvm; ++b) {
      const VMDesc& D = vms[b];
      double xb[3] = {0, 0, 0}, vb[3] = {0, 0, 0}, vol = 0;
      if (!vm_normal_sample(D, D.body >= 0 ? &bodies[D.body] : nullptr, p, h, ball, P.spacing, xb, vb, vol))
        continue;
      const double rx = p[0] - xb[0], ry = p[1] - xb[1], rz = p[2] - xb[2];
      const double vw = vol * kernel_w_r2<double>((rx * rx + ry * ry) + rz * rz, kd);
      if (quantity == 1) {
        s += vw;
      } else {
        sx += vb[0] * vw; sy += vb[1] * vw; sz += vb[2] * vw;
      }
    }
  }
  double val;
  switch (quantity) {
    case 0: val = sqrt((sx * sx + sy * sy) + sz * sz); break;
    case 1: val = V0 / s; break;
    case 3: val = 100.0 * s; break;
    default: val = s; break;
  }
  out[t] = (float)val;
}

// ---------------------------------------------------------------------------
// Boundary iteration helpers used by the acceleration passes
// ---------------------------------------------------------------------------
template <class R>
struct BoundaryArgs {
  int kind;  // 0 none, 1 sample boundaries, 2 volume maps
  SampleGrid<R> grid;
  const R4<R>* vmx;
  const R4<R>* vmv;
  const VMDesc* vms;
  int nvm;
  const Body* bodies;
  int any_dynamic;
  const R* bW;
  const R4<R>* bG;
  const R4<R>* bGu;
  double* body_partials;  // [gridDim][kMaxBodies][6] reaction force/torque partials
  int nbodies;
};

// Calls fn(xb, vb, Vb, body) for every boundary neighbor of the viscosity
// request mode: sample-boundary neighbors, or the 4 tangential volume-map
// samples at x_b +- r/2 t1, x_b +- r/2 t2 (volume_map_boundary.rs:1344-1377).
template <class R, class Fn>
__device__ __forceinline__ void for_each_visc_sample(const BoundaryArgs<R>& B, const R4<R>& xi,
                                                     int i, const StepParams<R>& P, Fn&& fn) {
  if (B.kind == 1) {
    const int cx = cell_coord((double)xi.x, P.range), cy = cell_coord((double)xi.y, P.range),
              cz = cell_coord((double)xi.z, P.range);
    for (int dz = -1; dz <= 1; ++dz)
      for (int dy = -1; dy <= 1; ++dy)
        for (int dx = -1; dx <= 1; ++dx) {
          const uint32_t k = morton_key(cx + dx, cy + dy, cz + dz, B.grid.mask);
          const uint32_t b = B.grid.start[k], e = B.grid.start[k + 1];
          for (uint32_t s = b; s < e; ++s) {
            const R4<R> xs = B.grid.xb[s];
            if (!in_range(xi, xs, P.range, P.range2_lo, P.range2_hi)) continue;
            const R4<R> vs = B.grid.vb[s];
            fn(V3<R>{xs.x, xs.y, xs.z}, V3<R>{vs.x, vs.y, vs.z}, xs.w, (int)B.grid.bid[s]);
          }
        }
  } else if (B.kind == 2) {
    for (int b = 0; b < B.nvm; ++b) {
      const size_t o = (size_t)b * P.Np + i;
      const R4<R> vv = B.vmv[o];
      if (vv.w == R(0)) continue;
      const R4<R> xx = B.vmx[o];
      const V3<R> xb{xx.x, xx.y, xx.z};
      const V3<R> u = xb - V3<R>{xi.x, xi.y, xi.z};
      const V3<R> tmp = vv.w == R(1) ? V3<R>{1, 0, 0} : V3<R>{0, 1, 0};
      V3<R> t1 = cross(u, tmp);
      V3<R> t2 = cross(u, t1);
      t1 = (R(1) / sqrt(dot(t1, t1))) * t1;
      t2 = (R(1) / sqrt(dot(t2, t2))) * t2;
      const R d = R(0.5) * (R)P.range;
      const V3<R> q[4] = {xb + d * t1, xb - d * t1, xb + d * t2, xb - d * t2};
      const int body = B.vms[b].body;
      for (int k = 0; k < 4; ++k) {
        V3<R> vq{0, 0, 0};
        if (body >= 0) {
          const double pq[3] = {(double)q[k].x, (double)q[k].y, (double)q[k].z};
          double vo[3];
          body_velocity_at(B.bodies[body], pq, vo);
          vq = V3<R>{(R)vo[0], (R)vo[1], (R)vo[2]};
        }
        fn(q[k], vq, R(0.25) * xx.w, body);
      }
    }
  }
}

// Calls fn(xb, Vb, body) for every boundary neighbor of the Normal mode.
template <class R, class Fn>
__device__ __forceinline__ void for_each_normal_sample(const BoundaryArgs<R>& B, const R4<R>& xi,
                                                       int i, const StepParams<R>& P, Fn&& fn) {
  if (B.kind == 1) {
    const int cx = cell_coord((double)xi.x, P.range), cy = cell_coord((double)xi.y, P.range),
              cz = cell_coord((double)xi.z, P.range);
    for (int dz = -1; dz <= 1; ++dz)
      for (int dy = -1; dy <= 1; ++dy)
        for (int dx = -1; dx <= 1; ++dx) {
          const uint32_t k = morton_key(cx + dx, cy + dy, cz + dz, B.grid.mask);
          const uint32_t b = B.grid.start[k], e = B.grid.start[k + 1];
          for (uint32_t s = b; s < e; ++s) {
            const R4<R> xs = B.grid.xb[s];
            if (!in_range(xi, xs, P.range, P.range2_lo, P.range2_hi)) continue;
            fn(V3<R>{xs.x, xs.y, xs.z}, xs.w, (int)B.grid.bid[s]);
          }
        }
  } else if (B.kind == 2) {
    for (int b = 0; b < B.nvm; ++b) {
      const size_t o = (size_t)b * P.Np + i;
      if (B.vmv[o].w == R(0)) continue;
      const R4<R> xx = B.vmx[o];
      fn(V3<R>{xx.x, xx.y, xx.z}, xx.w, B.vms[b].body);
    }
  }
}

// Per-block rigid-body force/torque accumulation in f64 (shared memory),
// flushed to per-block partials that a fixed-order kernel reduces.
struct BodyAccum {
  double* sh;  // [kMaxBodies][6]
  __device__ void add(const Body* bodies, int body, const double F[3], const double x[3]) {
    const Body& b = bodies[body];
    const double r[3] = {x[0] - b.com[0], x[1] - b.com[1], x[2] - b.com[2]};
    atomicAdd(&sh[body * 6 + 0], F[0]);
    atomicAdd(&sh[body * 6 + 1], F[1]);
    atomicAdd(&sh[body * 6 + 2], F[2]);
    atomicAdd(&sh[body * 6 + 3], r[1] * F[2] - r[2] * F[1]);
    atomicAdd(&sh[body * 6 + 4], r[2] * F[0] - r[0] * F[2]);
    atomicAdd(&sh[body * 6 + 5], r[0] * F[1] - r[1] * F[0]);
  }
};

__device__ __forceinline__ void body_accum_init(double* sh, int nbodies) {
  for (int t = threadIdx.x; t < nbodies * 6; t += blockDim.x) sh[t] = 0.0;
  __syncthreads();
}
__device__ __forceinline__ void body_accum_flush(double* sh, int nbodies, double* partials) {
  __syncthreads();
  for (int t = threadIdx.x; t < nbodies * 6; t += blockDim.x)
    partials[(size_t)blockIdx.x * kMaxBodies * 6 + t] = sh[t];
}

// ---------------------------------------------------------------------------
// Neighbor gather loop. The halo positions of NB neighbors are fetched first
// (streaming, evict-first 64-bit loads of four 16-bit positions), then the NB
// records are loaded, then consumed, so NB loads are in flight per thread.
// Slots past the count read position 0, which every non-empty halo has.
// ---------------------------------------------------------------------------
// The first D batches of a particle's list, requested ahead of use (a kernel
// can issue them before it waits for its halo staging).
template <int NB, int D = 1>
struct ListHead {
  uint2 g[D][NB / 4];
};
template <int NB, int D = 1>
__device__ __forceinline__ ListHead<NB, D> list_head(const uint16_t* __restrict__ nbr, int K, int i, int cnt) {
  ListHead<NB, D> h;
  const uint2* base = reinterpret_cast<const uint2*>(nbr) + nbr_slot(i, 0, K) / 4;
  const int ngroups = (cnt + 3) >> 2;
#pragma unroll
  for (int d = 0; d < D; ++d)
#pragma unroll
    for (int g = 0; g < NB / 4; ++g) {
      const int gi = d * (NB / 4) + g;
      h.g[d][g] = gi < ngroups ? __ldcs(base + (size_t)gi * 32) : make_uint2(0u, 0u);
    }
  return h;
}

// Visits the neighbors of particle i in batches of NB: while a batch is
// consumed, the list words of the batch D ahead are in flight.
template <int NB, int D, class Load, class Use>
__device__ __forceinline__ void for_each_neighbor(const uint16_t* __restrict__ nbr, int K, int i, int cnt,
                                                  const ListHead<NB, D>& head, Load&& load, Use&& use) {
  static_assert(NB % 4 == 0, "neighbors are read in groups of four");
  // group g of this lane sits 32 uint2 after group g-1
  const uint2* base = reinterpret_cast<const uint2*>(nbr) + nbr_slot(i, 0, K) / 4;
  const int ngroups = (cnt + 3) >> 2;
  uint2 q[D][NB / 4];
#pragma unroll
  for (int d = 0; d < D; ++d)
#pragma unroll
    for (int g = 0; g < NB / 4; ++g) q[d][g] = head.g[d][g];
  for (int k0 = 0; k0 < cnt; k0 += NB) {
    uint2 nxt[NB / 4];
#pragma unroll
    for (int g = 0; g < NB / 4; ++g) {
      const int gi = (k0 + D * NB) / 4 + g;
      nxt[g] = gi < ngroups ? __ldcs(base + (size_t)gi * 32) : make_uint2(0u, 0u);
    }
    uint32_t l[NB];
#pragma unroll
    for (int g = 0; g < NB / 4; ++g) {
      const uint2 w = q[0][g];
      l[4 * g + 0] = k0 + 4 * g + 0 < cnt ? (w.x & 0xffffu) : 0u;
      l[4 * g + 1] = k0 + 4 * g + 1 < cnt ? (w.x >> 16) : 0u;
      l[4 * g + 2] = k0 + 4 * g + 2 < cnt ? (w.y & 0xffffu) : 0u;
      l[4 * g + 3] = k0 + 4 * g + 3 < cnt ? (w.y >> 16) : 0u;
    }
    decltype(load(0u)) d[NB];
#pragma unroll
    for (int u = 0; u < NB; ++u) d[u] = load(l[u]);
#pragma unroll
    for (int u = 0; u < NB; ++u)
      if (k0 + u < cnt) use(d[u]);
#pragma unroll
    for (int e = 0; e + 1 < D; ++e)
#pragma unroll
      for (int g = 0; g < NB / 4; ++g) q[e][g] = q[e + 1][g];
#pragma unroll
    for (int g = 0; g < NB / 4; ++g) q[D - 1][g] = nxt[g];
  }
}
template <int NB, class Load, class Use>
__device__ __forceinline__ void for_each_neighbor(const uint16_t* __restrict__ nbr, int K, int i, int cnt,
                                                  Load&& load, Use&& use) {
  for_each_neighbor<NB, 1>(nbr, K, i, cnt, list_head<NB, 1>(nbr, K, i, cnt), load, use);
}

// Shared-memory layout of staged halo records: arrays of R4 then arrays of R,
// each `hs` records long.
template <class R>
__device__ __forceinline__ R4<R>* staged_vec(unsigned char* dsm, int hs, int which) {
  return reinterpret_cast<R4<R>*>(dsm) + (size_t)which * hs;
}
template <class R>
__device__ __forceinline__ R* staged_scalar(unsigned char* dsm, int hs, int nvec, int which) {
  return reinterpret_cast<R*>(reinterpret_cast<R4<R>*>(dsm) + (size_t)nvec * hs) + (size_t)which * hs;
}

template <class R>
struct XP {  // position+volume and one scalar
  R4<R> x;
  R s;
};
template <class R>
struct XV {  // position+volume and one vector
  R4<R> x;
  R4<R> v;
};
template <class R>
struct SweepList {
  const uint2* p;  // this particle's first group of four; group g sits 32 uint2 further
  int ng;          // groups
  uint2 w0, w1;    // the next two groups, in flight
  __device__ __forceinline__ void begin(const NbrArgs& N, int i, int cnt) {
    p = reinterpret_cast<const uint2*>(N.nbr) + nbr_slot(i, 0, N.K) / 4;
    ng = (cnt + 3) >> 2;
    w0 = ng > 0 ? __ldcs(p) : make_uint2(0u, 0u);
    w1 = ng > 1 ? __ldcs(p + 32) : make_uint2(0u, 0u);
  }
  // the group to use now; requests the one two groups ahead
  __device__ __forceinline__ uint2 next(int g) {
    const uint2 w = w0;
    w0 = w1;
    w1 = g + 2 < ng ? __ldcs(p + (size_t)(g + 2) * 32) : make_uint2(0u, 0u);
    return w;
  }
};

// Visits every slot of a particle's neighbor list in whole groups of four,
// padding included: the unused slots of the last group repeat the particle's
// own halo position, so a pass whose pair term is zero at r = 0 needs no
// per-neighbor count test. The four records of a group are gathered before
// they are used.
template <class R, class Load, class Use>
__device__ __forceinline__ void sweep_groups(SweepList<R>& L, Load&& load, Use&& use) {
  for (int g = 0; g < L.ng; ++g) {
    const uint2 w = L.next(g);
    const auto d0 = load(w.x & 0xffffu);
    const auto d1 = load(w.x >> 16);
    const auto d2 = load(w.y & 0xffffu);
    const auto d3 = load(w.y >> 16);
    use(d0); use(d1); use(d2); use(d3);
  }
}

// ---------------------------------------------------------------------------
// 6. accelerations: gravity + viscosity (+ SESPH pressure) (+ v* = v + dt a)
// ---------------------------------------------------------------------------
// PRESS: 0 none, 1 SESPH state equation from the volume on the fly
template <class R, int PRESS>
__global__ void __launch_bounds__(kBlock) k_accel(
    const Scalars* __restrict__ sc, const R4<R>* __restrict__ xv, const R4<R>* __restrict__ vel,
    NbrArgs N, BoundaryArgs<R> B, R4<R>* __restrict__ acc, R4<R>* __restrict__ vstar,
    R* __restrict__ press, int write_vstar, StepParams<R> P) {
  __shared__ double sh_body[kMaxBodies * 6];
  extern __shared__ __align__(32) unsigned char dsm[];
  const bool bodies = B.any_dynamic != 0;
  if (bodies) body_accum_init(sh_body, B.nbodies);
  const HaloView H = halo_view(N);
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  const bool act = i < sc->n_active;
  SweepList<R> L;  // the list head travels while the halo stages
  L.begin(N, act ? i : 0, act ? min((int)N.ncnt[i], N.K) : 0);
  R4<R>* s_x = staged_vec<R>(dsm, N.hs, 0);
  R4<R>* s_v = staged_vec<R>(dsm, N.hs, 1);
  if (H.staged)
    stage_halo(H, [&](int l, uint32_t g) {
      async_copy(&s_x[l], &xv[g]);
      async_copy(&s_v[l], &vel[g]);
    });
  stage_done();
  if (act) {
    const R4<R> xi = xv[i];
    const R4<R> vi = vel[i];
    const R mi = vi.w, Vi = xi.w;
    R ax, ay, az;
    if (P.gravity_mode == 0) {
      ax = 0; ay = 0; az = R(-9.81);
    } else {
      const R dx = P.gc[0] - xi.x, dy = P.gc[1] - xi.y, dz = P.gc[2] - xi.z;
      const R dist = sqrt(dx * dx + dy * dy + dz * dz + R(1e-4));
      ax = R(9.81) * dx / dist; ay = R(9.81) * dy / dist; az = R(9.81) * dz / dist;
    }
    R pi = 0;
    if (PRESS == 1) pi = P.stiffness * fmax(P.V0 / Vi - R(1), R(0));
    R sx = 0, sy = 0, sz = 0;   // viscosity
    R px = 0, py = 0, pz = 0;   // pressure
    // pair terms are zero at r = 0 (self padding adds nothing)
    auto pair = [&](const XV<R>& d) {
          const R4<R>& xj = d.x;
          const R4<R>& vj = d.v;
          const R rx = xi.x - xj.x, ry = xi.y - xj.y, rz = xi.z - xj.z;
          const R r2 = rx * rx + ry * ry + rz * rz;
          const R f = kernel_grad_factor(r2, P.k);
          const R vr = (vi.x - vj.x) * rx + (vi.y - vj.y) * ry + (vi.z - vj.z) * rz;
          const R s = P.visc_f * xj.w * vr / (r2 + P.eps_visc) * f;
          sx += s * rx; sy += s * ry; sz += s * rz;
          if (PRESS == 1) {
            const R pj = P.stiffness * fmax(P.V0 / xj.w - R(1), R(0));
            const R t = xj.w * (pi + pj) * f;
            px += t * rx; py += t * ry; pz += t * rz;
          }
        };
    if (H.staged)
      sweep_groups(L, [&](uint32_t l) { return XV<R>{s_x[l], s_v[l]}; }, pair);
    else
      sweep_groups(L, [&](uint32_t l) { const uint32_t g = H.idx[l]; return XV<R>{xv[g], vel[g]}; }, pair);
    if (B.kind != 0) {
      BodyAccum acc_b{sh_body};
      for_each_visc_sample<R>(B, xi, i, P, [&](V3<R> xb, V3<R> vb, R Vb, int body) {
        const R rx = xi.x - xb.x, ry = xi.y - xb.y, rz = xi.z - xb.z;
        const R r2 = rx * rx + ry * ry + rz * rz;
        const R f = kernel_grad_factor(r2, P.k);
        const R vr = (vi.x - vb.x) * rx + (vi.y - vb.y) * ry + (vi.z - vb.z) * rz;
        const R s = P.visc_b * Vb * vr / (r2 + P.eps_visc) * f;
        sx += s * rx; sy += s * ry; sz += s * rz;
        if (bodies && body >= 0 && B.bodies[body].dynamic) {
          const double F[3] = {-(double)mi * (double)(s * rx), -(double)mi * (double)(s * ry),
                               -(double)mi * (double)(s * rz)};
          const double xl[3] = {(double)xb.x, (double)xb.y, (double)xb.z};
          acc_b.add(B.bodies, body, F, xl);
        }
      });
      if (PRESS == 1) {
        const R4<R> g = B.bG[i];
        const R c = R(2) * P.gamma_p * pi;  // boundary: 2 gamma V_i V_b p_i gradW / m_i
        px += c * g.x; py += c * g.y; pz += c * g.z;
        if (bodies) {
          for_each_normal_sample<R>(B, xi, i, P, [&](V3<R> xb, R Vb, int body) {
            if (body < 0 || !B.bodies[body].dynamic) return;
            const R rx = xi.x - xb.x, ry = xi.y - xb.y, rz = xi.z - xb.z;
            const R f = kernel_grad_factor(rx * rx + ry * ry + rz * rz, P.k);
            const double c2 = 2.0 * (double)P.gamma_p * (double)Vi * (double)Vb * (double)pi * (double)f;
            const double F[3] = {c2 * rx, c2 * ry, c2 * rz};
            const double xl[3] = {(double)xb.x, (double)xb.y, (double)xb.z};
            acc_b.add(B.bodies, body, F, xl);
          });
        }
      }
    }
    const R vm = Vi / mi;
    ax += sx - vm * px;
    ay += sy - vm * py;
    az += sz - vm * pz;
    acc[i] = R4<R>{ax, ay, az, R(0)};
    if (write_vstar) {
      const R dt = (R)sc->dt;
      vstar[i] = R4<R>{vi.x + dt * ax, vi.y + dt * ay, vi.z + dt * az, mi};  // the mass rides along
    }
    if (PRESS == 1) press[i] = pi;
  }
  if (bodies) body_accum_flush(sh_body, B.nbodies, B.body_partials);
}

// ---------------------------------------------------------------------------
// 7. pressure acceleration from stored pressures (pressure_solver/mod.rs:121-195)
// ---------------------------------------------------------------------------
// MODE: 1 -> acc += accel (reaction forces if mirror)
//       2 -> acc  = accel (reaction forces if mirror)
// (the Jacobi sweep's own pressure accelerations are k_sweep_accel)
template <class R, int MODE>
__global__ void __launch_bounds__(kBlock) k_pressure_accel(
    const Scalars* __restrict__ sc, const R4<R>* __restrict__ xv, const R4<R>* __restrict__ vel,
    const R* __restrict__ press, NbrArgs N, BoundaryArgs<R> B, R4<R>* __restrict__ out, int mirror,
    StepParams<R> P) {
  __shared__ double sh_body[kMaxBodies * 6];
  extern __shared__ __align__(32) unsigned char dsm[];
  const bool bodies = mirror && B.any_dynamic != 0;
  if (bodies) body_accum_init(sh_body, B.nbodies);
  const HaloView H = halo_view(N);
  // this particle's own data and first list batch travel while the halo stages
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  const bool act = i < sc->n_active;
  SweepList<R> L;
  L.begin(N, act ? i : 0, act ? min((int)N.ncnt[i], N.K) : 0);
  R4<R> xi{};
  R mi = 1, pi = 0;
  if (act) {
    xi = xv[i];
    mi = vel[i].w;
    pi = press[i];
  }
  R4<R>* s_x = staged_vec<R>(dsm, N.hs, 0);
  R* s_p = staged_scalar<R>(dsm, N.hs, 1, 0);
  if (H.staged)
    stage_halo(H, [&](int l, uint32_t g) {
      async_copy(&s_x[l], &xv[g]);
      async_copy(&s_p[l], &press[g]);
    });
  stage_done();
  if (act) {
    const R Vi = xi.w;
    R px = 0, py = 0, pz = 0;
    auto pair = [&](const XP<R>& d) {  // zero at r = 0 (self padding)
      const R rx = xi.x - d.x.x, ry = xi.y - d.x.y, rz = xi.z - d.x.z;
      const R f = kernel_grad_factor(rx * rx + ry * ry + rz * rz, P.k);
      const R t = d.x.w * (pi + d.s) * f;
      px += t * rx; py += t * ry; pz += t * rz;
    };
    if (H.staged)
      sweep_groups(L, [&](uint32_t l) { return XP<R>{s_x[l], s_p[l]}; }, pair);
    else
      sweep_groups(L, [&](uint32_t l) { const uint32_t g = H.idx[l]; return XP<R>{xv[g], press[g]}; }, pair);
    if (B.kind != 0) {
      const R4<R> g = B.bG[i];
      const R c = R(2) * P.gamma_p * pi;
      px += c * g.x; py += c * g.y; pz += c * g.z;
      if (bodies) {
        BodyAccum acc_b{sh_body};
        for_each_normal_sample<R>(B, xi, i, P, [&](V3<R> xb, R Vb, int body) {
          if (body < 0 || !B.bodies[body].dynamic) return;
          const R rx = xi.x - xb.x, ry = xi.y - xb.y, rz = xi.z - xb.z;
          const R f = kernel_grad_factor(rx * rx + ry * ry + rz * rz, P.k);
          const double c2 = 2.0 * (double)P.gamma_p * (double)Vi * (double)Vb * (double)pi * (double)f;
          const double F[3] = {c2 * rx, c2 * ry, c2 * rz};
          const double xl[3] = {(double)xb.x, (double)xb.y, (double)xb.z};
          acc_b.add(B.bodies, body, F, xl);
        });
      }
    }
    const R vm = Vi / mi;
    const R4<R> a = R4<R>{-vm * px, -vm * py, -vm * pz, R(0)};
    if (MODE == 1) {
      R4<R> o = out[i];
      o.x += a.x; o.y += a.y; o.z += a.z;
      out[i] = o;
    } else {
      out[i] = a;
    }
  }
  if (bodies) body_accum_flush(sh_body, B.nbodies, B.body_partials);
}

// ---------------------------------------------------------------------------
// 8. IISPH: source term + diagonal + initial pressure (iisph.rs:117-376)
// ---------------------------------------------------------------------------
// VP = 1: volume-preserving source s = 1 - V0/V - dt sum ..., VP = 0: the
// velocity-divergence source of IISPHwOST's first solve.
template <class R, int VP>
__global__ void __launch_bounds__(kBlock) k_iisph_source_diag(
    const Scalars* __restrict__ sc, const R4<R>* __restrict__ xv, const R4<R>* __restrict__ vel,
    const R4<R>* __restrict__ vstar, NbrArgs N, BoundaryArgs<R> B, R* __restrict__ s_out,
    R* __restrict__ aii_out, R* __restrict__ press, R4<R>* __restrict__ TA, R4<R>* __restrict__ TB,
    R2<R>* __restrict__ SA, R4<R>* __restrict__ xq_out, StepParams<R> P) {
  extern __shared__ __align__(32) unsigned char dsm[];
  const HaloView H = halo_view(N);
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  const bool act = i < sc->n_active;
  SweepList<R> L;  // the list head travels while the halo stages
  L.begin(N, act ? i : 0, act ? min((int)N.ncnt[i], N.K) : 0);
  // records {x, V} and {v*, m} (the acceleration pass stores m in v*.w)
  R4<R>* s_x = staged_vec<R>(dsm, N.hs, 0);
  R4<R>* s_v = staged_vec<R>(dsm, N.hs, 1);
  if (H.staged)
    stage_halo(H, [&](int l, uint32_t g) {
      async_copy(&s_x[l], &xv[g]);
      async_copy(&s_v[l], &vstar[g]);
    });
  stage_done();
  if (!act) return;
  const R dt = (R)sc->dt;
  const R4<R> xi = xv[i];
  const R4<R> vsi = vstar[i];
  const R Vi = xi.w, mi = vsi.w;
  R div = 0;                       // sum V_j (v*_i - v*_j) . gradW
  R sfx = 0, sfy = 0, sfz = 0;     // S_f = sum V_j gradW
  R s2 = 0;                        // sum V_j^2 / m_j |gradW|^2
  auto pair = [&](const XV<R>& d) {  // zero at r = 0 (self padding)
    const R4<R>& xj = d.x;
    const R4<R>& vsj = d.v;
    const R rx = xi.x - xj.x, ry = xi.y - xj.y, rz = xi.z - xj.z;
    const R r2 = rx * rx + ry * ry + rz * rz;
    const R f = kernel_grad_factor(r2, P.k);
    const R Vf = xj.w * f;
    div += Vf * ((vsi.x - vsj.x) * rx + (vsi.y - vsj.y) * ry + (vsi.z - vsj.z) * rz);
    sfx += Vf * rx; sfy += Vf * ry; sfz += Vf * rz;
    s2 += xj.w * xj.w / vsj.w * (f * f * r2);
  };
  if (H.staged)
    sweep_groups(L, [&](uint32_t l) { return XV<R>{s_x[l], s_v[l]}; }, pair);
  else
    sweep_groups(L, [&](uint32_t l) { const uint32_t g = H.idx[l]; return XV<R>{xv[g], vstar[g]}; }, pair);
  R bx = 0, by = 0, bz = 0, bdiv = 0;
  if (B.kind != 0) {
    const R4<R> g = B.bG[i];
    bx = g.x; by = g.y; bz = g.z;
    bdiv = vsi.x * g.x + vsi.y * g.y + vsi.z * g.z - g.w;  // sum V_b (v*_i - v_b) . gradW
  }
  R s = VP ? R(1) - P.V0 / Vi : R(0);
  s -= dt * (div + bdiv);
  const R dt2 = dt * dt;
  const R c = -Vi / mi;
  const R cx = c * (sfx + R(2) * P.gamma_p * bx), cy = c * (sfy + R(2) * P.gamma_p * by),
          cz = c * (sfz + R(2) * P.gamma_p * bz);
  const R aii = dt2 * (cx * (sfx + bx) + cy * (sfy + by) + cz * (sfz + bz)) - dt2 * Vi * s2;
  s_out[i] = s;
  aii_out[i] = aii;
  R p0 = 0;
  if (aii > P.min_diag || aii < -P.min_diag) p0 = fmax(P.omega * s / aii, R(0));
  press[i] = p0;
  // the Jacobi sweeps' per-solve constants (S_i = sum_j V_j gradW_ij with the
  // boundary terms folded in) and the first pass A record {x, V p}
  const R g2 = R(2) * P.gamma_p;
  TA[i] = R4<R>{sfx + g2 * bx, sfy + g2 * by, sfz + g2 * bz, -(Vi / mi) * Vi};
  TB[i] = R4<R>{sfx + bx, sfy + by, sfz + bz, Vi};
  SA[i] = R2<R>{s, aii};
  xq_out[i] = R4<R>{xi.x, xi.y, xi.z, Vi * p0};
}

// ---------------------------------------------------------------------------
// Jacobi sweep (iisph.rs:401-560): pass A, the pressure accelerations of the
// current pressures (pressure_solver/mod.rs:121-195, overwrite, no reaction
// forces), then pass B, A_i, the relaxed pressure update and the residual.
// Positions and volumes are fixed during a solve, so the pair sums split:
//   sum_j V_j (p_i + p_j) gradW_ij    = p_i S_i + sum_j (V_j p_j) gradW_ij
//   sum_j V_j (a_i - a_j) . gradW_ij  = a_i . S_i - sum_j (V_j a_j) . gradW_ij
// with S_i = sum_j V_j gradW_ij from the source pass (stored with the boundary
// terms and the particle's own constants: TA = {S_i + 2 gamma_p bG_i, -V_i^2/m_i},
// TB = {S_i + bG_i, V_i}, SA = {s_i, a_ii}). Each pass then gathers
// one record per neighbor from the block's halo in shared memory:
//   pass A: xq = {x, y, z, V p}            (written by pass B and the source pass)
//   pass B: xu = {x, y, z, V a_x}, uu = {V a_y, V a_z}   (written by pass A)
// A neighbor group of four always holds four valid halo positions (unused
// slots repeat the particle's own, whose pair adds zero), so the loops carry
// no per-neighbor test. The kernel constant cg (-3 cg for pass A's piecewise
// gradient factor) multiplies each pair sum once.
// ---------------------------------------------------------------------------

// pass A: a_i = -(V_i/m_i) [p_i (S_i + 2 gamma_p bG_i) + sum_j (V_j p_j) gradW_ij],
// stored as the records of pass B (V_i a_i).
// (f32: at most 48 registers, so five blocks share an SM; the records are
// gathered two at a time to fit)
// OUT 0: the records of pass B; OUT 1: acc += a_i, OUT 2: acc = a_i (the
// final pressure acceleration of a solve, pressure_solver/mod.rs:121-195,
// when no boundary takes reaction forces).
template <class R, int OUT = 0>
__global__ void __launch_bounds__(kBlock, sizeof(R) == 4 ? 5 : 1) k_sweep_accel(
    const Scalars* __restrict__ sc, const R* __restrict__ press, const R4<R>* __restrict__ TA,
    const R4<R>* __restrict__ xq, NbrArgs N, R4<R>* __restrict__ xu, R2<R>* __restrict__ uu, StepParams<R> P,
    R4<R>* __restrict__ acc, const R4<R>* __restrict__ TB) {
  grid_dep_release();
  extern __shared__ __align__(32) unsigned char dsm[];
  const HaloView H = halo_view(N);
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  const bool act = i < sc->n_active;
  // what is fixed during a solve (list head, constants, halo indices) is read
  // before the wait on the previous pass; p and the records after it
  SweepList<R> L;
  L.begin(N, act ? i : 0, act ? min((int)N.ncnt[i], N.K) : 0);
  R4<R> xi{}, Ti{};
  R pi = 0;
  if (act) Ti = TA[i];
  const HaloFirst hf = halo_first(H);
  grid_dep_wait();
  if (OUT == 0 && sc->converged) return;
  if (act) {
    xi = xq[i];
    pi = press[i];
  }
  R4<R>* s_r = reinterpret_cast<R4<R>*>(dsm);
  stage_halo_from(H, hf, [&](int l, uint32_t g) { async_copy(&s_r[l], &xq[g]); });
  prefetch_ahead(N, sc->n_active, xq, TA, press);
  stage_done();
  if (!act) return;
  const R ih = P.k.inv_h;
  R px = 0, py = 0, pz = 0;
  auto pair = [&](const R4<R>& r) {
    const R rx = xi.x - r.x, ry = xi.y - r.y, rz = xi.z - r.z;
    const R t = r.w * grad_piecewise(rx * rx + ry * ry + rz * rz, ih);
    px += t * rx; py += t * ry; pz += t * rz;
  };
  if (H.staged) {
    for (int g = 0; g < L.ng; ++g) {
      const uint2 w = L.next(g);
      {
        const R4<R> r0 = s_r[w.x & 0xffffu], r1 = s_r[w.x >> 16];
        pair(r0); pair(r1);
      }
      {
        const R4<R> r2 = s_r[w.y & 0xffffu], r3 = s_r[w.y >> 16];
        pair(r2); pair(r3);
      }
    }
  } else {
    for (int g = 0; g < L.ng; ++g) {
      const uint2 w = L.next(g);
      const R4<R> r0 = xq[H.idx[w.x & 0xffffu]], r1 = xq[H.idx[w.x >> 16]], r2 = xq[H.idx[w.y & 0xffffu]],
                  r3 = xq[H.idx[w.y >> 16]];
      pair(r0); pair(r1); pair(r2); pair(r3);
    }
  }
  const R cg = R(-3) * P.k.cg;  // grad_piecewise is grad_core divided by -3
  const R fx = pi * Ti.x + cg * px, fy = pi * Ti.y + cg * py, fz = pi * Ti.z + cg * pz;
  const R c = Ti.w;  // V_i a_i = -(V_i^2 / m_i) F
  if (OUT == 0) {
    xu[i] = R4<R>{xi.x, xi.y, xi.z, c * fx};
    uu[i] = R2<R>{c * fy, c * fz};
  } else {
    const R m = c / TB[i].w;  // a_i = -(V_i / m_i) F, TB.w = V_i
    R4<R> o = OUT == 1 ? acc[i] : R4<R>{R(0), R(0), R(0), R(0)};
    o.x += m * fx; o.y += m * fy; o.z += m * fz;
    acc[i] = o;
  }
}

// pass B: A_i = dt^2 [a_i . (S_i + bG_i) - sum_j (V_j a_j) . gradW_ij];
// p_i <- max(p_i + omega (s_i - A_i) / a_ii, 0) where a_ii < -eps; the
// residual e_i = |A_i - s_i| where s_i < 0, summed in f64 over all N (last
// block: error, sweep count and the stop test of iisph.rs:378-393).
// AFTER >= 0: stop after AFTER+1 sweeps; AFTER < 0: target density error.
template <class R>
__global__ void __launch_bounds__(kBlock, sizeof(R) == 4 ? 5 : 1) k_sweep_jacobi(
    Scalars* __restrict__ sc, const R4<R>* __restrict__ TB, const R2<R>* __restrict__ SA,
    const R4<R>* __restrict__ xu, const R2<R>* __restrict__ uu, NbrArgs N, R* __restrict__ press,
    R4<R>* __restrict__ xq, double* __restrict__ partials, int after, StepParams<R> P) {
  grid_dep_release();
  __shared__ double sh[32];
  extern __shared__ __align__(32) unsigned char dsm[];
  const HaloView H = halo_view(N);
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  const int n = sc->n_active;
  const bool act = i < n;
  // fixed during a solve: read before the wait on pass A
  SweepList<R> L;
  L.begin(N, act ? i : 0, act ? min((int)N.ncnt[i], N.K) : 0);
  R4<R> Ti{}, u4{};
  R2<R> u2{}, sa{};
  R p0 = 0;
  if (act) {
    Ti = TB[i];
    sa = SA[i];
  }
  const HaloFirst hf = halo_first(H);
  grid_dep_wait();
  if (sc->converged) return;
  if (act) {
    u4 = xu[i];
    u2 = uu[i];
    p0 = press[i];
  }
  const R4<R> xi{u4.x, u4.y, u4.z, Ti.w};
  R4<R>* s_a = reinterpret_cast<R4<R>*>(dsm);
  R2<R>* s_b = reinterpret_cast<R2<R>*>(s_a + N.hs);
  stage_halo_from(H, hf, [&](int l, uint32_t g) {
    async_copy(&s_a[l], &xu[g]);
    async_copy(&s_b[l], &uu[g]);
  });
  prefetch_ahead(N, n, xu, uu, TB, SA, (const R*)press);
  stage_done();
  double e = 0.0;
  if (act) {
    const R ih = P.k.inv_h;
    R sum = 0;
    auto pair = [&](const R4<R>& a, const R2<R>& b) {
      const R rx = xi.x - a.x, ry = xi.y - a.y, rz = xi.z - a.z;
      sum += grad_core(rx * rx + ry * ry + rz * rz, ih) * (a.w * rx + b.x * ry + b.y * rz);
    };
    if (H.staged) {
      for (int g = 0; g < L.ng; ++g) {
        const uint2 w = L.next(g);
        const uint32_t l0 = w.x & 0xffffu, l1 = w.x >> 16, l2 = w.y & 0xffffu, l3 = w.y >> 16;
        const R4<R> a0 = s_a[l0], a1 = s_a[l1], a2 = s_a[l2], a3 = s_a[l3];
        const R2<R> b0 = s_b[l0], b1 = s_b[l1], b2 = s_b[l2], b3 = s_b[l3];
        pair(a0, b0); pair(a1, b1); pair(a2, b2); pair(a3, b3);
      }
    } else {
      for (int g = 0; g < L.ng; ++g) {
        const uint2 w = L.next(g);
        const uint32_t g0 = H.idx[w.x & 0xffffu], g1 = H.idx[w.x >> 16], g2 = H.idx[w.y & 0xffffu],
                       g3 = H.idx[w.y >> 16];
        const R4<R> a0 = xu[g0], a1 = xu[g1], a2 = xu[g2], a3 = xu[g3];
        const R2<R> b0 = uu[g0], b1 = uu[g1], b2 = uu[g2], b3 = uu[g3];
        pair(a0, b0); pair(a1, b1); pair(a2, b2); pair(a3, b3);
      }
    }
    const R dt = (R)sc->dt;
    const R iV = R(1) / xi.w;
    const R ax = u4.w * iV, ay = u2.x * iV, az = u2.y * iV;
    const R tot = ax * Ti.x + ay * Ti.y + az * Ti.z - P.k.cg * sum;
    const R A = dt * dt * tot;
    const R s = sa.x, aii = sa.y;
    R pn = p0;
    if (aii < -P.min_diag) pn = fmax(p0 + P.omega * (s - A) / aii, R(0));
    press[i] = pn;
    xq[i] = R4<R>{xi.x, xi.y, xi.z, xi.w * pn};
    if (s < R(0)) e = fabs((double)A - (double)s);
  }
  const double bs = block_sum(e, sh);
  double total;
  if (last_block_total(bs, partials, &sc->done_blocks, &total, sh)) {
    const double err = n > 0 ? total / (double)n * 100.0 : 0.0;
    const int it = sc->iterations + 1;
    sc->iterations = it;
    sc->err = err;
    bool stop;
    if (after >= 0) {
      stop = it > after;
    } else {
      stop = it > 2 && err < P.tde;
      if (!stop && P.iteration_cap > 0 && it >= P.iteration_cap) {
        stop = true;
        sc->status = 2;  // not converged within the cap
      }
    }
    if (stop) sc->converged = 1;
  }
}

// IISPHwOST between the solves: v* += dt a_p1 (iisph_optimized_source_term.rs:97-110)
template <class R>
__global__ void __launch_bounds__(kBlock) k_ost_predict(Scalars* __restrict__ sc,
                                                       const R4<R>* __restrict__ acc,
                                                       R4<R>* __restrict__ vstar) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i == 0) {
    sc->iterations_eqs1 = sc->iterations;
    sc->iterations = 0;
    sc->converged = 0;
    sc->err = INFINITY;
  }
  if (i >= sc->n_active) return;
  const R dt = (R)sc->dt;
  const R4<R> a = acc[i];
  R4<R> v = vstar[i];
  v.x += dt * a.x; v.y += dt * a.y; v.z += dt * a.z;
  vstar[i] = v;
}

// IISPHwOST commit: x_pred = x + dt v*, x_new = x_pred + dt^2 a, v_new = v* + dt a
// into the integrator slots (iisph_optimized_source_term.rs:139-216).
template <class R>
__global__ void __launch_bounds__(kBlock) k_ost_commit(const Scalars* __restrict__ sc,
                                                      const R4<R>* __restrict__ xv,
                                                      const R4<R>* __restrict__ vel,
                                                      const R4<R>* __restrict__ vstar,
                                                      const R4<R>* __restrict__ acc,
                                                      R4<R>* __restrict__ xint,
                                                      R4<R>* __restrict__ vint) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= sc->n_active) return;
  const R dt = (R)sc->dt;
  const R dt2 = dt * dt;
  const R4<R> x = xv[i], v = vstar[i], a = acc[i];
  const R xpx = x.x + dt * v.x, xpy = x.y + dt * v.y, xpz = x.z + dt * v.z;
  xint[i] = R4<R>{xpx + dt2 * a.x, xpy + dt2 * a.y, xpz + dt2 * a.z, R(0)};
  vint[i] = R4<R>{v.x + dt * a.x, v.y + dt * a.y, v.z + dt * a.z, vel[i].w};
}

// SESPHwSplitting predicted density (sesph_with_splitting.rs:90-152) and the
// state equation: rho* = sum_j [m_j W + dt (v*_i - v*_j) . gradW]
//                      + (m_i/V0) bW + dt v*_i . bGu, p = k max(V0/(m_i/rho*) - 1, 0)
template <class R, int NB>
__global__ void __launch_bounds__(kBlock) k_split_density(
    const Scalars* __restrict__ sc, const R4<R>* __restrict__ xv, const R4<R>* __restrict__ vel,
    const R4<R>* __restrict__ vstar, NbrArgs N, BoundaryArgs<R> B, R* __restrict__ press,
    R* __restrict__ rho_pred, StepParams<R> P) {
  extern __shared__ __align__(32) unsigned char dsm[];
  const HaloView H = halo_view(N);
  // records {x, V} and {v*, m} (the acceleration pass stores m in v*.w)
  R4<R>* s_x = staged_vec<R>(dsm, N.hs, 0);
  R4<R>* s_v = staged_vec<R>(dsm, N.hs, 1);
  if (H.staged)
    stage_halo(H, [&](int l, uint32_t g) {
      async_copy(&s_x[l], &xv[g]);
      async_copy(&s_v[l], &vstar[g]);
    });
  stage_done();
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= sc->n_active) return;
  const R dt = (R)sc->dt;
  const R4<R> xi = xv[i];
  const R4<R> vsi = vstar[i];
  const R mi = vsi.w;
  R rho = mi * P.k.cw * R(0.5), comp = 0;  // self term m_i W(0)
  const int cnt = min((int)N.ncnt[i], N.K);
  for_each_neighbor<NB>(
      N.nbr, N.K, i, cnt,
      [&](uint32_t l) {
        if (H.staged) return XV<R>{s_x[l], s_v[l]};
        const uint32_t g = H.idx[l];
        return XV<R>{xv[g], vstar[g]};
      },
      [&](const XV<R>& d) {
        const R4<R>& xj = d.x;
        const R4<R>& vsj = d.v;
        const R rx = xi.x - xj.x, ry = xi.y - xj.y, rz = xi.z - xj.z;
        R w, f;
        kernel_w_and_grad(rx * rx + ry * ry + rz * rz, P.k, w, f);
        const R t = vsj.w * w + dt * f * ((vsi.x - vsj.x) * rx + (vsi.y - vsj.y) * ry + (vsi.z - vsj.z) * rz);
        kahan_add(rho, comp, t);
      });
  if (B.kind != 0) {
    const R4<R> gu = B.bGu[i];
    rho += B.bW[i] * mi / P.V0 + dt * (vsi.x * gu.x + vsi.y * gu.y + vsi.z * gu.z);
  }
  rho_pred[i] = rho;
  const R vol = mi / rho;
  press[i] = P.stiffness * fmax(P.V0 / vol - R(1), R(0));
}

// ---------------------------------------------------------------------------
// 9. reductions: average density after the update (sph/mod.rs:444-486) and
//    measurement sums (density error, kinetic energy) in f64
// ---------------------------------------------------------------------------
template <class R>
__global__ void __launch_bounds__(kBlock) k_avg_density(Scalars* __restrict__ sc,
                                                       const R4<R>* __restrict__ xv,
                                                       const R4<R>* __restrict__ vel,
                                                       double* __restrict__ partials,
                                                       StepParams<R> P) {
  __shared__ double sh[32];
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  const int n = sc->n_active;
  double d = 0.0;
  if (i < n) {
    const double V = (double)xv[i].w, m = (double)vel[i].w, V0 = (double)P.V0;
    d = V < V0 ? m / V : m / V0;
  }
  double total;
  if (last_block_total(block_sum(d, sh), partials, &sc->done_blocks, &total, sh))
    sc->avg_density = n > 0 ? total / (double)n : 0.0;
}

// out[0] = sum (V < V0 ? V0/V : 1), out[1] = sum 1/2 m |v|^2
template <class R>
__global__ void __launch_bounds__(kBlock) k_measure(Scalars* __restrict__ sc,
                                                   const R4<R>* __restrict__ xv,
                                                   const R4<R>* __restrict__ vel,
                                                   double* __restrict__ partials,
                                                   double* __restrict__ out, StepParams<R> P) {
  __shared__ double sh[32];
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  const int n = sc->n_active;
  double de = 0.0, ke = 0.0;
  if (i < n) {
    const double V = (double)xv[i].w, V0 = (double)P.V0;
    de = V < V0 ? V0 / V : 1.0;
    const R4<R> v = vel[i];
    const double vx = v.x, vy = v.y, vz = v.z;
    ke = 0.5 * (double)v.w * ((vx * vx + vy * vy) + vz * vz);
  }
  const double b0 = block_sum(de, sh);
  const double b1 = block_sum(ke, sh);
  // one completion counter for both sums
  __shared__ bool is_last;
  if (threadIdx.x == 0) {
    partials[blockIdx.x] = b0;
    partials[gridDim.x + blockIdx.x] = b1;
    __threadfence();
    is_last = atomicAdd(&sc->done_blocks, 1u) == gridDim.x - 1;
  }
  __syncthreads();
  if (!is_last) return;
  __threadfence();
  double s0 = 0, s1 = 0;
  for (unsigned b = threadIdx.x; b < gridDim.x; b += blockDim.x) {
    s0 += ((volatile double*)partials)[b];
    s1 += ((volatile double*)partials)[gridDim.x + b];
  }
  s0 = block_sum(s0, sh);
  s1 = block_sum(s1, sh);
  if (threadIdx.x == 0) {
    out[0] = s0;
    out[1] = s1;
    sc->done_blocks = 0;
  }
}

// ---------------------------------------------------------------------------
// 10. rigid bodies (f64)
// ---------------------------------------------------------------------------
// Gravity on dynamic bodies: F += m g at the center of mass
// (non_pressure_accelerations.rs:79-100, static_sample_boundary.rs:328-341).
__global__ void k_body_gravity(Body* bodies, int nb, int mode, double gx, double gy, double gz) {
  const int b = threadIdx.x;
  if (b >= nb || !bodies[b].dynamic) return;
  Body& B = bodies[b];
  double a[3];
  if (mode == 0) {
    a[0] = 0.0; a[1] = 0.0; a[2] = -9.81;
  } else {
    const double d[3] = {gx - B.com[0], gy - B.com[1], gz - B.com[2]};
    const double dist = sqrt(((d[0] * d[0] + d[1] * d[1]) + d[2] * d[2]) + 1e-4);
    for (int c = 0; c < 3; ++c) a[c] = 9.81 * d[c] / dist;
  }
  for (int c = 0; c < 3; ++c) B.F[c] += a[c] * B.mass;
}

// Fixed-order sum of per-block reaction partials into the body accumulators.
__global__ void k_body_reduce(Body* bodies, int nb, const double* partials, int nblocks) {
  const int b = blockIdx.x;
  if (b >= nb || !bodies[b].dynamic) return;
  __shared__ double sh[32];
  for (int c = 0; c < 6; ++c) {
    double s = 0.0;
    for (int k = threadIdx.x; k < nblocks; k += blockDim.x)
      s += partials[(size_t)k * kMaxBodies * 6 + b * 6 + c];
    s = block_sum(s, sh);
    if (threadIdx.x == 0) {
      if (c < 3) bodies[b].F[c] += s;
      else bodies[b].T[c - 3] += s;
    }
    __syncthreads();
  }
}

__device__ void mat_rot(const double q[4], double R_[9]) {
  const double ww = q[0] * q[0], ii = q[1] * q[1], jj = q[2] * q[2], kk = q[3] * q[3];
  const double ij = q[1] * q[2] * 2.0, wk = q[0] * q[3] * 2.0, wj = q[0] * q[2] * 2.0;
  const double ik = q[1] * q[3] * 2.0, jk = q[2] * q[3] * 2.0, wi = q[0] * q[1] * 2.0;
  R_[0] = ww + ii - jj - kk; R_[1] = ij - wk; R_[2] = wj + ik;
  R_[3] = wk + ij; R_[4] = ww - ii + jj - kk; R_[5] = jk - wi;
  R_[6] = ik - wj; R_[7] = wi + jk; R_[8] = ww - ii - jj + kk;
}
__device__ void body_update_derived(Body& B) {
  double Rm[9], t[9];
  mat_rot(B.q, Rm);
  for (int r = 0; r < 3; ++r)
    for (int c = 0; c < 3; ++c)
      t[r * 3 + c] = (Rm[r * 3 + 0] * B.inv_inertia_body[0 * 3 + c] +
                      Rm[r * 3 + 1] * B.inv_inertia_body[1 * 3 + c]) +
                     Rm[r * 3 + 2] * B.inv_inertia_body[2 * 3 + c];
  for (int r = 0; r < 3; ++r)
    for (int c = 0; c < 3; ++c)
      B.inv_inertia_world[r * 3 + c] =
          (t[r * 3 + 0] * Rm[c * 3 + 0] + t[r * 3 + 1] * Rm[c * 3 + 1]) + t[r * 3 + 2] * Rm[c * 3 + 2];
  for (int r = 0; r < 3; ++r)
    B.omega[r] = (B.inv_inertia_world[r * 3 + 0] * B.L[0] + B.inv_inertia_world[r * 3 + 1] * B.L[1]) +
                 B.inv_inertia_world[r * 3 + 2] * B.L[2];
}

// Euler-Cromer body step with q <- exp(omega dt / 2) q (rigid_body_motion.rs:183-201).
__global__ void k_body_step(Body* bodies, int nb, const Scalars* sc) {
  const int b = threadIdx.x;
  if (b >= nb || !bodies[b].dynamic) return;
  Body& B = bodies[b];
  const double dt = sc->dt;
  for (int c = 0; c < 3; ++c) {
    const double a = B.F[c] / B.mass;
    B.v[c] += a * dt;
  }
  for (int c = 0; c < 3; ++c) B.com[c] += B.v[c] * dt;
  for (int c = 0; c < 3; ++c) B.L[c] += B.T[c] * dt;
  for (int r = 0; r < 3; ++r)
    B.omega[r] = (B.inv_inertia_world[r * 3 + 0] * B.L[0] + B.inv_inertia_world[r * 3 + 1] * B.L[1]) +
                 B.inv_inertia_world[r * 3 + 2] * B.L[2];
  const double h[3] = {B.omega[0] * dt / 2.0, B.omega[1] * dt / 2.0, B.omega[2] * dt / 2.0};
  const double nn = (h[0] * h[0] + h[1] * h[1]) + h[2] * h[2];
  double e[4] = {1.0, 0.0, 0.0, 0.0};
  if (nn > DBL_EPSILON * DBL_EPSILON) {
    const double nrm = sqrt(nn), s = sin(nrm) / nrm;
    e[0] = cos(nrm); e[1] = h[0] * s; e[2] = h[1] * s; e[3] = h[2] * s;
  }
  const double* q = B.q;
  const double nq[4] = {e[0] * q[0] - e[1] * q[1] - e[2] * q[2] - e[3] * q[3],
                        e[0] * q[1] + e[1] * q[0] + e[2] * q[3] - e[3] * q[2],
                        e[0] * q[2] - e[1] * q[3] + e[2] * q[0] + e[3] * q[1],
                        e[0] * q[3] + e[1] * q[2] - e[2] * q[1] + e[3] * q[0]};
  for (int c = 0; c < 4; ++c) B.q[c] = nq[c];
  for (int c = 0; c < 3; ++c) { B.F[c] = 0.0; B.T[c] = 0.0; }
  body_update_derived(B);
}

// World positions/velocities of dynamic sample-boundary samples
// (static_sample_boundary.rs:392-412): x = R x_body + c, v = v + omega x (x - c).
template <class R>
__global__ void __launch_bounds__(kBlock) k_body_samples(const int* __restrict__ n_ptr,
                                                        const Body* __restrict__ bodies,
                                                        const R4<R>* __restrict__ x_body,
                                                        const uint32_t* __restrict__ orig,
                                                        const uint32_t* __restrict__ bid,
                                                        R4<R>* __restrict__ xb,
                                                        R4<R>* __restrict__ vb) {
  const int d = blockIdx.x * blockDim.x + threadIdx.x;
  if (d >= *n_ptr) return;
  const Body& B = bodies[bid[d]];
  if (!B.dynamic) return;
  const R4<R> xl = x_body[orig[d]];
  const double pl[3] = {(double)xl.x, (double)xl.y, (double)xl.z};
  double pw[3];
  qrot(B.q, pl, pw);
  for (int c = 0; c < 3; ++c) pw[c] += B.com[c];
  double vw[3];
  body_velocity_at(B, pw, vw);
  const R V = xb[d].w;
  xb[d] = R4<R>{(R)pw[0], (R)pw[1], (R)pw[2], V};
  vb[d] = R4<R>{(R)vw[0], (R)vw[1], (R)vw[2], R(0)};
}

// Boundary pseudo-volumes V_b = gamma_V / sum_{b' same boundary} W_bb'
// (static_sample_boundary.rs:354-390), on the sorted sample grid.
template <class R>
__global__ void __launch_bounds__(kBlock) k_sample_volumes(const int* __restrict__ n_ptr,
                                                          SampleGrid<R> G, R4<R>* __restrict__ xb,
                                                          double gamma_v, StepParams<R> P) {
  const int d = blockIdx.x * blockDim.x + threadIdx.x;
  if (d >= *n_ptr) return;
  const R4<R> xi = G.xb[d];
  const uint32_t myb = G.bid[d];
  const int cx = cell_coord((double)xi.x, P.range), cy = cell_coord((double)xi.y, P.range),
            cz = cell_coord((double)xi.z, P.range);
  R sum = 0, comp = 0;
  for (int dz = -1; dz <= 1; ++dz)
    for (int dy = -1; dy <= 1; ++dy)
      for (int dx = -1; dx <= 1; ++dx) {
        const uint32_t k = morton_key(cx + dx, cy + dy, cz + dz, G.mask);
        const uint32_t b = G.start[k], e = G.start[k + 1];
        for (uint32_t s = b; s < e; ++s) {
          if (G.bid[s] != myb) continue;
          const R4<R> xs = G.xb[s];
          if (!in_range(xi, xs, P.range, P.range2_lo, P.range2_hi)) continue;
          const R rx = xi.x - xs.x, ry = xi.y - xs.y, rz = xi.z - xs.z;
          kahan_add(sum, comp, kernel_w_r2(rx * rx + ry * ry + rz * rz, P.k));
        }
      }
  R4<R> o = xi;
  o.w = (R)(gamma_v / (double)sum);
  xb[d] = o;
}

// ---------------------------------------------------------------------------
// graph-captured stepping
// ---------------------------------------------------------------------------
// Opens a chunk of graph launches: simulated time enters, flags clear.
__global__ void k_chunk_begin(Scalars* sc, double time) {
  sc->time_acc = time;
  sc->trouble = 0;
  sc->status_any = 0;
  sc->loop_sweeps = 0;
  sc->chunk_max_nbrs = 0;
  sc->chunk_max_halo = 0;
}

// Condition of the while-node that runs the Jacobi sweeps of one solve: go on
// until the sweep kernel sets `converged` or `limit` sweeps have run. Every
// body execution either finds `converged` set or adds one to `iterations`,
// so the loop ends after at most `limit` bodies.
__global__ void k_loop_cond(cudaGraphConditionalHandle h, const Scalars* __restrict__ sc, int limit) {
  grid_dep_wait();
  const unsigned int more = (!sc->converged && sc->iterations < limit) ? 1u : 0u;
  cudaGraphSetConditional(h, more);
}

// End of a graph-captured step: records what the per-step host check would
// have acted on (then the host replays the chunk on the per-step path) and
// prepares the scalars of the next update exactly as that check does.
__global__ void k_step_epilogue(Scalars* sc, int K, int hcap, int solver_loop) {
  unsigned int t = 0;
  if (sc->max_nbrs > K || sc->max_halo > hcap) t |= 1u;
  sc->chunk_max_nbrs = max(sc->chunk_max_nbrs, sc->max_nbrs);
  sc->chunk_max_halo = max(sc->chunk_max_halo, sc->max_halo);
  if (sc->n_below > 0) t |= 2u;
  if (solver_loop && !sc->converged) t |= 4u;
  sc->trouble |= t;
  if (sc->status == 2) sc->status_any = 2;
  if (solver_loop) sc->loop_sweeps += (unsigned long long)sc->iterations;
  sc->n = sc->n_active;
  sc->n_below = 0;
  sc->max_speed = 0;
}

// ---------------------------------------------------------------------------
// Rigid-rigid contact of volume-map bodies (volume_map_boundary.rs:55-1102,
// 1440-1453), run before the body step. k_contact_tasks cuts the overlap of
// every pair of world bounding boxes (at least one body dynamic) into
// sub-cells; k_contact_build evaluates one sub-cell per block, one 8^3
// Gauss-Legendre point per thread, and reduces the contact cell's volume,
// center and unit force/torque sensitivities (build_contact_cell and
// compute_diagonal); k_contact_solve runs the NNCG-accelerated projected
// Jacobi iteration for all cells in one block and adds the contact forces
// and torques to the bodies. Everything is f64.
// ---------------------------------------------------------------------------
__device__ __forceinline__ bool vm_phi(const VMDesc& D, const Body* bodies, const double p[3], double& phi) {
  double pl[3] = {p[0], p[1], p[2]};
  if (D.body >= 0) body_world_to_local(bodies[D.body], p, pl);
  return ser_function(D.sdf, pl[0], pl[1], pl[2], phi);
}
__device__ __forceinline__ bool vm_phi_grad(const VMDesc& D, const Body* bodies, const double p[3], double g[3]) {
  double pl[3] = {p[0], p[1], p[2]};
  if (D.body >= 0) body_world_to_local(bodies[D.body], p, pl);
  if (!ser_gradient(D.sdf, pl[0], pl[1], pl[2], g)) return false;
  if (D.body >= 0) {
    double gw[3];
    qrot(bodies[D.body].q, g, gw);
    g[0] = gw[0]; g[1] = gw[1]; g[2] = gw[2];
  }
  return true;
}

// cubic_extension_fn and its derivative (:1717-1745): the cubic spline's
// W(x) / W(0) on (0, h), 1 below and 0 above.
__device__ __forceinline__ double cubic_ext(double x, double h) {
  if (x >= h) return 0.;
  if (x <= 0.) return 1.;
  const double q = x / h, a = fmax(1. - q, 0.), b = fmax(0.5 - q, 0.);
  const double c = 16. / 3.14159265358979323846 / (h * h * h);
  return (c * (a * a * a - 4. * (b * b * b))) / (c * 0.5);
}
__device__ __forceinline__ double cubic_ext_derivative(double x, double h) {
  if (x >= h || x <= 0.) return 0.;
  const double q = x / h, a = fmax(1. - q, 0.), b = fmax(0.5 - q, 0.);
  const double alpha = 16. / 3.14159265358979323846;
  const double c4 = alpha / (h * h * h * h);
  return (((c4 * x) / x) * (-3. * (a * a) + 12. * (b * b))) / (alpha / (h * h * h) * 0.5);
}

// World bounding box (BoundaryType::world_aabb, :2122-2151).
__device__ void vm_world_box(const VMDesc& D, const Body* bodies, double lo[3], double hi[3]) {
  if (D.body < 0) {
    for (int d = 0; d < 3; ++d) {
      lo[d] = D.aabb_c[d] - D.aabb_h[d];
      hi[d] = D.aabb_c[d] + D.aabb_h[d];
    }
    return;
  }
  const Body& B = bodies[D.body];
  double Rm[9], c[3];
  mat_rot(B.q, Rm);
  qrot(B.q, D.aabb_c, c);
  for (int d = 0; d < 3; ++d) {
    const double he = (fabs(Rm[d * 3]) * D.aabb_h[0] + fabs(Rm[d * 3 + 1]) * D.aabb_h[1]) +
                      fabs(Rm[d * 3 + 2]) * D.aabb_h[2];
    const double cw = c[d] + B.com[d];
    lo[d] = cw - he;
    hi[d] = cw + he;
  }
}

// broad_phase (:70-96) and the task list of generate_contact_cells
// (:98-117) with subdivide_overlap (:1813-1844); one thread.
__global__ void k_contact_tasks(const VMDesc* __restrict__ vms, const Body* __restrict__ bodies, int nb,
                                double target, ContactPair* __restrict__ pairs, ContactScalars* __restrict__ cs,
                                int task_cap) {
  if (threadIdx.x != 0 || blockIdx.x != 0) return;
  int np = 0, nt = 0, overflow = 0;
  for (int i = 0; i < nb; ++i) {
    if (!vms[i].has_aabb) continue;
    double li[3], hi_[3];
    vm_world_box(vms[i], bodies, li, hi_);
    for (int j = i + 1; j < nb; ++j) {
      if (!vms[j].has_aabb) continue;
      if (vms[i].body < 0 && vms[j].body < 0) continue;
      double lj[3], hj[3];
      vm_world_box(vms[j], bodies, lj, hj);
      bool overlap = true;
      for (int d = 0; d < 3; ++d) overlap = overlap && li[d] <= hj[d] && hi_[d] >= lj[d];
      if (!overlap) continue;
      double mn[3], mx[3];
      bool inter = true;
      for (int d = 0; d < 3; ++d) {
        mn[d] = fmax(li[d], lj[d]);
        mx[d] = fmin(hi_[d], hj[d]);
        inter = inter && mn[d] <= mx[d];
      }
      if (!inter) continue;
      ContactPair P;
      P.a = i;
      P.b = j;
      double cnt = 1.0;
      for (int d = 0; d < 3; ++d) {
        const double ext = mx[d] - mn[d];
        const double nd = fmax(ceil(ext / target), 1.0);
        cnt *= nd;
        P.n[d] = nd < 1e7 ? (int)nd : 10000000;
        P.min[d] = mn[d];
      }
      if (cnt > (double)(task_cap - nt)) {
        overflow = 1;
        continue;
      }
      for (int d = 0; d < 3; ++d) P.cs[d] = (mx[d] - mn[d]) / (double)P.n[d];
      P.first = nt;
      pairs[np++] = P;
      nt += P.n[0] * P.n[1] * P.n[2];
    }
  }
  cs->npairs = np;
  cs->ntasks = nt;
  cs->ncells = 0;
  cs->iterations = 0;
  cs->overflow = overflow;
  cs->capped = 0;
}

// build_contact_cell (:700-782) and compute_diagonal (:835-926): block per
// sub-cell, thread per quadrature point (x slowest, z fastest as
// quadrature_points orders them).
constexpr int kContactThreads = kContactQuad * kContactQuad * kContactQuad;
__global__ void __launch_bounds__(kContactThreads) k_contact_build(
    const VMDesc* __restrict__ vms, const Body* __restrict__ bodies, const ContactPair* __restrict__ pairs,
    const ContactScalars* __restrict__ cs, ContactCell* __restrict__ cells, ContactGL gl, double h,
    const Scalars* __restrict__ sc) {
  __shared__ double red[kContactThreads / 32][17];
  __shared__ double tot[17];
  __shared__ int go;
  const int ntasks = cs->ntasks, npairs = cs->npairs;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  for (int t = blockIdx.x; t < ntasks; t += gridDim.x) {
    int pi = 0;
    while (pi + 1 < npairs && pairs[pi + 1].first <= t) ++pi;
    const ContactPair P = pairs[pi];
    const int local = t - P.first;
    const int idx[3] = {local % P.n[0], (local / P.n[0]) % P.n[1], local / (P.n[0] * P.n[1])};
    double from[3], dd[3], half[3], center[3];
    for (int d = 0; d < 3; ++d) {
      from[d] = P.min[d] + (double)idx[d] * P.cs[d];
      dd[d] = (from[d] + P.cs[d]) - from[d];
      half[d] = dd[d] * 0.5;
      center[d] = from[d] + half[d];
    }
    const VMDesc& A = vms[P.a];
    const VMDesc& B = vms[P.b];
    if (threadIdx.x == 0) {
      // pruning (:128-159): both solids within twice the half diagonal
      const double bound = 2.0 * (sqrt((dd[0] * dd[0] + dd[1] * dd[1]) + dd[2] * dd[2]) * 0.5);
      double pa, pb;
      const bool oka = vm_phi(A, bodies, center, pa);
      const bool okb = vm_phi(B, bodies, center, pb);
      go = oka && okb && pa - bound < 0. && pb - bound < 0.;
      if (!go) cells[t].valid = 0;
    }
    __syncthreads();
    if (!go) {
      __syncthreads();
      continue;
    }
    const int q = threadIdx.x;
    const int i = q >> 6, j = (q >> 3) & 7, k = q & 7;
    const double pos[3] = {center[0] + gl.x[i] * half[0], center[1] + gl.x[j] * half[1],
                           center[2] + gl.x[k] * half[2]};
    const double w = gl.w[i] * gl.w[j] * gl.w[k] * half[0] * half[1] * half[2];
    // 0 count, 1 volume, 2-4 x V, 5-7 f_a, 8-10 tau_a, 11-13 f_b, 14-16 tau_b
    double v[17];
    for (int c = 0; c < 17; ++c) v[c] = 0.0;
    double pa, pb, ga[3], gb[3];
    if (vm_phi(A, bodies, pos, pa) && vm_phi(B, bodies, pos, pb)) {
      const double sa = cubic_ext(2.0 * pa + h, h), sb = cubic_ext(2.0 * pb + h, h);
      if (sa > 0.0 && sb > 0.0 && vm_phi_grad(A, bodies, pos, ga) && vm_phi_grad(B, bodies, pos, gb)) {
        const double spa = 2.0 * cubic_ext_derivative(2.0 * pa + h, h);
        const double spb = 2.0 * cubic_ext_derivative(2.0 * pb + h, h);
        const double wg = w * sa * sb, wa = w * spa * sb, wb = w * spb * sa;
        v[0] = 1.0;
        v[1] = wg;
        for (int d = 0; d < 3; ++d) {
          v[2 + d] = wg * pos[d];
          v[5 + d] = wa * ga[d];
          v[11 + d] = wb * gb[d];
        }
        if (A.body >= 0) {
          const double* c = bodies[A.body].com;
          const double r[3] = {pos[0] - c[0], pos[1] - c[1], pos[2] - c[2]};
          v[8] = wa * (r[1] * ga[2] - r[2] * ga[1]);
          v[9] = wa * (r[2] * ga[0] - r[0] * ga[2]);
          v[10] = wa * (r[0] * ga[1] - r[1] * ga[0]);
        }
        if (B.body >= 0) {
          const double* c = bodies[B.body].com;
          const double r[3] = {pos[0] - c[0], pos[1] - c[1], pos[2] - c[2]};
          v[14] = wb * (r[1] * gb[2] - r[2] * gb[1]);
          v[15] = wb * (r[2] * gb[0] - r[0] * gb[2]);
          v[16] = wb * (r[0] * gb[1] - r[1] * gb[0]);
        }
      }
    }
    for (int c = 0; c < 17; ++c) {
      const double s = warp_sum(v[c]);
      if (lane == 0) red[warp][c] = s;
    }
    __syncthreads();
    if (warp == 0) {
      for (int c = 0; c < 17; ++c) {
        double s = lane < kContactThreads / 32 ? red[lane][c] : 0.0;
        s = warp_sum(s);
        if (lane == 0) tot[c] = s;
      }
    }
    __syncthreads();
    if (threadIdx.x == 0) {
      ContactCell& C = cells[t];
      const double vol = tot[1];
      if (!(vol > 0.0) || tot[0] == 0.0) {
        C.valid = 0;
      } else {
        const double dt = sc->dt;
        C.valid = 1;
        C.a = P.a;
        C.b = P.b;
        C.volume = vol;
        for (int d = 0; d < 3; ++d) {
          C.center[d] = tot[2 + d] / vol;
          C.f_a[d] = tot[5 + d];
          C.tau_a[d] = tot[8 + d];
          C.f_b[d] = tot[11 + d];
          C.tau_b[d] = tot[14 + d];
        }
        const double fn = fmax(sqrt((C.f_a[0] * C.f_a[0] + C.f_a[1] * C.f_a[1]) + C.f_a[2] * C.f_a[2]), 1e-15);
        const double nrm[3] = {C.f_a[0] / fn, C.f_a[1] / fn, C.f_a[2] / fn};
        for (int r = 0; r < 3; ++r)
          for (int c = 0; c < 3; ++c) C.tproj[r * 3 + c] = (r == c ? 1.0 : 0.0) - nrm[r] * nrm[c];
        double acc_p = 0.0, T[9];
        for (int e = 0; e < 9; ++e) T[e] = 0.0;
        for (int side = 0; side < 2; ++side) {
          const VMDesc& D = side ? B : A;
          if (D.body < 0) continue;
          const Body& M = bodies[D.body];
          const double* f = side ? C.f_b : C.f_a;
          const double* tq = side ? C.tau_b : C.tau_a;
          const double* I = M.inv_inertia_world;
          double It[3];
          for (int r = 0; r < 3; ++r) It[r] = (I[r * 3] * tq[0] + I[r * 3 + 1] * tq[1]) + I[r * 3 + 2] * tq[2];
          acc_p += ((f[0] * f[0] + f[1] * f[1]) + f[2] * f[2]) / M.mass + ((tq[0] * It[0] + tq[1] * It[1]) + tq[2] * It[2]);
          // I / m - [r]x I^-1 [r]x with r = center - com
          const double r[3] = {C.center[0] - M.com[0], C.center[1] - M.com[1], C.center[2] - M.com[2]};
          const double X[9] = {0.0, -r[2], r[1], r[2], 0.0, -r[0], -r[1], r[0], 0.0};
          double XI[9], XIX[9];
          for (int a = 0; a < 3; ++a)
            for (int b = 0; b < 3; ++b)
              XI[a * 3 + b] = (X[a * 3] * I[b] + X[a * 3 + 1] * I[3 + b]) + X[a * 3 + 2] * I[6 + b];
          for (int a = 0; a < 3; ++a)
            for (int b = 0; b < 3; ++b)
              XIX[a * 3 + b] = (XI[a * 3] * X[b] + XI[a * 3 + 1] * X[3 + b]) + XI[a * 3 + 2] * X[6 + b];
          for (int a = 0; a < 3; ++a)
            for (int b = 0; b < 3; ++b) T[a * 3 + b] += (a == b ? 1.0 / M.mass : 0.0) - XIX[a * 3 + b];
        }
        C.acc_p = dt * dt * acc_p;
        double tr = 0.0;
        for (int a = 0; a < 3; ++a) {
          const double row = ((dt * C.tproj[a * 3]) * T[a] + (dt * C.tproj[a * 3 + 1]) * T[3 + a]) +
                             (dt * C.tproj[a * 3 + 2]) * T[6 + a];
          tr += row;
        }
        C.acc_f = 1. / 3. * tr;
      }
    }
    __syncthreads();
  }
}

__device__ __forceinline__ double block_sum_all(double v, double* sh, double* out) {
  const double t = block_sum(v, sh);
  if (threadIdx.x == 0) *out = t;
  __syncthreads();
  const double r = *out;
  __syncthreads();
  return r;
}

// solve_for_p_c (:186-645) with accumulate_extra_forces (:928-965),
// compute_trial_velocities (:967-994), predicted_volume_error (:996-1009),
// predicted_tangential_velocity (:1011-1033), projected_jacobi (:1035-1102)
// and mean_fischer_burmeister (utilities/mod.rs:27-41); one block of 1024
// threads, warp b gathering body b's cells. The reference iterates until the
// merits converge; here at most `sweep_cap` sweeps run (`capped` is set).
constexpr int kContactSolveThreads = 1024;
__global__ void __launch_bounds__(kContactSolveThreads) k_contact_solve(
    Body* __restrict__ bodies, int nb, const ContactCell* __restrict__ cells, ContactScalars* __restrict__ cs,
    int* __restrict__ cell_idx, ContactState* __restrict__ st, const Scalars* __restrict__ sc, int sweep_cap,
    int fixed_sweeps) {
  constexpr double kMu = 0.5, kOmega = 0.5, kMinDiag = 1e-35, kTolP = 1e-6, kTolF = 1e-3;
  __shared__ double sh[32];
  __shared__ double bc;
  __shared__ int scan[32];
  __shared__ int base;
  __shared__ double ef[kMaxBodies][3], et[kMaxBodies][3], vt[kMaxBodies][3], wt[kMaxBodies][3];
  __shared__ int nact[kMaxBodies];
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5, nthreads = blockDim.x;
  const double dt = sc->dt;
  const int ntasks = cs->ntasks;
  // valid cells in task order
  if (tid == 0) base = 0;
  __syncthreads();
  for (int c0 = 0; c0 < ntasks; c0 += nthreads) {
    const int t = c0 + tid;
    const int f = (t < ntasks && cells[t].valid) ? 1 : 0;
    int x = f;
    for (int o = 1; o < 32; o <<= 1) {
      const int y = __shfl_up_sync(0xffffffffu, x, o);
      if (lane >= o) x += y;
    }
    if (lane == 31) scan[warp] = x;
    __syncthreads();
    if (warp == 0) {
      int y = lane < nthreads / 32 ? scan[lane] : 0;
      for (int o = 1; o < 32; o <<= 1) {
        const int z = __shfl_up_sync(0xffffffffu, y, o);
        if (lane >= o) y += z;
      }
      scan[lane] = y;
    }
    __syncthreads();
    const int before = (warp ? scan[warp - 1] : 0) + x - f;
    if (f) cell_idx[base + before] = t;
    __syncthreads();
    if (tid == 0) base += scan[nthreads / 32 - 1];
    __syncthreads();
  }
  const int n = base;
  if (n == 0) {
    if (tid == 0) cs->ncells = 0;
    return;
  }
  for (int c = tid; c < n; c += nthreads) {
    ContactState& S = st[c];
    S.p = S.s_p = S.v_err = S.pj = S.gp = 0.0;
    for (int d = 0; d < 3; ++d) S.lambda[d] = S.s_l[d] = S.v_tang[d] = S.lj[d] = S.gl[d] = 0.0;
  }
  __syncthreads();

  auto accumulate = [&]() {
    if (warp < nb) {
      const int b = warp;
      const bool dyn = bodies[b].dynamic != 0;
      double f[3] = {0.0, 0.0, 0.0}, tq[3] = {0.0, 0.0, 0.0};
      for (int c = lane; c < n; c += 32) {
        const ContactCell& C = cells[cell_idx[c]];
        const ContactState& S = st[c];
        if (C.a != b && C.b != b) continue;
        const bool is_a = C.a == b;
        const double sgn = is_a ? 1.0 : -1.0;
        const double* fv = is_a ? C.f_a : C.f_b;
        const double* tv = is_a ? C.tau_a : C.tau_b;
        for (int d = 0; d < 3; ++d) f[d] += S.p * fv[d] + sgn * S.lambda[d];
        if (dyn) {
          const double* com = bodies[b].com;
          const double r[3] = {C.center[0] - com[0], C.center[1] - com[1], C.center[2] - com[2]};
          const double* l = S.lambda;
          const double cr[3] = {r[1] * l[2] - r[2] * l[1], r[2] * l[0] - r[0] * l[2], r[0] * l[1] - r[1] * l[0]};
          for (int d = 0; d < 3; ++d) tq[d] += S.p * tv[d] + sgn * cr[d];
        }
      }
      for (int d = 0; d < 3; ++d) {
        const double fs = warp_sum(f[d]), ts = warp_sum(tq[d]);
        if (lane == 0) {
          ef[b][d] = fs;
          et[b][d] = ts;
        }
      }
    }
    __syncthreads();
  };
  auto predict = [&]() {
    if (tid < nb) {
      const Body& M = bodies[tid];
      if (!M.dynamic) {
        for (int d = 0; d < 3; ++d) vt[tid][d] = wt[tid][d] = 0.0;
      } else {
        double l[3];
        for (int d = 0; d < 3; ++d) {
          vt[tid][d] = M.v[d] + dt / M.mass * (M.F[d] + ef[tid][d]);
          l[d] = M.L[d] + dt * (M.T[d] + et[tid][d]);
        }
        const double* I = M.inv_inertia_world;
        for (int r = 0; r < 3; ++r) wt[tid][r] = (I[r * 3] * l[0] + I[r * 3 + 1] * l[1]) + I[r * 3 + 2] * l[2];
      }
    }
    __syncthreads();
    for (int c = tid; c < n; c += nthreads) {
      const ContactCell& C = cells[cell_idx[c]];
      ContactState& S = st[c];
      const int a = C.a, b = C.b;
      auto dot3 = [](const double* x, const double* y) { return (x[0] * y[0] + x[1] * y[1]) + x[2] * y[2]; };
      S.v_err = -C.volume + dt * (((dot3(vt[a], C.f_a) + dot3(wt[a], C.tau_a)) + dot3(vt[b], C.f_b)) +
                                  dot3(wt[b], C.tau_b));
      if (bodies[a].dynamic && bodies[b].dynamic) {
        double vr[3];
        const double ra[3] = {C.center[0] - bodies[a].com[0], C.center[1] - bodies[a].com[1],
                              C.center[2] - bodies[a].com[2]};
        const double rb[3] = {C.center[0] - bodies[b].com[0], C.center[1] - bodies[b].com[1],
                              C.center[2] - bodies[b].com[2]};
        const double* wa = wt[a];
        const double* wb = wt[b];
        const double ca[3] = {wa[1] * ra[2] - wa[2] * ra[1], wa[2] * ra[0] - wa[0] * ra[2], wa[0] * ra[1] - wa[1] * ra[0]};
        const double cb[3] = {wb[1] * rb[2] - wb[2] * rb[1], wb[2] * rb[0] - wb[0] * rb[2], wb[0] * rb[1] - wb[1] * rb[0]};
        for (int d = 0; d < 3; ++d) vr[d] = ((vt[a][d] + ca[d]) - vt[b][d]) - cb[d];
        for (int r = 0; r < 3; ++r)
          S.v_tang[r] = (C.tproj[r * 3] * vr[0] + C.tproj[r * 3 + 1] * vr[1]) + C.tproj[r * 3 + 2] * vr[2];
      } else {
        S.v_tang[0] = S.v_tang[1] = S.v_tang[2] = 0.0;
      }
    }
    __syncthreads();
  };
  auto norm3 = [](const double* x) { return sqrt((x[0] * x[0] + x[1] * x[1]) + x[2] * x[2]); };
  auto jacobi = [&]() {
    if (warp < nb) {
      int cnt = 0;
      for (int c = lane; c < n; c += 32) {
        const ContactCell& C = cells[cell_idx[c]];
        if ((C.a == warp || C.b == warp) && (st[c].v_err < 0.0 || st[c].p > 0.0)) ++cnt;
      }
      for (int o = 16; o > 0; o >>= 1) cnt += __shfl_down_sync(0xffffffffu, cnt, o);
      if (lane == 0) nact[warp] = cnt;
    }
    __syncthreads();
    for (int c = tid; c < n; c += nthreads) {
      const ContactCell& C = cells[cell_idx[c]];
      ContactState& S = st[c];
      const double n_max = (double)max(max(nact[C.a], nact[C.b]), 1);
      const double alpha = kOmega / n_max / fmax(C.acc_p, kMinDiag);
      S.pj = fmax(S.p - alpha * S.v_err, 0.0);
      const double lmax = kMu * S.p * norm3(C.f_a);
      double star[3];
      const double af = fmax(C.acc_f, kMinDiag);
      for (int d = 0; d < 3; ++d) star[d] = -S.v_tang[d] / af;
      const double sn = norm3(star);
      if (sn > lmax)
        for (int d = 0; d < 3; ++d) star[d] = lmax * star[d] / sn;
      double ln[3];
      for (int d = 0; d < 3; ++d) ln[d] = S.lambda[d] + kOmega / n_max * star[d];
      const double lnn = norm3(ln);
      for (int d = 0; d < 3; ++d) S.lj[d] = lnn > lmax ? lmax * ln[d] / lnn : ln[d];
    }
    __syncthreads();
  };
  auto converged = [&]() {
    double fp = 0.0, ff = 0.0;
    for (int c = tid; c < n; c += nthreads) {
      const ContactCell& C = cells[cell_idx[c]];
      const ContactState& S = st[c];
      const double pp = S.p * fmax(C.acc_p, kMinDiag);
      fp += fabs(pp + S.v_err - sqrt(pp * pp + S.v_err * S.v_err));
      const double vtn = norm3(S.v_tang);
      const double dev = fmax(C.acc_f, kMinDiag) * (kMu * S.p * norm3(C.f_a) - norm3(S.lambda));
      ff += fabs(vtn + dev - sqrt(vtn * vtn + dev * dev));
    }
    fp = block_sum_all(fp, sh, &bc);
    ff = block_sum_all(ff, sh, &bc);
    return fp / (double)n < kTolP && ff / (double)n < kTolF;
  };

  accumulate();
  predict();
  jacobi();
  double prev = 0.0;
  {
    double g2 = 0.0;
    for (int c = tid; c < n; c += nthreads) {
      ContactState& S = st[c];
      S.gp = -(S.pj - S.p);
      S.s_p = -S.gp;
      g2 += S.gp * S.gp;
      double gl2 = 0.0;
      for (int d = 0; d < 3; ++d) {
        S.gl[d] = -(S.lj[d] - S.lambda[d]);
        S.s_l[d] = -S.gl[d];
      }
      gl2 = (S.gl[0] * S.gl[0] + S.gl[1] * S.gl[1]) + S.gl[2] * S.gl[2];
      g2 += gl2;
      S.p = S.pj;
      for (int d = 0; d < 3; ++d) S.lambda[d] = S.lj[d];
    }
    prev = block_sum_all(g2, sh, &bc);
  }
  accumulate();
  predict();
  int it = 0;
  // fixed_sweeps > 0: exactly that many sweeps, no merit test
  bool done = fixed_sweeps > 0 ? false : converged();
  while (fixed_sweeps > 0 ? it < fixed_sweeps : (!done && it < sweep_cap)) {
    jacobi();
    double g2 = 0.0;
    for (int c = tid; c < n; c += nthreads) {
      ContactState& S = st[c];
      S.gp = -(S.pj - S.p);
      g2 += S.gp * S.gp;
      for (int d = 0; d < 3; ++d) S.gl[d] = -(S.lj[d] - S.lambda[d]);
      g2 += (S.gl[0] * S.gl[0] + S.gl[1] * S.gl[1]) + S.gl[2] * S.gl[2];
    }
    const double gsum = block_sum_all(g2, sh, &bc);
    const double beta = gsum / fmax(prev, DBL_MIN);
    for (int c = tid; c < n; c += nthreads) {
      const ContactCell& C = cells[cell_idx[c]];
      ContactState& S = st[c];
      if (beta > 1.0) {
        S.s_p = 0.0;
        for (int d = 0; d < 3; ++d) S.s_l[d] = 0.0;
        S.p = S.pj;
        for (int d = 0; d < 3; ++d) S.lambda[d] = S.lj[d];
        continue;
      }
      // the friction cone of the iterate before this update (:452-467)
      const double lmax = kMu * S.p * norm3(C.f_a);
      const double p_nncg = S.pj + beta * S.s_p;
      if (p_nncg < 0.0) {
        S.p = S.pj;
        S.s_p = 0.0;
      } else {
        S.p = p_nncg;
        S.s_p = beta * S.s_p - S.gp;
      }
      double ln[3], tp[3];
      for (int d = 0; d < 3; ++d) ln[d] = S.lj[d] + beta * S.s_l[d];
      for (int r = 0; r < 3; ++r) tp[r] = (C.tproj[r * 3] * ln[0] + C.tproj[r * 3 + 1] * ln[1]) + C.tproj[r * 3 + 2] * ln[2];
      if (norm3(tp) > lmax) {
        for (int d = 0; d < 3; ++d) {
          S.lambda[d] = S.lj[d];
          S.s_l[d] = 0.0;
        }
      } else {
        for (int d = 0; d < 3; ++d) {
          S.lambda[d] = tp[d];
          S.s_l[d] = beta * S.s_l[d] - S.gl[d];
        }
      }
    }
    __syncthreads();
    prev = gsum;
    accumulate();
    predict();
    if (fixed_sweeps == 0) done = converged();
    ++it;
  }
  accumulate();
  if (tid < nb && bodies[tid].dynamic) {  // add_force_and_torque (rigid_body_motion.rs:156-159)
    for (int d = 0; d < 3; ++d) {
      bodies[tid].F[d] += ef[tid][d];
      bodies[tid].T[d] += et[tid][d];
    }
  }
  if (tid == 0) {
    cs->ncells = n;
    cs->iterations = it;
    cs->capped = (fixed_sweeps > 0 || done) ? 0 : 1;
  }
}

}  // namespace sph
