// Fluid surface reconstruction for render frames (Fluid::reconstruct_surfaces,
// SL/sph/fluid.rs:212-347, around the third-party splashsurf_lib 0.14.1
// `reconstruct_surface`, restated from its published method). One fluid id
// at a time, on the device:
//   k_surf_density    particle densities rho_i = sum_j m W(x_i - x_j) among
//                     the group's particles (compact support h) -> m / rho_i
//   k_surf_bounds     the group's bounding box (exact f64 min/max)
//   k_surf_levelset   phi(x) = sum_i (m / rho_i) W(x - x_i) at every lattice
//                     point (cube size 0.75 r, aligned to multiples of it)
//   k_surf_edges      lattice edges whose ends straddle the iso value (0.6)
//   k_surf_cells      triangles per cell from the case table
//   k_surf_vertices   linear interpolation on the crossing edges
//   k_surf_triangles  the cells' triangles as vertex indices
//   k_surf_normals    area-weighted vertex normals (fluid.rs:296-323)
// Vertices are numbered by (lattice point, direction) and triangles by cell,
// so the mesh does not depend on thread scheduling (the normals' f64 sums
// do, at the rounding level). Both the particle sums and the lattice sums
// walk the 27 buckets of the step's cell grid (cell size h).
#pragma once

#include "sph_kernels.cuh"

namespace sph {

constexpr double kSurfaceIso = 0.6;  // iso_surface_threshold (fluid.rs:265)
constexpr int kSurfaceMaxTris = 8;   // triangles of one cell case at most

// The marching-cubes case table: for each of the 256 inside patterns of a
// cell's corners (corner c = bx + 2 by + 4 bz), its triangles as local edges
// (edge e = 4 dir + rank of its lower corner among the corners with bit
// `dir` clear). Built on the host (surface_case_table) and passed by value.
struct SurfaceCases {
  unsigned char count[256];
  signed char edges[256][kSurfaceMaxTris * 3];
};

__device__ __forceinline__ double surf_w(double r2, double h) {
  const double q = sqrt(r2) / h;
  const double a = q < 1.0 ? 1.0 - q : 0.0, b = q < 0.5 ? 0.5 - q : 0.0;
  return 16.0 / 3.14159265358979323846 / (h * h * h) * (a * a * a - 4.0 * (b * b * b));
}

// Sum of f(j) W over the group's particles j within h of p (27 buckets).
template <class R, class F>
__device__ __forceinline__ double surf_gather(const double p[3], double h, uint32_t mask,
                                              const uint32_t* __restrict__ start, const R4<R>* __restrict__ xv,
                                              const uint32_t* __restrict__ fid, uint32_t group, F f) {
  const int cx = cell_coord(p[0], h), cy = cell_coord(p[1], h), cz = cell_coord(p[2], h);
  double s = 0.0;
  for (int dz = -1; dz <= 1; ++dz)
    for (int dy = -1; dy <= 1; ++dy)
      for (int dx = -1; dx <= 1; ++dx) {
        const uint32_t k = morton_key(cx + dx, cy + dy, cz + dz, mask);
        const uint32_t e = start[k + 1];
        for (uint32_t j = start[k]; j < e; ++j) {
          if (fid[j] != group) continue;
          const R4<R> x = xv[j];
          const double qx = (double)x.x, qy = (double)x.y, qz = (double)x.z;
          if (!in_range_exact(p[0], p[1], p[2], qx, qy, qz, h)) continue;
          const double rx = p[0] - qx, ry = p[1] - qy, rz = p[2] - qz;
          s += f(j) * surf_w((rx * rx + ry * ry) + rz * rz, h);
        }
      }
  return s;
}

template <class R>
__global__ void __launch_bounds__(kBlock) k_surf_density(int n, const uint32_t* __restrict__ start,
                                                        const R4<R>* __restrict__ xv,
                                                        const uint32_t* __restrict__ fid, uint32_t group,
                                                        double m, double h, uint32_t mask,
                                                        double* __restrict__ vol) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n || fid[i] != group) return;
  const R4<R> x = xv[i];
  const double p[3] = {(double)x.x, (double)x.y, (double)x.z};
  const double rho = surf_gather(p, h, mask, start, xv, fid, group, [&](uint32_t) { return m; });
  vol[i] = m / rho;
}

// Monotonic u64 keys of doubles, so that integer min/max order them.
__device__ __forceinline__ unsigned long long surf_key(double v) {
  const unsigned long long b = (unsigned long long)__double_as_longlong(v);
  return (b >> 63) ? ~b : (b | 0x8000000000000000ull);
}
__host__ __device__ inline double surf_unkey(unsigned long long k) {
  const unsigned long long b = (k >> 63) ? (k & 0x7fffffffffffffffull) : ~k;
  double v;
  memcpy(&v, &b, sizeof v);
  return v;
}

// bounds[0..2] = min keys, bounds[3..5] = max keys, bounds[6] = particle count
template <class R>
__global__ void __launch_bounds__(kBlock) k_surf_bounds(int n, const R4<R>* __restrict__ xv,
                                                       const uint32_t* __restrict__ fid, uint32_t group,
                                                       unsigned long long* __restrict__ bounds) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n || fid[i] != group) return;
  const R4<R> x = xv[i];
  const double p[3] = {(double)x.x, (double)x.y, (double)x.z};
  for (int d = 0; d < 3; ++d) {
    atomicMin(&bounds[d], surf_key(p[d]));
    atomicMax(&bounds[3 + d], surf_key(p[d]));
  }
  atomicAdd(&bounds[6], 1ull);
}

// The lattice: point (i, j, k) at cube * (k0 + (i, j, k)), n points per axis.
struct SurfaceLattice {
  long long k0[3];
  long long n[3];
  double cube;
};
__device__ __forceinline__ double surf_coord(const SurfaceLattice& L, int d, long long k) {
  return L.cube * (double)(L.k0[d] + k);
}

template <class R>
__global__ void __launch_bounds__(kBlock) k_surf_levelset(SurfaceLattice L, long long npoints,
                                                         const uint32_t* __restrict__ start,
                                                         const R4<R>* __restrict__ xv,
                                                         const uint32_t* __restrict__ fid, uint32_t group,
                                                         const double* __restrict__ vol, double h, uint32_t mask,
                                                         double* __restrict__ phi) {
  const long long q = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (q >= npoints) return;
  const long long i = q % L.n[0], j = (q / L.n[0]) % L.n[1], k = q / (L.n[0] * L.n[1]);
  const double p[3] = {surf_coord(L, 0, i), surf_coord(L, 1, j), surf_coord(L, 2, k)};
  phi[q] = surf_gather(p, h, mask, start, xv, fid, group, [&](uint32_t jj) { return vol[jj]; });
}

// flag[3 q + d] = 1 when the edge from point q along d crosses the iso value
__global__ void __launch_bounds__(kBlock) k_surf_edges(SurfaceLattice L, long long npoints,
                                                      const double* __restrict__ phi,
                                                      uint32_t* __restrict__ flag) {
  const long long q = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (q >= npoints) return;
  const long long idx[3] = {q % L.n[0], (q / L.n[0]) % L.n[1], q / (L.n[0] * L.n[1])};
  const long long step[3] = {1, L.n[0], L.n[0] * L.n[1]};
  const bool in = phi[q] > kSurfaceIso;
  for (int d = 0; d < 3; ++d) {
    uint32_t f = 0;
    if (idx[d] + 1 < L.n[d]) f = (in != (phi[q + step[d]] > kSurfaceIso)) ? 1u : 0u;
    flag[3 * q + d] = f;
  }
}

__device__ __forceinline__ int surf_case(const SurfaceLattice& L, const double* __restrict__ phi, long long c,
                                         long long corner_q[8]) {
  const long long nc0 = L.n[0] - 1, nc1 = L.n[1] - 1;
  const long long i = c % nc0, j = (c / nc0) % nc1, k = c / (nc0 * nc1);
  int code = 0;
  for (int b = 0; b < 8; ++b) {
    const long long q = (i + (b & 1)) + L.n[0] * ((j + ((b >> 1) & 1)) + L.n[1] * (k + ((b >> 2) & 1)));
    corner_q[b] = q;
    if (phi[q] > kSurfaceIso) code |= 1 << b;
  }
  return code;
}

__global__ void __launch_bounds__(kBlock) k_surf_cells(SurfaceLattice L, long long ncells,
                                                      const double* __restrict__ phi, SurfaceCases T,
                                                      uint32_t* __restrict__ tris) {
  const long long c = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= ncells) return;
  long long cq[8];
  tris[c] = T.count[surf_case(L, phi, c, cq)];
}

// Vertex of a crossing edge (q, d): its id is the exclusive scan of the
// crossing flags (which the scan clears, so the crossing is tested again).
__global__ void __launch_bounds__(kBlock) k_surf_vertices(SurfaceLattice L, long long nedges,
                                                         const double* __restrict__ phi,
                                                         const uint32_t* __restrict__ vid,
                                                         double* __restrict__ vtx) {
  const long long e = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (e >= nedges) return;
  const long long q = e / 3;
  const int d = (int)(e % 3);
  const long long idx[3] = {q % L.n[0], (q / L.n[0]) % L.n[1], q / (L.n[0] * L.n[1])};
  const long long step[3] = {1, L.n[0], L.n[0] * L.n[1]};
  if (idx[d] + 1 >= L.n[d]) return;
  const double fa = phi[q], fb = phi[q + step[d]];
  if ((fa > kSurfaceIso) == (fb > kSurfaceIso)) return;
  const double t = (kSurfaceIso - fa) / (fb - fa);
  double* v = vtx + 6 * (size_t)vid[e];
  for (int c = 0; c < 3; ++c) {
    const double a = surf_coord(L, c, idx[c]);
    const double b = surf_coord(L, c, idx[c] + (c == d ? 1 : 0));
    v[c] = a + t * (b - a);
    v[3 + c] = 0.0;
  }
}

__global__ void __launch_bounds__(kBlock) k_surf_triangles(SurfaceLattice L, long long ncells,
                                                          const double* __restrict__ phi, SurfaceCases T,
                                                          const uint32_t* __restrict__ tri_off,
                                                          const uint32_t* __restrict__ vid,
                                                          uint32_t* __restrict__ idx_out) {
  const long long c = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= ncells) return;
  long long cq[8];
  const int code = surf_case(L, phi, c, cq);
  const int nt = T.count[code];
  uint32_t* out = idx_out + 3 * (size_t)tri_off[c];
  for (int t = 0; t < 3 * nt; ++t) {
    const int e = T.edges[code][t];
    const int d = e >> 2;
    // the lower corner of local edge e: rank (e & 3) among corners with bit d clear
    int rank = e & 3, lo = 0;
    for (int b = 0; b < 8; ++b)
      if (!((b >> d) & 1) && rank-- == 0) {
        lo = b;
        break;
      }
    out[t] = vid[3 * cq[lo] + d];
  }
}

__global__ void __launch_bounds__(kBlock) k_surf_normals(long long ntris, const uint32_t* __restrict__ idx,
                                                        double* __restrict__ vtx) {
  const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= ntris) return;
  const double* p0 = vtx + 6 * (size_t)idx[3 * t];
  const double* p1 = vtx + 6 * (size_t)idx[3 * t + 1];
  const double* p2 = vtx + 6 * (size_t)idx[3 * t + 2];
  const double e1[3] = {p1[0] - p0[0], p1[1] - p0[1], p1[2] - p0[2]};
  const double e2[3] = {p2[0] - p0[0], p2[1] - p0[1], p2[2] - p0[2]};
  const double fn[3] = {e1[1] * e2[2] - e1[2] * e2[1], e1[2] * e2[0] - e1[0] * e2[2], e1[0] * e2[1] - e1[1] * e2[0]};
  for (int c = 0; c < 3; ++c) {
    double* nrm = vtx + 6 * (size_t)idx[3 * t + c] + 3;
    atomicAdd(&nrm[0], fn[0]);
    atomicAdd(&nrm[1], fn[1]);
    atomicAdd(&nrm[2], fn[2]);
  }
}

__global__ void __launch_bounds__(kBlock) k_surf_normalize(long long nverts, double* __restrict__ vtx) {
  const long long v = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (v >= nverts) return;
  double* n = vtx + 6 * (size_t)v + 3;
  const double len = sqrt(n[0] * n[0] + n[1] * n[1] + n[2] * n[2]);
  if (len > 1e-10) {
    n[0] /= len;
    n[1] /= len;
    n[2] /= len;
  }
}

// Host: the case table, from the same face rule the oracle applies per cell:
// on each face (corners counter-clockwise seen from outside) a run of inside
// corners gives a segment from the edge entering it to the edge leaving it;
// the segments chain through shared edges into loops, each loop is fanned
// from its first edge, loops start at their smallest edge.
inline SurfaceCases surface_case_table() {
  auto bit = [](int c, int d) { return (c >> d) & 1; };
  auto edge_of = [&](int a, int b) {
    const int x = a ^ b, d = x == 1 ? 0 : (x == 2 ? 1 : 2), lo = a < b ? a : b;
    int rank = 0;
    for (int c = 0; c < lo; ++c)
      if (!bit(c, d)) ++rank;
    return 4 * d + rank;
  };
  int faces[6][4];
  for (int a = 0, f = 0; a < 3; ++a)
    for (int s = 0; s < 2; ++s, ++f) {
      const int u = (a + 1) % 3, v = (a + 2) % 3;
      const int uv[4][2] = {{0, 0}, {1, 0}, {1, 1}, {0, 1}};
      for (int k = 0; k < 4; ++k) {
        const int kk = s == 1 ? k : 3 - k;
        faces[f][k] = (s << a) | (uv[kk][0] << u) | (uv[kk][1] << v);
      }
    }
  SurfaceCases T;
  memset(&T, 0, sizeof T);
  for (int code = 0; code < 256; ++code) {
    int next[12];
    bool has[12] = {false}, used[12] = {false};
    for (int f = 0; f < 6; ++f) {
      int cross[4], enter[4], nc = 0;
      for (int k = 0; k < 4; ++k) {
        const int a = faces[f][k], b = faces[f][(k + 1) % 4];
        const bool ia = (code >> a) & 1, ib = (code >> b) & 1;
        if (ia != ib) {
          cross[nc] = edge_of(a, b);
          enter[nc] = ib ? 1 : 0;
          ++nc;
        }
      }
      for (int k = 0; k < nc; ++k)
        if (enter[k]) {
          next[cross[k]] = cross[(k + 1) % nc];
          has[cross[k]] = true;
        }
    }
    int nt = 0;
    for (int e = 0; e < 12; ++e) {
      if (!has[e] || used[e]) continue;
      int loop[12], nl = 0, cur = e;
      while (!used[cur]) {
        used[cur] = true;
        loop[nl++] = cur;
        cur = next[cur];
      }
      for (int t = 1; t + 1 < nl; ++t) {
        if (nt >= kSurfaceMaxTris) throw std::logic_error("surface case table overflow");
        T.edges[code][3 * nt] = (signed char)loop[0];
        T.edges[code][3 * nt + 1] = (signed char)loop[t];
        T.edges[code][3 * nt + 2] = (signed char)loop[t + 1];
        ++nt;
      }
    }
    T.count[code] = (unsigned char)nt;
  }
  return T;
}

}  // namespace sph
