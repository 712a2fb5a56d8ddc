// GPU builder of a boundary's volume-map fields (reference:
// sph/boundary_handling/volume_map_boundary.rs:1547-1741 and
// utilities/discretization.rs:33-245): the mesh signed-distance field and the
// volume map, each a cubic-serendipity node lattice with the reference's
// pruning. Setup-time work, but at the million-particle scale the reference
// spends CPU-hours here (27,000 quadrature points per volume-map node), so it
// runs on the device: one block per volume-map node, the Gauss-Legendre
// quadrature nested exactly like the reference (r outer, theta, phi inner)
// with every level summed in node order.
#pragma once

#include <cmath>
#include <vector>

#include "sph_kernels.cuh"

namespace sph {

// ---- mesh signed distance --------------------------------------------------------
// Per triangle: vertices (9), unit face normal (3), pseudo-normals of its
// edges ab, bc, ca (9, sums of the adjacent face normals) and of its vertices
// (9, angle-weighted sums of the incident face normals).
struct MeshDev {
  const double* tri;
  const double* fn;
  const double* en;
  const double* vn;
  int nt;
};

__device__ __forceinline__ double dot3(const double* a, const double* b) {
  return add_(add_(mul_(a[0], b[0]), mul_(a[1], b[1])), mul_(a[2], b[2]));
}

// Closest point on triangle abc to p (Ericson, Real-Time Collision Detection
// 5.1.5); feature: 0 face, 1..3 vertex a,b,c, 4 edge ab, 5 edge bc, 6 edge ca.
__device__ void closest_on_tri(const double* p, const double* a, const double* b, const double* c,
                               double* q, int& feat) {
  double ab[3], ac[3], ap[3];
  for (int d = 0; d < 3; ++d) { ab[d] = sub_(b[d], a[d]); ac[d] = sub_(c[d], a[d]); ap[d] = sub_(p[d], a[d]); }
  const double d1 = dot3(ab, ap), d2 = dot3(ac, ap);
  if (d1 <= 0 && d2 <= 0) { feat = 1; for (int d = 0; d < 3; ++d) q[d] = a[d]; return; }
  double bp[3];
  for (int d = 0; d < 3; ++d) bp[d] = sub_(p[d], b[d]);
  const double d3 = dot3(ab, bp), d4 = dot3(ac, bp);
  if (d3 >= 0 && d4 <= d3) { feat = 2; for (int d = 0; d < 3; ++d) q[d] = b[d]; return; }
  const double vc = sub_(mul_(d1, d4), mul_(d3, d2));
  if (vc <= 0 && d1 >= 0 && d3 <= 0) {
    feat = 4;
    const double v = div_(d1, sub_(d1, d3));
    for (int d = 0; d < 3; ++d) q[d] = add_(a[d], mul_(ab[d], v));
    return;
  }
  double cp[3];
  for (int d = 0; d < 3; ++d) cp[d] = sub_(p[d], c[d]);
  const double d5 = dot3(ab, cp), d6 = dot3(ac, cp);
  if (d6 >= 0 && d5 <= d6) { feat = 3; for (int d = 0; d < 3; ++d) q[d] = c[d]; return; }
  const double vb = sub_(mul_(d5, d2), mul_(d1, d6));
  if (vb <= 0 && d2 >= 0 && d6 <= 0) {
    feat = 6;
    const double w = div_(d2, sub_(d2, d6));
    for (int d = 0; d < 3; ++d) q[d] = add_(a[d], mul_(ac[d], w));
    return;
  }
  const double va = sub_(mul_(d3, d6), mul_(d5, d4));
  if (va <= 0 && sub_(d4, d3) >= 0 && sub_(d5, d6) >= 0) {
    feat = 5;
    const double w = div_(sub_(d4, d3), add_(sub_(d4, d3), sub_(d5, d6)));
    for (int d = 0; d < 3; ++d) q[d] = add_(b[d], mul_(sub_(c[d], b[d]), w));
    return;
  }
  feat = 0;
  const double denom = div_(1.0, add_(add_(va, vb), vc));
  const double v = mul_(vb, denom), w = mul_(vc, denom);
  for (int d = 0; d < 3; ++d) q[d] = add_(add_(a[d], mul_(ab[d], v)), mul_(ac[d], w));
}

// Signed distance: negative where p - proj points against the closest
// feature's pseudo-normal (volume_map_boundary.rs:1655-1671).
__device__ double mesh_sd(const MeshDev& M, const double* p) {
  double best = INFINITY, bq[3] = {0, 0, 0};
  int bt = 0, bf = 0;
  for (int t = 0; t < M.nt; ++t) {
    const double* T = M.tri + 9 * t;
    double q[3];
    int f;
    closest_on_tri(p, T, T + 3, T + 6, q, f);
    const double dx = sub_(p[0], q[0]), dy = sub_(p[1], q[1]), dz = sub_(p[2], q[2]);
    const double d2 = add_(add_(mul_(dx, dx), mul_(dy, dy)), mul_(dz, dz));
    if (d2 < best) { best = d2; bt = t; bf = f; bq[0] = q[0]; bq[1] = q[1]; bq[2] = q[2]; }
  }
  const double* n;
  if (bf == 0) n = M.fn + 3 * bt;
  else if (bf <= 3) n = M.vn + 9 * bt + 3 * (bf - 1);
  else n = M.en + 9 * bt + 3 * (bf - 4);
  const double diff[3] = {sub_(p[0], bq[0]), sub_(p[1], bq[1]), sub_(p[2], bq[2])};
  const double dist = __dsqrt_rn(dot3(diff, diff));
  return dot3(diff, n) < 0.0 ? -dist : dist;
}

// ---- lattice helpers ----------------------------------------------------------------
struct LatticeDesc {
  double xmin[3], dx;
  long long n[3], NX, NY, NZ;
};

// Nodes of the lattice that belong to a cell: at most one coordinate off the
// corner positions (multiples of 3).
__device__ __forceinline__ bool is_cell_node(long long kx, long long ky, long long kz) {
  return (int)(kx % 3 != 0) + (int)(ky % 3 != 0) + (int)(kz % 3 != 0) <= 1;
}

__global__ void k_sdf_nodes(MeshDev M, LatticeDesc L, double* __restrict__ raw) {
  const long long k = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  const long long total = L.NX * L.NY * L.NZ;
  if (k >= total) return;
  const long long kx = k % L.NX, ky = (k / L.NX) % L.NY, kz = k / (L.NX * L.NY);
  if (!is_cell_node(kx, ky, kz)) { raw[k] = NAN; return; }
  // discretization.rs:160-166: x_min + key / 3 * dx
  const double p[3] = {add_(L.xmin[0], mul_(div_((double)kx, 3.0), L.dx)),
                       add_(L.xmin[1], mul_(div_((double)ky, 3.0), L.dx)),
                       add_(L.xmin[2], mul_(div_((double)kz, 3.0), L.dx))};
  raw[k] = mesh_sd(M, p);
}

// Pruning (discretization.rs:186-236): a cell keeps its 32 nodes when all are
// valid and they are not all below `lo` (has_lo) nor all above `hi` (has_hi).
__global__ void k_prune_cells(LatticeDesc L, const double* __restrict__ raw, int has_lo, double lo,
                              int has_hi, double hi, unsigned char* __restrict__ keep) {
  const long long c = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  const long long ncell = L.n[0] * L.n[1] * L.n[2];
  if (c >= ncell) return;
  const long long cx = c % L.n[0], cy = (c / L.n[0]) % L.n[1], cz = c / (L.n[0] * L.n[1]);
  long long idx[32];
  bool all_lo = true, all_hi = true;
  for (int a = 0; a < 32; ++a) {
    idx[a] = ((3 * cz + c_ser_off[a][2]) * L.NY + (3 * cy + c_ser_off[a][1])) * L.NX + 3 * cx + c_ser_off[a][0];
    const double v = raw[idx[a]];
    if (v != v) return;
    if (!(v < lo)) all_lo = false;
    if (!(v > hi)) all_hi = false;
  }
  if ((has_lo && all_lo) || (has_hi && all_hi)) return;
  for (int a = 0; a < 32; ++a) keep[idx[a]] = 1;
}

__global__ void k_apply_keep(long long total, const double* __restrict__ raw,
                             const unsigned char* __restrict__ keep, double* __restrict__ out) {
  const long long k = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= total) return;
  out[k] = keep[k] ? raw[k] : NAN;
}

// ---- volume map ---------------------------------------------------------------------
constexpr int kMaxGL = 64;
__constant__ double c_gl_x[kMaxGL];
__constant__ double c_gl_w[kMaxGL];

// Cubic extension function gamma*(sd) (volume_map_boundary.rs:1717-1727).
__device__ __forceinline__ double cubic_extension(double sd, double r) {
  if (sd >= r) return 0.0;
  if (sd <= 0.0) return 1.0;
  const double q = div_(sd, r);
  const double a = sub_(1.0, q), b = q < 0.5 ? sub_(0.5, q) : 0.0;
  return div_(sub_(mul_(mul_(a, a), a), mul_(4.0, mul_(mul_(b, b), b))), 0.5);
}

// One block per volume-map node: SDFnWrapper::volume (volume_map_boundary.rs:
// 1684-1715) with gauss_legendre_integrate_ball (discretization.rs:33-79),
// clamped to [0, 4/3 pi r^3] (:1616). Absent (NaN) when a quadrature point
// leaves the evaluable SDF.
__global__ void __launch_bounds__(256) k_volume_map_nodes(DevField sdf, LatticeDesc L, double r,
                                                          int deg, double* __restrict__ raw) {
  const long long k = blockIdx.x;
  const long long kx = k % L.NX, ky = (k / L.NX) % L.NY, kz = k / (L.NX * L.NY);
  __shared__ double inner[kMaxGL * kMaxGL];
  __shared__ double mid[kMaxGL];
  __shared__ int state;  // 0 integrate, 1 value set, 2 error
  __shared__ double value;
  __shared__ int err;
  const double c[3] = {add_(L.xmin[0], mul_(div_((double)kx, 3.0), L.dx)),
                       add_(L.xmin[1], mul_(div_((double)ky, 3.0), L.dx)),
                       add_(L.xmin[2], mul_(div_((double)kz, 3.0), L.dx))};
  const double PI = 3.14159265358979323846;
  const double ball = 4.0 / 3.0 * PI * (r * r * r);
  if (threadIdx.x == 0) {
    err = 0;
    state = 0;
    if (!is_cell_node(kx, ky, kz)) {
      state = 2;
    } else {
      double sdc;
      if (!ser_function(sdf, c[0], c[1], c[2], sdc)) { state = 1; value = 0.0; }
      else if (sdc >= 2.0 * r) { state = 1; value = 0.0; }
      else if (sdc <= -r) { state = 1; value = ball; }
    }
  }
  __syncthreads();
  if (state != 0) {
    if (threadIdx.x == 0) raw[k] = state == 1 ? fmin(fmax(value, 0.0), ball) : NAN;
    return;
  }
  // innermost integrals over phi for every (r_i, theta_j) pair
  for (int pj = threadIdx.x; pj < deg * deg; pj += blockDim.x) {
    const int i = pj / deg, j = pj % deg;
    const double rr = mul_(0.5, add_(mul_(r, c_gl_x[i]), r));
    const double th = mul_(0.5, add_(mul_(PI, c_gl_x[j]), PI));
    const double st = sin(th), ct = cos(th);
    double s = 0.0;
    for (int q = 0; q < deg; ++q) {
      const double ph = mul_(0.5, add_(mul_(2.0 * PI, c_gl_x[q]), 2.0 * PI));
      const double rs = mul_(rr, st);
      const double p0 = add_(c[0], mul_(rs, cos(ph)));
      const double p1 = add_(c[1], mul_(rs, sin(ph)));
      const double p2 = add_(c[2], mul_(rr, ct));
      double sd;
      if (!ser_function(sdf, p0, p1, p2, sd)) { err = 1; break; }
      s = add_(s, mul_(cubic_extension(sd, r), c_gl_w[q]));
    }
    inner[pj] = mul_(mul_(0.5, 2.0 * PI), s);
  }
  __syncthreads();
  if (threadIdx.x < deg) {
    const int i = threadIdx.x;
    double s = 0.0;
    for (int j = 0; j < deg; ++j) {
      const double th = mul_(0.5, add_(mul_(PI, c_gl_x[j]), PI));
      s = add_(s, mul_(mul_(sin(th), inner[i * deg + j]), c_gl_w[j]));
    }
    mid[i] = mul_(mul_(0.5, PI), s);
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    if (err) {
      raw[k] = NAN;
      return;
    }
    double s = 0.0;
    for (int i = 0; i < deg; ++i) {
      const double rr = mul_(0.5, add_(mul_(r, c_gl_x[i]), r));
      s = add_(s, mul_(mul_(mul_(rr, rr), mid[i]), c_gl_w[i]));
    }
    raw[k] = fmin(fmax(mul_(mul_(0.5, r), s), 0.0), ball);
  }
}

// Gauss-Legendre nodes and weights on [-1, 1] (Newton iteration on P_n).
inline void gauss_legendre_nodes(int deg, std::vector<double>& x, std::vector<double>& w) {
  const double PI = 3.14159265358979323846;
  x.assign(deg, 0);
  w.assign(deg, 0);
  for (int i = 0; i < deg; ++i) {
    double z = std::cos(PI * (i + 0.75) / (deg + 0.5));
    for (int it = 0; it < 100; ++it) {
      double p1 = 1, p2 = 0;
      for (int j = 1; j <= deg; ++j) {
        const double p3 = p2;
        p2 = p1;
        p1 = ((2.0 * j - 1) * z * p2 - (j - 1.0) * p3) / j;
      }
      const double pp = deg * (z * p1 - p2) / (z * z - 1.0);
      const double z1 = z;
      z = z1 - p1 / pp;
      if (std::fabs(z - z1) < 1e-16) break;
    }
    double p1 = 1, p2 = 0;
    for (int j = 1; j <= deg; ++j) {
      const double p3 = p2;
      p2 = p1;
      p1 = ((2.0 * j - 1) * z * p2 - (j - 1.0) * p3) / j;
    }
    const double pp = deg * (z * p1 - p2) / (z * z - 1.0);
    x[i] = -z;
    w[i] = 2.0 / ((1.0 - z * z) * pp * pp);
  }
}

}  // namespace sph
