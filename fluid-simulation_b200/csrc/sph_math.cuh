// Device math for the SPH step engine: packed particle vectors, the cubic
// B-spline kernel, the reference's exact neighbor-range predicate and the
// Morton cell key. Every kernel is templated on the state precision R
// (float for production, double for the precision-study twin).
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

namespace sph {

// 4-wide packed vector: {x, y, z, w}. The w lane carries a per-particle
// scalar that the same passes need (volume for positions, mass for
// velocities), so one 16-byte (f32) load brings both.
template <class R>
struct alignas(4 * sizeof(R)) R4 {
  R x, y, z, w;
};

// 2-wide packed pair (the second record of a sweep gather).
template <class R>
struct alignas(2 * sizeof(R)) R2 {
  R x, y;
};

template <class R>
struct V3 {
  R x, y, z;
};

template <class R>
__host__ __device__ __forceinline__ V3<R> v3(R x, R y, R z) { return {x, y, z}; }
template <class R>
__host__ __device__ __forceinline__ V3<R> xyz(const R4<R>& a) { return {a.x, a.y, a.z}; }
template <class R>
__host__ __device__ __forceinline__ V3<R> operator+(V3<R> a, V3<R> b) { return {a.x + b.x, a.y + b.y, a.z + b.z}; }
template <class R>
__host__ __device__ __forceinline__ V3<R> operator-(V3<R> a, V3<R> b) { return {a.x - b.x, a.y - b.y, a.z - b.z}; }
template <class R>
__host__ __device__ __forceinline__ V3<R> operator*(R s, V3<R> a) { return {s * a.x, s * a.y, s * a.z}; }
template <class R>
__host__ __device__ __forceinline__ V3<R>& operator+=(V3<R>& a, V3<R> b) { a.x += b.x; a.y += b.y; a.z += b.z; return a; }
template <class R>
__host__ __device__ __forceinline__ R dot(V3<R> a, V3<R> b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
template <class R>
__host__ __device__ __forceinline__ V3<R> cross(V3<R> a, V3<R> b) {
  return {a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x};
}

// ---------------------------------------------------------------------------
// Cubic B-spline kernel (reference: simulation_lib/src/sph/kernel/mod.rs:17-46,
// kernel/cubic_spline.rs:7-17). h is the support radius; alpha = 16/pi.
//   W(r)    = alpha/h^3 * w(q),  w(q)  = (1-q)_+^3 - 4 (1/2-q)_+^3
//   gradW(r)= alpha/h^4 * r/|r| * w'(q), w'(q) = -3(1-q)_+^2 + 12 (1/2-q)_+^2
// ---------------------------------------------------------------------------
template <class R>
struct KernelConst {
  R h, inv_h, cw, cg;  // cw = alpha/h^3, cg = alpha/h^4
};

template <class R>
__host__ KernelConst<R> make_kernel_const(double h) {
  const double alpha = 16.0 / 3.14159265358979323846;
  KernelConst<R> k;
  k.h = (R)h;
  k.inv_h = (R)(1.0 / h);
  k.cw = (R)(alpha / (h * h * h));
  k.cg = (R)(alpha / (h * h * h * h));
  return k;
}

template <class R>
__device__ __forceinline__ R sq(R x) { return x * x; }

// W from the squared distance; zero outside the support.
template <class R>
__device__ __forceinline__ R kernel_w_r2(R r2, const KernelConst<R>& k) {
  R q = sqrt(r2) * k.inv_h;
  R a = q < R(1) ? R(1) - q : R(0);
  R b = q < R(0.5) ? R(0.5) - q : R(0);
  return k.cw * (a * a * a - R(4) * (b * b * b));
}

// Scalar factor f with gradW(r) = f * r (zero at r = 0 and outside support).
template <class R>
__device__ __forceinline__ R kernel_grad_factor(R r2, const KernelConst<R>& k) {
  if (!(r2 > R(0))) return R(0);
  R rn = sqrt(r2);
  R q = rn * k.inv_h;
  R a = q < R(1) ? R(1) - q : R(0);
  R b = q < R(0.5) ? R(0.5) - q : R(0);
  R dw = R(-3) * (a * a) + R(12) * (b * b);
  return k.cg * dw / rn;
}

// f32: reciprocal square root instead of IEEE sqrt + division (relative
// error ~1e-7, far inside the f32 state's tolerance); f64 keeps the exact form.
template <>
__device__ __forceinline__ float kernel_grad_factor<float>(float r2, const KernelConst<float>& k) {
  if (!(r2 > 0.f)) return 0.f;
  const float inv = rsqrtf(r2);
  const float q = r2 * inv * k.inv_h;
  const float a = q < 1.f ? 1.f - q : 0.f;
  const float b = q < 0.5f ? 0.5f - q : 0.f;
  return k.cg * (-3.f * (a * a) + 12.f * (b * b)) * inv;
}

// The gradient factor without its constant: gradW(r) = cg * grad_core(r2) * r,
// grad_core = w'(q) / |r| with w'(q) = 12 (1/2-q)_+^2 - 3 (1-q)_+^2 (zero at
// r = 0 and outside the support). Sums of grad_core terms are scaled by cg
// once, after the loop.
template <class R>
__device__ __forceinline__ R grad_core(R r2, R inv_h) {
  const R rn = sqrt(r2);
  const R q = rn * inv_h;
  const R a = q < R(1) ? R(1) - q : R(0);
  const R b = q < R(0.5) ? R(0.5) - q : R(0);
  return r2 > R(0) ? (R(12) * (b * b) - R(3) * (a * a)) / rn : R(0);
}
// f32: one approximate reciprocal square root (relative error ~2^-23, far
// inside the f32 state's tolerance) and no branch.
template <>
__device__ __forceinline__ float grad_core<float>(float r2, float inv_h) {
  float inv;
  asm("rsqrt.approx.ftz.f32 %0, %1;" : "=f"(inv) : "f"(r2));
  inv = r2 > 0.f ? inv : 0.f;
  const float q = r2 * inv * inv_h;
  const float a = fmaxf(1.f - q, 0.f), b = fmaxf(0.5f - q, 0.f);
  return fmaf(12.f * b, b, -3.f * a * a) * inv;
}

// The same factor in its piecewise form, divided by -3: with q = |r|/h,
// w'(q) = 9q^2 - 6q for q < 1/2 and -3 (1-q)^2 for 1/2 <= q < 1, so
// grad_core / -3 = (2 - 3q) / h, resp. (1-q)^2 / |r| (no division in f32;
// the caller scales its sums by -3 cg once). Its product with r is zero at
// r = 0.
template <class R>
__device__ __forceinline__ R grad_piecewise(R r2, R inv_h) {
  const R rn = sqrt(r2);
  const R q = rn * inv_h;
  if (q < R(0.5)) return (R(2) - R(3) * q) * inv_h;
  const R t = R(1) - q;
  return q < R(1) ? t * t / rn : R(0);
}
// f32: r2 is clamped away from 0 so that the self pair (r = 0) gives a finite
// factor; one approximate reciprocal square root.
template <>
__device__ __forceinline__ float grad_piecewise<float>(float r2, float inv_h) {
  const float r2c = fmaxf(r2, 1e-30f);
  float inv;
  asm("rsqrt.approx.ftz.f32 %0, %1;" : "=f"(inv) : "f"(r2c));
  const float q = r2c * inv * inv_h;
  const float t = fmaxf(1.f - q, 0.f);
  return q < 0.5f ? fmaf(-3.f * inv_h, q, 2.f * inv_h) : t * t * inv;
}

// Both W and the gradient factor from one square root.
template <class R>
__device__ __forceinline__ void kernel_w_and_grad(R r2, const KernelConst<R>& k, R& w, R& f) {
  R rn = sqrt(r2);
  R q = rn * k.inv_h;
  R a = q < R(1) ? R(1) - q : R(0);
  R b = q < R(0.5) ? R(0.5) - q : R(0);
  w = k.cw * (a * a * a - R(4) * (b * b * b));
  R dw = R(-3) * (a * a) + R(12) * (b * b);
  f = rn > R(0) ? k.cg * dw / rn : R(0);
}

// ---------------------------------------------------------------------------
// The reference's neighbor predicate, bit for bit: f64 difference of the two
// positions, squared norm summed as (dx^2 + dy^2) + dz^2 without contraction,
// IEEE sqrt, strict `< range` (spatial_hashing.rs:94, neighbor_search/mod.rs:31).
// ---------------------------------------------------------------------------
__device__ __forceinline__ bool in_range_exact(double ax, double ay, double az, double bx,
                                               double by, double bz, double range) {
  double dx = __dsub_rn(ax, bx), dy = __dsub_rn(ay, by), dz = __dsub_rn(az, bz);
  double s = __dadd_rn(__dadd_rn(__dmul_rn(dx, dx), __dmul_rn(dy, dy)), __dmul_rn(dz, dz));
  return __dsqrt_rn(s) < range;
}

// Fast pre-filter in the state precision with a relative guard band; only
// pairs inside the band fall back to the exact f64 predicate. For R = float
// the f32 squared distance is within a few ulp of the exact value, far inside
// the 1e-5 band.
template <class R>
__device__ __forceinline__ bool in_range(const R4<R>& a, const R4<R>& b, double range,
                                         R range2_lo, R range2_hi) {
  R dx = a.x - b.x, dy = a.y - b.y, dz = a.z - b.z;
  R r2 = dx * dx + dy * dy + dz * dz;
  if (r2 < range2_lo) return true;
  if (r2 > range2_hi) return false;
  return in_range_exact((double)a.x, (double)a.y, (double)a.z, (double)b.x, (double)b.y,
                        (double)b.z, range);
}

// Cell of a position: floor(p / cell_size) in f64, saturated to i32 like
// Rust's `as i32` (spatial_hashing.rs:40-46).
__device__ __forceinline__ int cell_coord(double p, double cell_size) {
  double f = floor(__ddiv_rn(p, cell_size));
  if (f != f) return 0;
  if (f >= 2147483647.0) return 2147483647;
  if (f <= -2147483648.0) return (int)0x80000000;
  return (int)f;
}

// Morton key of the low `bits` bits of each cell coordinate. Cells that wrap
// onto the same key share a bucket; the distance test separates them. Any
// two cells of one 3x3x3 stencil get distinct keys when bits >= 2.
__device__ __forceinline__ uint32_t spread3(uint32_t v) {
  v &= 0x3ff;
  v = (v | (v << 16)) & 0x030000FF;
  v = (v | (v << 8)) & 0x0300F00F;
  v = (v | (v << 4)) & 0x030C30C3;
  v = (v | (v << 2)) & 0x09249249;
  return v;
}
__device__ __forceinline__ uint32_t morton_key(int cx, int cy, int cz, uint32_t mask) {
  return spread3((uint32_t)cx & mask) | (spread3((uint32_t)cy & mask) << 1) |
         (spread3((uint32_t)cz & mask) << 2);
}

}  // namespace sph
