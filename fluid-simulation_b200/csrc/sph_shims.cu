// Per-trait compatibility entry points of the C ABI: the reference's trait
// seams pass host arrays on every call (neighbor_search/mod.rs:18-28,
// kernel/mod.rs:17-46), so these upload, run one kernel and download. They
// exist for per-trait parity checks; the device-resident System is the
// production path.
#include <algorithm>
#include <cmath>
#include <string>
#include <vector>

#include "../../include/sphgpu.h"
#include "sph_math.cuh"

namespace sph {
extern thread_local std::string g_last_error;
}

namespace {

std::string& g_err_ref() { return sph::g_last_error; }
#define g_err g_err_ref()

struct ShimError {
  int code;
  std::string msg;
};

void check(cudaError_t e, const char* what) {
  if (e != cudaSuccess)
    throw ShimError{e == cudaErrorMemoryAllocation ? SPH_ERR_OOM : SPH_ERR_CUDA,
                    std::string(what) + ": " + cudaGetErrorString(e)};
}

template <class T>
struct Buf {
  T* p = nullptr;
  explicit Buf(size_t n) {
    if (n) check(cudaMalloc((void**)&p, n * sizeof(T)), "cudaMalloc");
  }
  ~Buf() {
    if (p) cudaFree(p);
  }
};

template <class F>
int run(int device, F&& f) {
  try {
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0)
      throw ShimError{SPH_ERR_CUDA, "no CUDA device available"};
    if (device < 0 || device >= ndev) throw ShimError{SPH_ERR_INVALID, "device ordinal out of range"};
    check(cudaSetDevice(device), "cudaSetDevice");
    return f();
  } catch (const ShimError& e) {
    g_err = e.msg;
    return e.code;
  } catch (const std::exception& e) {
    g_err = e.what();
    return SPH_ERR_OOM;
  }
}

// Neighbor enumeration over a cell-sorted sample set: stencil order dx, dy, dz
// (outer to inner) and ascending sample index inside a cell, the order of
// SpatialHashing::get_particles_in_range (spatial_hashing.rs:75-103).
__global__ void k_find_samples(int n, const double* __restrict__ pos, const double* __restrict__ samp,
                               const uint32_t* __restrict__ sorted_idx, const uint32_t* __restrict__ start,
                               uint32_t mask, double cell, double range, uint32_t* __restrict__ counts,
                               const uint64_t* __restrict__ offs, uint32_t* __restrict__ out) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const double px = pos[3 * i], py = pos[3 * i + 1], pz = pos[3 * i + 2];
  const int cx = sph::cell_coord(px, cell), cy = sph::cell_coord(py, cell), cz = sph::cell_coord(pz, cell);
  uint32_t c = 0;
  for (int dx = -1; dx <= 1; ++dx)
    for (int dy = -1; dy <= 1; ++dy)
      for (int dz = -1; dz <= 1; ++dz) {
        const uint32_t k = sph::morton_key(cx + dx, cy + dy, cz + dz, mask);
        for (uint32_t s = start[k]; s < start[k + 1]; ++s) {
          const uint32_t j = sorted_idx[s];
          if (!sph::in_range_exact(px, py, pz, samp[3 * j], samp[3 * j + 1], samp[3 * j + 2], range)) continue;
          if (out) out[offs[i] + c] = j;
          ++c;
        }
      }
  if (!out) counts[i] = c;
}

template <class R>
__global__ void k_kernel_eval(int n, const double* __restrict__ r, double h, int grad, double* __restrict__ out) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const sph::KernelConst<R> k = [&] {
    const double alpha = 16.0 / 3.14159265358979323846;
    sph::KernelConst<R> c;
    c.h = (R)h;
    c.inv_h = (R)(1.0 / h);
    c.cw = (R)(alpha / (h * h * h));
    c.cg = (R)(alpha / (h * h * h * h));
    return c;
  }();
  const R x = (R)r[3 * i], y = (R)r[3 * i + 1], z = (R)r[3 * i + 2];
  const R r2 = x * x + y * y + z * z;
  if (!grad) {
    out[i] = (double)sph::kernel_w_r2(r2, k);
  } else {
    const R f = sph::kernel_grad_factor(r2, k);
    out[3 * i] = (double)(f * x);
    out[3 * i + 1] = (double)(f * y);
    out[3 * i + 2] = (double)(f * z);
  }
}

uint32_t spread3_host(uint32_t v) {
  v &= 0x3ff;
  v = (v | (v << 16)) & 0x030000FF;
  v = (v | (v << 8)) & 0x0300F00F;
  v = (v | (v << 4)) & 0x030C30C3;
  v = (v | (v << 2)) & 0x09249249;
  return v;
}
int cell_host(double p, double cs) {
  const double f = std::floor(p / cs);
  if (f != f) return 0;
  if (f >= 2147483647.0) return 2147483647;
  if (f <= -2147483648.0) return (int)0x80000000;
  return (int)f;
}

}  // namespace

extern "C" {

int sph_spatial_hashing_find_samples(double range, size_t n, const double* positions, size_t ns,
                                     const double* samples, uint64_t* offsets, uint32_t* indices,
                                     size_t capacity, size_t* total, int device) {
  if (!total || (n && !positions) || (ns && !samples) || !(range > 0)) {
    g_err = "invalid argument";
    return SPH_ERR_INVALID;
  }
  return run(device, [&]() -> int {
    // bucket grid over the sample extent (cells beyond it wrap onto buckets
    // whose samples the exact distance test rejects)
    double mn[3] = {0, 0, 0}, mx[3] = {0, 0, 0};
    for (size_t s = 0; s < ns; ++s)
      for (int d = 0; d < 3; ++d) {
        const double v = samples[3 * s + d];
        if (s == 0 || v < mn[d]) mn[d] = v;
        if (s == 0 || v > mx[d]) mx[d] = v;
      }
    double ext = 4;
    for (int d = 0; d < 3; ++d) ext = std::max(ext, (mx[d] - mn[d]) / range + 3.0);
    int m = 2;
    while (m < 8 && (double)(1u << m) < ext) ++m;
    const uint32_t mask = (1u << m) - 1u, T = 1u << (3 * m);
    std::vector<uint32_t> key(ns), order(ns);
    for (size_t s = 0; s < ns; ++s) {
      const int c[3] = {cell_host(samples[3 * s], range), cell_host(samples[3 * s + 1], range),
                        cell_host(samples[3 * s + 2], range)};
      key[s] = spread3_host((uint32_t)c[0] & mask) | (spread3_host((uint32_t)c[1] & mask) << 1) |
               (spread3_host((uint32_t)c[2] & mask) << 2);
      order[s] = (uint32_t)s;
    }
    std::stable_sort(order.begin(), order.end(), [&](uint32_t a, uint32_t b) { return key[a] < key[b]; });
    std::vector<uint32_t> start(T + 2, 0);
    for (size_t s = 0; s < ns; ++s) start[key[s] + 1]++;
    for (uint32_t k = 0; k <= T; ++k) start[k + 1] += start[k];
    Buf<double> dpos(3 * n), dsamp(3 * ns);
    Buf<uint32_t> dorder(ns), dstart(T + 2), dcount(n);
    if (n) check(cudaMemcpy(dpos.p, positions, 3 * n * sizeof(double), cudaMemcpyHostToDevice), "memcpy");
    if (ns) check(cudaMemcpy(dsamp.p, samples, 3 * ns * sizeof(double), cudaMemcpyHostToDevice), "memcpy");
    if (ns) check(cudaMemcpy(dorder.p, order.data(), ns * sizeof(uint32_t), cudaMemcpyHostToDevice), "memcpy");
    check(cudaMemcpy(dstart.p, start.data(), (T + 2) * sizeof(uint32_t), cudaMemcpyHostToDevice), "memcpy");
    const int blocks = (int)std::max<size_t>(1, (n + 255) / 256);
    if (n)
      k_find_samples<<<blocks, 256>>>((int)n, dpos.p, dsamp.p, dorder.p, dstart.p, mask, range, range, dcount.p,
                                      nullptr, nullptr);
    check(cudaGetLastError(), "k_find_samples");
    std::vector<uint32_t> cnt(n);
    if (n) check(cudaMemcpy(cnt.data(), dcount.p, n * sizeof(uint32_t), cudaMemcpyDeviceToHost), "memcpy");
    std::vector<uint64_t> off(n + 1, 0);
    for (size_t i = 0; i < n; ++i) off[i + 1] = off[i] + cnt[i];
    *total = off[n];
    if (!offsets || !indices || capacity < off[n]) return SPH_ERR_CAPACITY;
    Buf<uint64_t> doff(n + 1);
    Buf<uint32_t> dout(std::max<uint64_t>(off[n], 1));
    check(cudaMemcpy(doff.p, off.data(), (n + 1) * sizeof(uint64_t), cudaMemcpyHostToDevice), "memcpy");
    if (n)
      k_find_samples<<<blocks, 256>>>((int)n, dpos.p, dsamp.p, dorder.p, dstart.p, mask, range, range, dcount.p,
                                      doff.p, dout.p);
    check(cudaGetLastError(), "k_find_samples");
    std::copy(off.begin(), off.end(), offsets);
    if (off[n]) check(cudaMemcpy(indices, dout.p, off[n] * sizeof(uint32_t), cudaMemcpyDeviceToHost), "memcpy");
    return SPH_OK;
  });
}

static int kernel_eval(size_t n, const double* r, double h, double* out, int precision, int device, int grad) {
  if ((n && (!r || !out)) || !(h > 0)) {
    g_err = "invalid argument";
    return SPH_ERR_INVALID;
  }
  return run(device, [&]() -> int {
    if (!n) return SPH_OK;
    const size_t outn = grad ? 3 * n : n;
    Buf<double> dr(3 * n), dout(outn);
    check(cudaMemcpy(dr.p, r, 3 * n * sizeof(double), cudaMemcpyHostToDevice), "memcpy");
    const int blocks = (int)((n + 255) / 256);
    if (precision == SPH_F64)
      k_kernel_eval<double><<<blocks, 256>>>((int)n, dr.p, h, grad, dout.p);
    else
      k_kernel_eval<float><<<blocks, 256>>>((int)n, dr.p, h, grad, dout.p);
    check(cudaGetLastError(), "k_kernel_eval");
    check(cudaMemcpy(out, dout.p, outn * sizeof(double), cudaMemcpyDeviceToHost), "memcpy");
    return SPH_OK;
  });
}

int sph_kernel_function(size_t n, const double* r, double h, double* out_w, int precision, int device) {
  return kernel_eval(n, r, h, out_w, precision, device, 0);
}
int sph_kernel_gradient(size_t n, const double* r, double h, double* out_grad, int precision, int device) {
  return kernel_eval(n, r, h, out_grad, precision, device, 1);
}

}  // extern "C"
