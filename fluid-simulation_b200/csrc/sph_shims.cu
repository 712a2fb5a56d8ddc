// Per-trait compatibility entry points of the C ABI: the reference's trait
// seams pass host arrays on every call (neighbor_search/mod.rs:18-28,
// kernel/mod.rs:17-46), so these upload, run one kernel and download. They
// exist for per-trait parity checks; the device-resident System is the
// production path.
#include <algorithm>
#include <mutex>
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

// ===========================================================================
// Allocation-free neighbor search
//
// For callers that cannot allocate device memory: code that runs while its
// process's allocator is owned by another runtime (a framework memory pool,
// a real-time loop that forbids allocation, a host that hands the engine only
// pre-registered buffers). The caller passes its inputs and outputs as device
// pointers; every temporary lives in one file-scope device array that each
// GPU loading this library keeps until the process exits.
// ===========================================================================
namespace {

constexpr size_t kStaticMaxSamples = size_t(1) << 20;    // sample positions
constexpr size_t kStaticMaxPositions = size_t(1) << 20;  // query positions
constexpr int kStaticBits = 6;                           // 2^(3*6) buckets
constexpr size_t kStaticBuckets = size_t(1) << (3 * kStaticBits);
// The bucket order comes from a stable LSD radix sort of the 18-bit keys:
// three passes of 6-bit digits over tiles of 256 samples in index order.
constexpr int kRadixBits = 6;
constexpr int kRadixDigits = 1 << kRadixBits;
constexpr int kRadixPasses = 3 * kStaticBits / kRadixBits;
constexpr int kRadixTile = 256;
constexpr size_t kStaticMaxTiles = kStaticMaxSamples / kRadixTile;
// keys, two order buffers (radix ping-pong), bucket counts and starts, and the
// per-(digit, tile) offsets of one radix pass
constexpr size_t kStaticScratchBytes = 3 * kStaticMaxSamples * sizeof(uint32_t) +
                                       2 * (kStaticBuckets + 2) * sizeof(uint32_t) +
                                       kRadixDigits * kStaticMaxTiles * sizeof(uint32_t);

static __device__ __align__(256) unsigned char g_find_scratch[kStaticScratchBytes];

struct StaticScratch {
  uint32_t* key;
  uint32_t* order;   // sorted sample indices (radix output of the last pass)
  uint32_t* order2;  // ping-pong buffer of the radix passes
  uint32_t* count;
  uint32_t* start;
  uint32_t* digit;   // [kRadixDigits][tiles] digit counts, then their offsets
};

StaticScratch carve(void* base) {
  unsigned char* p = (unsigned char*)base;
  StaticScratch s;
  s.key = (uint32_t*)p;
  s.order = s.key + kStaticMaxSamples;
  s.order2 = s.order + kStaticMaxSamples;
  s.count = s.order2 + kStaticMaxSamples;
  s.start = s.count + (kStaticBuckets + 2);
  s.digit = s.start + (kStaticBuckets + 2);
  return s;
}

// Device address of the scratch array, resolved once per device with that
// device current (a host-side reference to the array names only its shadow).
void* static_scratch_address(int device) {
  static std::mutex mu;
  static void* addr[64] = {nullptr};
  if (device < 0 || device >= 64) throw ShimError{SPH_ERR_INVALID, "device ordinal out of range"};
  std::lock_guard<std::mutex> lock(mu);
  if (!addr[device]) {
    void* p = nullptr;
    check(cudaGetSymbolAddress(&p, g_find_scratch), "cudaGetSymbolAddress");
    addr[device] = p;
  }
  return addr[device];
}

__global__ void k_static_zero(uint32_t* __restrict__ a, size_t n) {
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x)
    a[i] = 0u;
}

// Bucket key of every sample and the bucket sizes (the counts do not depend
// on the order of the atomic additions).
__global__ void k_static_keys(int ns, const double* __restrict__ samp, double cell, uint32_t mask,
                              uint32_t* __restrict__ key, uint32_t* __restrict__ count) {
  const int s = blockIdx.x * blockDim.x + threadIdx.x;
  if (s >= ns) return;
  const uint32_t k = sph::morton_key(sph::cell_coord(samp[3 * s], cell), sph::cell_coord(samp[3 * s + 1], cell),
                                     sph::cell_coord(samp[3 * s + 2], cell), mask);
  key[s] = k;
  atomicAdd(&count[k], 1u);
}

// Scan by one block (exclusive, or inclusive when INCL): each thread scans a
// contiguous chunk. `in` and `out` may be the same array (each element is
// read before it is written).
template <class T, bool INCL>
__global__ void __launch_bounds__(1024) k_static_scan(const T* in, T* out, size_t m) {
  __shared__ T part[1024];
  const size_t per = (m + blockDim.x - 1) / blockDim.x;
  const size_t b = threadIdx.x * per, e = b + per < m ? b + per : m;
  T s = 0;
  for (size_t i = b; i < e; ++i) s += in[i];
  part[threadIdx.x] = s;
  __syncthreads();
  if (threadIdx.x == 0) {
    T run = 0;
    for (unsigned t = 0; t < blockDim.x; ++t) {
      const T v = part[t];
      part[t] = run;
      run += v;
    }
  }
  __syncthreads();
  T run = part[threadIdx.x];
  for (size_t i = b; i < e; ++i) {
    const T v = in[i];
    if (INCL) {
      run += v;
      out[i] = run;
    } else {
      out[i] = run;
      run += v;
    }
  }
}

// Radix pass `shift`, step 1: per tile of 256 entries of `in` (sample indices
// in the current order; the identity when `in` is null), the count of each
// digit, stored digit-major so that one exclusive scan gives every (digit,
// tile) its first output slot.
__global__ void __launch_bounds__(kRadixTile) k_radix_hist(int ns, const uint32_t* __restrict__ in,
                                                           const uint32_t* __restrict__ key, int shift,
                                                           uint32_t* __restrict__ digit, int tiles) {
  __shared__ uint32_t h[kRadixDigits];
  if (threadIdx.x < kRadixDigits) h[threadIdx.x] = 0u;
  __syncthreads();
  const int e = blockIdx.x * kRadixTile + threadIdx.x;
  if (e < ns) {
    const uint32_t s = in ? in[e] : (uint32_t)e;
    atomicAdd(&h[(key[s] >> shift) & (kRadixDigits - 1)], 1u);
  }
  __syncthreads();
  if (threadIdx.x < kRadixDigits) digit[(size_t)threadIdx.x * tiles + blockIdx.x] = h[threadIdx.x];
}

// Radix pass step 2: stable scatter. An entry's slot is its (digit, tile)
// offset plus the number of entries of the tile before it with the same
// digit: lanes of equal digit within the warp (match), then the counts of
// the warps before it.
__global__ void __launch_bounds__(kRadixTile) k_radix_scatter(int ns, const uint32_t* __restrict__ in,
                                                              const uint32_t* __restrict__ key, int shift,
                                                              const uint32_t* __restrict__ digit, int tiles,
                                                              uint32_t* __restrict__ out) {
  constexpr int kWarps = kRadixTile / 32;
  __shared__ uint32_t wc[kWarps][kRadixDigits];
  for (int t = threadIdx.x; t < kWarps * kRadixDigits; t += kRadixTile) (&wc[0][0])[t] = 0u;
  __syncthreads();
  const int e = blockIdx.x * kRadixTile + threadIdx.x;
  const bool valid = e < ns;
  const unsigned act = __ballot_sync(0xffffffffu, valid);
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  uint32_t s = 0, d = 0, rank = 0;
  if (valid) {
    s = in ? in[e] : (uint32_t)e;
    d = (key[s] >> shift) & (kRadixDigits - 1);
    const unsigned peers = __match_any_sync(act, d);
    rank = __popc(peers & ((1u << lane) - 1u));
    if (lane == __ffs(peers) - 1) wc[w][d] = __popc(peers);
  }
  __syncthreads();
  if (valid) {
    for (int v = 0; v < w; ++v) rank += wc[v][d];
    out[digit[(size_t)d * tiles + blockIdx.x] + rank] = s;
  }
}

// Per-position neighbor counts into offsets[i + 1] (offsets[0] = 0).
// Per-position neighbor counts into offsets[i + 1] (offsets[0] = 0).
__global__ void k_static_count(int n, const double* __restrict__ pos, const double* __restrict__ samp,
                               const uint32_t* __restrict__ order, const uint32_t* __restrict__ start,
                               uint32_t mask, double range, uint64_t* __restrict__ counts) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i == 0) counts[0] = 0;
  if (i >= n) return;
  const double px = pos[3 * i], py = pos[3 * i + 1], pz = pos[3 * i + 2];
  const int cx = sph::cell_coord(px, range), cy = sph::cell_coord(py, range), cz = sph::cell_coord(pz, range);
  uint64_t c = 0;
  for (int dx = -1; dx <= 1; ++dx)
    for (int dy = -1; dy <= 1; ++dy)
      for (int dz = -1; dz <= 1; ++dz) {
        const uint32_t k = sph::morton_key(cx + dx, cy + dy, cz + dz, mask);
        for (uint32_t s = start[k]; s < start[k + 1]; ++s) {
          const uint32_t j = order[s];
          c += sph::in_range_exact(px, py, pz, samp[3 * j], samp[3 * j + 1], samp[3 * j + 2], range) ? 1 : 0;
        }
      }
  counts[i + 1] = c;
}

}  // namespace

extern "C" int sph_spatial_hashing_find_samples_noalloc(double search_range, size_t n, const double* d_positions,
                                                        size_t ns, const double* d_samples, uint64_t* d_offsets,
                                                        uint32_t* d_indices, size_t capacity, size_t* total,
                                                        int device) {
  if (!total || !d_offsets || (n && !d_positions) || (ns && !d_samples) || !(search_range > 0)) {
    g_err = "invalid argument";
    return SPH_ERR_INVALID;
  }
  if (ns > kStaticMaxSamples || n > kStaticMaxPositions) {
    g_err = "sph_spatial_hashing_find_samples_noalloc: at most 1048576 samples and 1048576 positions";
    return SPH_ERR_INVALID;
  }
  return run(device, [&]() -> int {
    const StaticScratch S = carve(static_scratch_address(device));
    const uint32_t mask = (1u << kStaticBits) - 1u;
    const uint32_t T = (uint32_t)kStaticBuckets;
    // the array keeps the previous call's contents: clear the bucket counts
    k_static_zero<<<256, 256>>>(S.count, (size_t)T + 2);
    const unsigned sb = (unsigned)((ns + 255) / 256);
    if (ns) k_static_keys<<<sb, 256>>>((int)ns, d_samples, search_range, mask, S.key, S.count);
    k_static_scan<uint32_t, false><<<1, 1024>>>(S.count, S.start, (size_t)T + 2);
    if (ns) {
      // bucket order with ascending sample index inside each bucket, as
      // SpatialHashing::populate pushes them (spatial_hashing.rs:27-37)
      const int tiles = (int)((ns + kRadixTile - 1) / kRadixTile);
      const uint32_t* in = nullptr;
      uint32_t* bufs[2] = {(kRadixPasses & 1) ? S.order : S.order2, (kRadixPasses & 1) ? S.order2 : S.order};
      for (int pass = 0; pass < kRadixPasses; ++pass) {
        uint32_t* out = bufs[pass & 1];
        k_radix_hist<<<tiles, kRadixTile>>>((int)ns, in, S.key, pass * kRadixBits, S.digit, tiles);
        k_static_scan<uint32_t, false><<<1, 1024>>>(S.digit, S.digit, (size_t)kRadixDigits * tiles);
        k_radix_scatter<<<tiles, kRadixTile>>>((int)ns, in, S.key, pass * kRadixBits, S.digit, tiles, out);
        in = out;
      }
    }
    const unsigned nb = (unsigned)std::max<size_t>(1, (n + 255) / 256);
    k_static_count<<<nb, 256>>>((int)n, d_positions, d_samples, S.order, S.start, mask, search_range, d_offsets);
    k_static_scan<uint64_t, true><<<1, 1024>>>(d_offsets, d_offsets, n + 1);
    check(cudaGetLastError(), "find_samples_noalloc");
    uint64_t tot = 0;
    check(cudaMemcpy(&tot, d_offsets + n, sizeof(uint64_t), cudaMemcpyDeviceToHost), "cudaMemcpy");
    *total = (size_t)tot;
    if (!d_indices || capacity < tot) return SPH_ERR_CAPACITY;
    if (n)
      k_find_samples<<<nb, 256>>>((int)n, d_positions, d_samples, S.order, S.start, mask, search_range,
                                  search_range, nullptr, d_offsets, d_indices);
    check(cudaGetLastError(), "find_samples_noalloc");
    check(cudaDeviceSynchronize(), "find_samples_noalloc");
    return SPH_OK;
  });
}
