// Host orchestration of the SPH step engine and the C ABI of include/sphgpu.h.
//
// A `System<R>` owns one scene's device state and its CUDA stream and runs
// the reference's step (sph/mod.rs:125-144, update :674-731) as a fixed
// sequence of kernel launches. The only host synchronisation per step is the
// final read of the step scalars (and, for IISPH with a target density
// error, a convergence check after the first batch of sweeps).
#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <limits>
#include <map>
#include <memory>
#include <mutex>
#include <stdexcept>
#include <string>
#include <type_traits>
#include <vector>

#include "../../include/sphgpu.h"
#include "sph_fields.cuh"
#include "sph_formats.hpp"
#include "sph_host.hpp"
#include "sph_kernels.cuh"
#include "sph_surface.cuh"

namespace sph {

// ---------------------------------------------------------------------------
// errors and buffers
// ---------------------------------------------------------------------------
thread_local std::string g_last_error;

template <class T>
struct DBuf {
  T* p = nullptr;
  size_t n = 0;
  DBuf() = default;
  DBuf(const DBuf&) = delete;
  DBuf& operator=(const DBuf&) = delete;
  ~DBuf() { release(); }
  void release() {
    if (p) cudaFree(p);
    p = nullptr;
    n = 0;
  }
  void alloc(size_t count) {
    if (count == n && p) return;
    release();
    if (count == 0) return;
    cuda_check(cudaMalloc((void**)&p, count * sizeof(T)), "cudaMalloc");
    n = count;
  }
  void zero(cudaStream_t s) {
    if (p) cuda_check(cudaMemsetAsync(p, 0, n * sizeof(T), s), "cudaMemsetAsync");
  }
  size_t bytes() const { return n * sizeof(T); }
};

// Opts a kernel into more than 48 KB of dynamic shared memory (once per
// device and kernel).
static void allow_smem(const void* fn, size_t bytes) {
  static std::mutex mu;
  static std::map<std::pair<int, const void*>, size_t> done;
  int dev = 0;
  cudaGetDevice(&dev);
  std::lock_guard<std::mutex> lock(mu);
  size_t& have = done[{dev, fn}];
  if (have >= bytes) return;
  cuda_check(cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes),
             "cudaFuncSetAttribute");
  have = bytes;
}

// Shared memory one block may use (sm_100: 227 KB with the opt-in) and what
// the staging passes keep aside for their static arrays.
constexpr size_t kMaxSmemPerBlock = 232448;
constexpr size_t kStaticSmemReserve = 4096;
static int blocks_for(long long n) { return (int)std::max(1LL, (n + kBlock - 1) / kBlock); }
static size_t round_up(size_t n, size_t m) { return (n + m - 1) / m * m; }

// ---------------------------------------------------------------------------
// serendipity reference node tables (discretization.rs:267-300)
// ---------------------------------------------------------------------------
static void upload_serendipity_tables() {
  static std::mutex mu;
  static bool done_for[64] = {false};
  std::lock_guard<std::mutex> lock(mu);
  int dev = 0;
  cudaGetDevice(&dev);
  if (dev >= 0 && dev < 64 && done_for[dev]) return;
  double ref[32][3];
  int off[32][3];
  int kind[32];
  int a = 0;
  const double s[2] = {-1.0, 1.0}, t[2] = {-1.0 / 3.0, 1.0 / 3.0};
  auto push = [&](double x, double y, double z) {
    ref[a][0] = x; ref[a][1] = y; ref[a][2] = z;
    const double r[3] = {x, y, z};
    for (int d = 0; d < 3; ++d) off[a][d] = (int)std::llround((r[d] + 1.0) * 1.5);
    auto corner = [](double c) { return std::fabs(std::fabs(c) - 1.0) < 1e-9; };
    const bool cx = corner(x), cy = corner(y), cz = corner(z);
    kind[a] = (cx && cy && cz) ? 0 : (!cx ? 1 : (!cy ? 2 : 3));
    ++a;
  };
  for (double z : s) for (double y : s) for (double x : s) push(x, y, z);
  for (double z : s) for (double y : s) for (double q : t) push(q, y, z);
  for (double z : s) for (double x : s) for (double q : t) push(x, q, z);
  for (double y : s) for (double x : s) for (double q : t) push(x, y, q);
  cuda_check(cudaMemcpyToSymbol(c_ser_ref, ref, sizeof ref), "serendipity tables");
  cuda_check(cudaMemcpyToSymbol(c_ser_off, off, sizeof off), "serendipity tables");
  cuda_check(cudaMemcpyToSymbol(c_ser_kind, kind, sizeof kind), "serendipity tables");
  if (dev >= 0 && dev < 64) done_for[dev] = true;
}

// Host-buffer state exchange in reference index order (sph_step_host).
template <class R>
__global__ void k_state_in(int n, const uint32_t* __restrict__ ref, const double* __restrict__ x,
                           const double* __restrict__ v, R4<R>* __restrict__ pos, R4<R>* __restrict__ vel) {
  const int d = blockIdx.x * blockDim.x + threadIdx.x;
  if (d >= n) return;
  const size_t r = ref[d];
  if (x) {
    R4<R> p = pos[d];
    p.x = (R)x[3 * r]; p.y = (R)x[3 * r + 1]; p.z = (R)x[3 * r + 2];
    pos[d] = p;
  }
  if (v) {
    R4<R> q = vel[d];
    q.x = (R)v[3 * r]; q.y = (R)v[3 * r + 1]; q.z = (R)v[3 * r + 2];
    vel[d] = q;
  }
}
template <class R>
__global__ void k_state_out(int n, const uint32_t* __restrict__ ref, const R4<R>* __restrict__ xv,
                            const R4<R>* __restrict__ vel, double* __restrict__ x, double* __restrict__ v) {
  const int d = blockIdx.x * blockDim.x + threadIdx.x;
  if (d >= n) return;
  const size_t r = ref[d];
  if (x) {
    const R4<R> p = xv[d];
    x[3 * r] = (double)p.x; x[3 * r + 1] = (double)p.y; x[3 * r + 2] = (double)p.z;
  }
  if (v) {
    const R4<R> q = vel[d];
    v[3 * r] = (double)q.x; v[3 * r + 1] = (double)q.y; v[3 * r + 2] = (double)q.z;
  }
}

// ---------------------------------------------------------------------------
// System<R>
// ---------------------------------------------------------------------------
template <class R>
class System : public SystemBase {
 public:
  explicit System(const sph_config& c) : cfg_(c) {
    device = c.device;
    if (const char* e = std::getenv("SPHGPU_SORTED_LISTS")) sorted_lists_ = std::atoi(e) != 0;
    if (const char* e = std::getenv("SPHGPU_DEPENDENT_LAUNCH")) pdl_ = std::atoi(e) != 0;
    if (const char* e = std::getenv("SPHGPU_SWEEP_PREFETCH")) prefetch_ = std::atoi(e) != 0;
    if (const char* e = std::getenv("SPHGPU_HALO_STAGE")) {
      // the same bound as set_tuning: the widest staged record ({x, v, m})
      // times the capacity must fit one block's shared memory
      const size_t record = 2 * sizeof(R4<R>) + sizeof(R);
      const int fit = (int)((kMaxSmemPerBlock - kStaticSmemReserve) / record);
      hs_ = std::max(0, std::min(std::atoi(e), std::min(fit, 4096)));
    }
    if (const char* e = std::getenv("SPHGPU_HALO_CAPACITY")) hcap_ = std::max(64, std::min(std::atoi(e), 65535));
    if (const char* e = std::getenv("SPHGPU_GATHER_BATCH")) {
      const int v = std::atoi(e);
      nb_ = (v == 4 || v == 8) ? v : 4;
    }
    cuda_check(cudaSetDevice(c.device), "cudaSetDevice");
    cuda_check(cudaStreamCreateWithFlags(&stream_, cudaStreamNonBlocking), "cudaStreamCreate");
    cuda_check(cudaMallocHost((void**)&h_sc_, sizeof(Scalars)), "cudaMallocHost");
    cuda_check(cudaMallocHost((void**)&h_meas_, 2 * sizeof(double)), "cudaMallocHost");
    d_sc_.alloc(1);
    d_meas_.alloc(2);
    std::memset(h_sc_, 0, sizeof(Scalars));
    upload_serendipity_tables();
  }
  ~System() override {
    if (chunk_steps_) cudaEventSynchronize(chunk_event_);
    destroy_graphs();
    if (chunk_event_) cudaEventDestroy(chunk_event_);
    if (body_stream_) cudaStreamDestroy(body_stream_);
    if (io_stream_) {
      cudaStreamSynchronize(io_stream_);
      cudaStreamDestroy(io_stream_);
    }
    if (io_ready_) cudaEventDestroy(io_ready_);
    if (h_chunk_sc_) cudaFreeHost(h_chunk_sc_);
    for (auto& kv : prof_) {
      for (auto& e : kv.second.pool) {
        cudaEventDestroy(e.first);
        cudaEventDestroy(e.second);
      }
    }
    if (h_sc_) cudaFreeHost(h_sc_);
    if (h_meas_) cudaFreeHost(h_meas_);
    if (stream_) cudaStreamDestroy(stream_);
  }

  SystemBase* clone() const override;

  // ---- setup ---------------------------------------------------------------
  void upload_fluid(size_t n, const double* x, const double* v, const double* m,
                    const uint32_t* fid) override {
    if (n > 0x7fffffffULL) throw Error(SPH_ERR_INVALID, "too many particles");
    n_ = n;
    cap_ = std::max<size_t>(n, 1);
    np_ = round_up(cap_, 32);
    alloc_particles();
    std::vector<R4<R>> hp(cap_), hv(cap_);
    std::vector<uint32_t> hr(cap_), hf(cap_);
    for (size_t i = 0; i < n; ++i) {
      hp[i] = R4<R>{(R)x[3 * i], (R)x[3 * i + 1], (R)x[3 * i + 2], R(0)};
      const double vx = v ? v[3 * i] : 0.0, vy = v ? v[3 * i + 1] : 0.0, vz = v ? v[3 * i + 2] : 0.0;
      hv[i] = R4<R>{(R)vx, (R)vy, (R)vz, (R)m[i]};
      hr[i] = (uint32_t)i;
      hf[i] = fid ? fid[i] : 0u;
    }
    copy_h2d(pos_.p, hp.data(), cap_);
    copy_h2d(vel_.p, hv.data(), cap_);
    copy_h2d(ref_.p, hr.data(), cap_);
    copy_h2d(fid_.p, hf.data(), cap_);
    acc_.zero(stream_);
    xint_.zero(stream_);
    vint_.zero(stream_);
    host_bbox_.clear();
    for (size_t i = 0; i < n; ++i) bbox_add(x[3 * i], x[3 * i + 1], x[3 * i + 2]);
    fluid_uploaded_ = true;
  }

  int add_sample_boundary(size_t nb, const double* x, const sph_rigid_init* rigid) override {
    if (cfg_.boundary_handling != SPH_STATIC_SAMPLE_BOUNDARY)
      throw Error(SPH_ERR_INVALID, "system uses VolumeMapBoundary; sample boundary rejected");
    if ((int)bodies_.size() >= kMaxBodies) throw Error(SPH_ERR_INVALID, "too many boundaries");
    const int bi = (int)bodies_.size();
    bodies_.push_back(make_body(rigid));
    sample_offsets_.push_back(h_sample_x_.size() / 3);
    sample_counts_.push_back(nb);
    for (size_t s = 0; s < nb; ++s) {
      h_sample_x_.push_back(x[3 * s]);
      h_sample_x_.push_back(x[3 * s + 1]);
      h_sample_x_.push_back(x[3 * s + 2]);
      h_sample_bid_.push_back((uint32_t)bi);
    }
    return bi;
  }

  int add_volume_map(const sph_grid_desc& sd, const double* sn, const sph_grid_desc& vd,
                     const double* vn, const sph_rigid_init* rigid) override {
    if (cfg_.boundary_handling != SPH_VOLUME_MAP_BOUNDARY)
      throw Error(SPH_ERR_INVALID, "system uses StaticSampleBoundary; volume map rejected");
    if ((int)bodies_.size() >= kMaxBodies) throw Error(SPH_ERR_INVALID, "too many boundaries");
    const int bi = (int)bodies_.size();
    bodies_.push_back(make_body(rigid));
    auto f = std::make_unique<FieldPair>();
    f->sdf_desc = sd;
    f->vm_desc = vd;
    for (int which = 0; which < 2; ++which) {
      const sph_grid_desc& g = which ? vd : sd;
      for (int d = 0; d < 3; ++d)
        if (g.n[d] < 1 || g.n[d] > 100000) throw Error(SPH_ERR_INVALID, "bad field grid size");
      const size_t cnt = (size_t)(3 * g.n[0] + 1) * (size_t)(3 * g.n[1] + 1) * (size_t)(3 * g.n[2] + 1);
      DBuf<double>& buf = which ? f->vm : f->sdf;
      buf.alloc(cnt);
      copy_h2d(buf.p, which ? vn : sn, cnt);
      if (!rigid)
        bbox_add(g.x_min[0], g.x_min[1], g.x_min[2]), bbox_add(g.x_max[0], g.x_max[1], g.x_max[2]);
    }
    fields_.push_back(std::move(f));
    return bi;
  }

  void initialize() override {
    if (!fluid_uploaded_) throw Error(SPH_ERR_STATE, "upload fluid before initialize");
    const bool has_dyn = std::any_of(bodies_.begin(), bodies_.end(), [](const Body& b) { return b.dynamic; });
    const bool iisph_ost = cfg_.pressure_solver == SPH_IISPH_W_OST;
    const bool takes_pred = cfg_.integration_scheme == SPH_TAKE_PREDICTED;
    if (iisph_ost != takes_pred)  // sph/setup/mod.rs:229-231
      throw Error(SPH_ERR_INVALID, "IISPHwOST must pair with TakePredicted (and only it)");
    if (iisph_ost && has_dyn)  // sph/setup/mod.rs:236-238
      throw Error(SPH_ERR_INVALID, "IISPHwOST does not support dynamic boundaries");
    choose_grid();
    setup_params();
    // bodies
    nbodies_ = (int)bodies_.size();
    any_dynamic_ = has_dyn;
    bodies_d_.alloc(std::max(1, nbodies_));
    if (nbodies_) copy_h2d(bodies_d_.p, bodies_.data(), (size_t)nbodies_);
    body_partials_.alloc((size_t)blocks_for((long long)cap_) * kMaxBodies * 6);
    // boundaries
    if (cfg_.boundary_handling == SPH_STATIC_SAMPLE_BOUNDARY && !h_sample_bid_.empty())
      init_sample_boundaries();
    if (cfg_.boundary_handling == SPH_VOLUME_MAP_BOUNDARY && !fields_.empty()) {
      init_volume_maps();
      init_contacts();
    }
    boundary_kind_ = !h_sample_bid_.empty() ? 1 : (!fields_.empty() ? 2 : 0);
    // scalars
    Scalars s{};
    s.n = (int)n_;
    s.n_active = (int)n_;
    s.dt = cfg_.cfl_time_step ? 0.0 : cfg_.time_increment;
    s.err = 0.0;
    copy_h2d(d_sc_.p, &s, 1);
    *h_sc_ = s;
    steps_ = 0;
    current_time_ = 0.0;
    update(2);  // System::new_boxed's first update (sph/mod.rs:418-419)
    initialized_ = true;
  }

  // ---- stepping ------------------------------------------------------------
  int step(uint32_t nsteps) override {
    if (!initialized_) throw Error(SPH_ERR_STATE, "initialize before stepping");
    if (chunk_steps_) throw Error(SPH_ERR_STATE, "a chunk of graph steps is in flight");
    if (graph_chunk_ == 0 || profiling_) return step_plain(nsteps);
    int status = SPH_OK;
    for (uint32_t left = nsteps; left > 0;) {
      const uint32_t c = std::min(left, graph_chunk_);
      chunk_begin(c);
      const ChunkOutcome o = chunk_finish();
      if (o.status != SPH_OK) status = o.status;
      left -= c;
    }
    return status;
  }

  // System::step_forward_in_time (sph/mod.rs:125-144), one host check per step.
  int step_plain(uint32_t nsteps) {
    int status = SPH_OK;
    for (uint32_t s = 0; s < nsteps; ++s) {
      const auto t0 = std::chrono::steady_clock::now();
      const double dt_used = h_sc_->dt;
      // integrate happens inside update(mode) fused with the cell keys; the
      // rigid-body step must come between it and the neighbor search, and
      // only needs the time increment, so it is issued first on the stream.
      issue_contacts();
      if (any_dynamic_) launch("body_step", k_body_step, dim3(1), dim3(32), bodies_d_.p, nbodies_, (const Scalars*)d_sc_.p);
      ++steps_;
      if (cfg_.cfl_time_step) current_time_ += dt_used;
      update(cfg_.integration_scheme == SPH_TAKE_PREDICTED ? 1 : 0);
      if (h_sc_->status == 2) status = SPH_NOT_CONVERGED;
      wall_ = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
    }
    return status;
  }

  double time() const override {
    if (cfg_.cfl_time_step) return current_time_;
    return time_offset_ + (double)(steps_ - time_offset_steps_) * cfg_.time_increment;
  }
  uint64_t steps() const override { return steps_; }
  size_t num_particles() const override { return n_; }

  void measurement(sph_measurement* m) override {
    const int nb = blocks_for((long long)n_);
    ensure_partials(2 * (size_t)nb);
    launch("measure", k_measure<R>, dim3(nb), dim3(kBlock), d_sc_.p, (const R4<R>*)xv_.p,
           (const R4<R>*)vel_.p, partials_.p, d_meas_.p, P_);
    cuda_check(cudaMemcpyAsync(h_meas_, d_meas_.p, 2 * sizeof(double), cudaMemcpyDeviceToHost, stream_), "memcpy");
    sync();
    std::memset(m, 0, sizeof *m);
    const double nn = (double)n_;
    const bool sesph_like = cfg_.pressure_solver == SPH_SESPH || cfg_.pressure_solver == SPH_SESPH_W_SPLITTING;
    m->time = time();
    m->density = avg_density_;
    m->density_error = n_ ? 100.0 * (h_meas_[0] / nn - 1.0) : 0.0;
    m->kinetic_energy = n_ ? h_meas_[1] / nn : 0.0;
    m->stiffness = sesph_like ? cfg_.stiffness : 0.0;
    m->fluid_viscosity = cfg_.fluid_viscosity;
    m->boundary_viscosity = cfg_.boundary_viscosity;
    m->fluid_depth = 0.0;
    m->rest_density_grid_spacing = cfg_.rest_density_grid_spacing;
    m->kernel_support_radius = cfg_.kernel_support_radius;
    m->time_step_size = h_sc_->dt;
    m->target_density_error = sesph_like ? 0.0 : cfg_.target_density_error;
    m->solver_iterations = sesph_like ? 0u : (uint32_t)h_sc_->iterations;
    m->relaxation_factor = sesph_like ? 0.0 : cfg_.relaxation_factor;
    m->time_step_wall_clock_time = wall_;
    m->predicted_density_error = sesph_like ? 0.0 : h_sc_->err;
  }

  // ---- readback ------------------------------------------------------------
  void download(int field, double* out) override {
    std::vector<uint32_t> ref = fetch(ref_.p, n_);
    auto vec = [&](const R4<R>* src) {
      std::vector<R4<R>> h = fetch(src, n_);
      for (size_t d = 0; d < n_; ++d) {
        const size_t r = ref[d];
        out[3 * r] = (double)h[d].x; out[3 * r + 1] = (double)h[d].y; out[3 * r + 2] = (double)h[d].z;
      }
    };
    auto scal = [&](const R* src) {
      std::vector<R> h = fetch(src, n_);
      for (size_t d = 0; d < n_; ++d) out[ref[d]] = (double)h[d];
    };
    switch (field) {
      case SPH_FIELD_POSITION: vec(xv_.p); return;
      case SPH_FIELD_VELOCITY: vec(vel_.p); return;
      case SPH_FIELD_ACCELERATION: vec(acc_.p); return;
      case SPH_FIELD_MASS: {
        std::vector<R4<R>> h = fetch(vel_.p, n_);
        for (size_t d = 0; d < n_; ++d) out[ref[d]] = (double)h[d].w;
        return;
      }
      case SPH_FIELD_VOLUME: {
        std::vector<R4<R>> h = fetch(xv_.p, n_);
        for (size_t d = 0; d < n_; ++d) out[ref[d]] = (double)h[d].w;
        return;
      }
      case SPH_FIELD_PRESSURE: scal(press_.p); return;
      case SPH_FIELD_FLUID_ID: {
        std::vector<uint32_t> h = fetch(fid_.p, n_);
        for (size_t d = 0; d < n_; ++d) out[ref[d]] = (double)h[d];
        return;
      }
      case SPH_FIELD_SOURCE_TERM: need_iisph(); scal(s_.p); return;
      case SPH_FIELD_DIAGONAL: need_iisph(); scal(aii_.p); return;
      case SPH_FIELD_PREDICTED_VELOCITY:
        if (cfg_.pressure_solver == SPH_SESPH) throw Error(SPH_ERR_INVALID, "SESPH has no velocity slot");
        vec(vstar_.p);
        return;
      case SPH_FIELD_INTEGRATOR_POSITION:
        if (cfg_.integration_scheme != SPH_TAKE_PREDICTED) throw Error(SPH_ERR_INVALID, "no integrator slot");
        vec(xint_.p);
        return;
      case SPH_FIELD_INTEGRATOR_VELOCITY:
        if (cfg_.integration_scheme != SPH_TAKE_PREDICTED) throw Error(SPH_ERR_INVALID, "no integrator slot");
        vec(vint_.p);
        return;
    }
    throw Error(SPH_ERR_INVALID, "unknown field");
  }

  void fluid_ids(uint32_t* out) override {
    std::vector<uint32_t> ref = fetch(ref_.p, n_), h = fetch(fid_.p, n_);
    for (size_t d = 0; d < n_; ++d) out[ref[d]] = h[d];
  }
  void fluid_pos(float* out) override {
    std::vector<uint32_t> ref = fetch(ref_.p, n_);
    std::vector<R4<R>> h = fetch(xv_.p, n_);
    for (size_t d = 0; d < n_; ++d) {
      const size_t r = ref[d];
      out[3 * r] = (float)(double)h[d].x; out[3 * r + 1] = (float)(double)h[d].y; out[3 * r + 2] = (float)(double)h[d].z;
    }
  }
  void quantity(int q, float* out) override {  // sph/mod.rs:202-239
    std::vector<uint32_t> ref = fetch(ref_.p, n_);
    std::vector<R4<R>> x = fetch(xv_.p, n_), v = fetch(vel_.p, n_);
    std::vector<R> p;
    if (q == SPH_Q_PRESSURE) p = fetch(press_.p, n_);
    const double V0 = cfg_.rest_density_grid_spacing * cfg_.rest_density_grid_spacing * cfg_.rest_density_grid_spacing;
    for (size_t d = 0; d < n_; ++d) {
      const double vx = v[d].x, vy = v[d].y, vz = v[d].z, m = v[d].w, V = x[d].w;
      double val;
      switch (q) {
        case SPH_Q_SPEED: val = std::sqrt((vx * vx + vy * vy) + vz * vz); break;
        case SPH_Q_VOLUME: val = V; break;
        case SPH_Q_DENSITY: val = m / V; break;
        case SPH_Q_DENSITY_ERROR: val = V < V0 ? 100. * (V0 / V - 1.) : 0.; break;
        case SPH_Q_PRESSURE: val = (double)p[d]; break;
        case SPH_Q_KINETIC_ENERGY: val = 0.5 * m * ((vx * vx + vy * vy) + vz * vz); break;
        default: throw Error(SPH_ERR_INVALID, "unknown quantity");
      }
      out[ref[d]] = (float)val;
    }
  }

  // sph/mod.rs:241-341: quantity at n host positions (3n floats) into n
  // floats, from the state of the last update; the system's state is not
  // changed.
  void quantity_at(int q, size_t n, const float* pos, float* out) override {
    if (q < SPH_Q_SPEED || q > SPH_Q_KINETIC_ENERGY) throw Error(SPH_ERR_INVALID, "unknown quantity");
    if (chunk_steps_) throw Error(SPH_ERR_STATE, "a chunk of graph steps is in flight");
    if (n == 0) return;
    if (n > (size_t)INT32_MAX / 3) throw Error(SPH_ERR_CAPACITY, "too many evaluation positions");
    if (eval_pos_.n < 3 * n) eval_pos_.alloc(3 * n);
    if (eval_out_.n < n) eval_out_.alloc(n);
    cuda_check(cudaMemcpyAsync(eval_pos_.p, pos, 3 * n * sizeof(float), cudaMemcpyHostToDevice, stream_),
               "cudaMemcpyAsync");
    const double h = cfg_.kernel_support_radius, sp = cfg_.rest_density_grid_spacing;
    SampleGrid<R> G = sample_grid();
    if (boundary_kind_ != 1 || ns_ == 0) G.start = nullptr;
    const int nvm = boundary_kind_ == 2 ? (int)fields_.size() : 0;
    launch("quantity_at", k_quantity_at<R>, dim3(blocks_for((long long)n)), dim3(kBlock), q, (int)n,
           (const float*)eval_pos_.p, eval_out_.p, n_ ? (const uint32_t*)start_.p : (const uint32_t*)nullptr,
           (const R4<R>*)xv_.p, (const R4<R>*)vel_.p, (const R*)press_.p, G, (const VMDesc*)vms_.p, nvm,
           (const Body*)bodies_d_.p, make_kernel_const<double>(h), sp * sp * sp, P_);
    cuda_check(cudaMemcpyAsync(out, eval_out_.p, n * sizeof(float), cudaMemcpyDeviceToHost, stream_),
               "cudaMemcpyAsync");
    cuda_check(cudaStreamSynchronize(stream_), "cudaStreamSynchronize");
  }

  // Fluid::reconstruct_surfaces (fluid.rs:212-347): one mesh per fluid id in
  // ascending order, each group's rest density from its first particle's mass
  // (reference index order); groups without triangles are left out.
  void reconstruct_surfaces(std::vector<SurfaceMeshOut>& out) override {
    out.clear();
    if (chunk_steps_) throw Error(SPH_ERR_STATE, "a chunk of graph steps is in flight");
    const size_t n = n_;
    if (n == 0) return;
    std::vector<uint32_t> ids(n);
    fluid_ids(ids.data());
    std::vector<double> mass(n);
    download(SPH_FIELD_MASS, mass.data());
    std::map<uint32_t, double> groups;
    for (size_t i = 0; i < n; ++i)
      if (!groups.count(ids[i])) groups[ids[i]] = mass[i];
    static const SurfaceCases cases = surface_case_table();
    const double h = cfg_.kernel_support_radius, sp = cfg_.rest_density_grid_spacing;
    const double V0 = sp * sp * sp, r = 0.5 * sp, cube = 0.75 * r;
    auto grow = [](auto& buf, size_t cnt) {
      if (buf.n < cnt) buf.alloc(cnt);
    };
    grow(surf_vol_, n);
    grow(surf_bounds_, 7);
    const int nb = blocks_for((long long)n);
    auto blocks = [](long long m) { return dim3((unsigned)((m + kBlock - 1) / kBlock)); };
    auto scan_u32 = [&](uint32_t* count, long long m, uint32_t* outp) {
      const long long tiles = (m + kScanTile - 1) / kScanTile;
      grow(surf_tiles_, (size_t)tiles);
      launch("surface_scan", k_scan_tiles, dim3((unsigned)tiles), dim3(kBlock), (const uint32_t*)count, (int)m,
             surf_tiles_.p);
      launch("surface_scan", k_scan_tile_sums, dim3(1), dim3(1024), surf_tiles_.p, (int)tiles);
      launch("surface_scan", k_scan_apply, dim3((unsigned)tiles), dim3(kBlock), count, (int)m,
             (const uint32_t*)surf_tiles_.p, outp);
    };
    for (const auto& g : groups) {
      const uint32_t group = g.first;
      const double rest_density = g.second / V0;
      const double m = rest_density * (4.0 / 3.0 * 3.14159265358979323846 * (r * r * r));
      launch("surface_density", k_surf_density<R>, dim3(nb), dim3(kBlock), (int)n, (const uint32_t*)start_.p,
             (const R4<R>*)xv_.p, (const uint32_t*)fid_.p, group, m, h, mask_, surf_vol_.p);
      const unsigned long long init[7] = {~0ull, ~0ull, ~0ull, 0ull, 0ull, 0ull, 0ull};
      copy_h2d(surf_bounds_.p, init, 7);
      launch("surface_bounds", k_surf_bounds<R>, dim3(nb), dim3(kBlock), (int)n, (const R4<R>*)xv_.p,
             (const uint32_t*)fid_.p, group, surf_bounds_.p);
      std::vector<unsigned long long> bk = fetch(surf_bounds_.p, 7);
      SurfaceLattice L;
      L.cube = cube;
      double npts = 1.0;
      for (int d = 0; d < 3; ++d) {
        const double lo = surf_unkey(bk[d]), hi = surf_unkey(bk[3 + d]);
        const long long a = (long long)std::floor((lo - h) / cube) - 1;
        const long long b = (long long)std::floor((hi + h) / cube) + 1;
        L.k0[d] = a;
        L.n[d] = b - a + 1;
        npts *= (double)L.n[d];
      }
      if (npts > 6.0e8) throw Error(SPH_ERR_CAPACITY, "surface lattice larger than 6e8 points");
      const long long np = (long long)npts;
      const long long nc = (L.n[0] - 1) * (L.n[1] - 1) * (L.n[2] - 1);
      grow(surf_phi_, (size_t)np);
      grow(surf_flag_, (size_t)(3 * np + 1));
      grow(surf_vid_, (size_t)(3 * np + 1));
      grow(surf_tris_, (size_t)(nc + 1));
      grow(surf_toff_, (size_t)(nc + 1));
      launch("surface_levelset", k_surf_levelset<R>, blocks(np), dim3(kBlock), L, np, (const uint32_t*)start_.p,
             (const R4<R>*)xv_.p, (const uint32_t*)fid_.p, group, (const double*)surf_vol_.p, h, mask_,
             surf_phi_.p);
      launch("surface_edges", k_surf_edges, blocks(np), dim3(kBlock), L, np, (const double*)surf_phi_.p,
             surf_flag_.p);
      cuda_check(cudaMemsetAsync(surf_flag_.p + 3 * np, 0, sizeof(uint32_t), stream_), "cudaMemsetAsync");
      scan_u32(surf_flag_.p, 3 * np + 1, surf_vid_.p);
      launch("surface_cells", k_surf_cells, blocks(nc), dim3(kBlock), L, nc, (const double*)surf_phi_.p, cases,
             surf_tris_.p);
      cuda_check(cudaMemsetAsync(surf_tris_.p + nc, 0, sizeof(uint32_t), stream_), "cudaMemsetAsync");
      scan_u32(surf_tris_.p, nc + 1, surf_toff_.p);
      uint32_t nv = 0, nt = 0;
      cuda_check(cudaMemcpyAsync(&nv, surf_vid_.p + 3 * np, sizeof nv, cudaMemcpyDeviceToHost, stream_), "D2H");
      cuda_check(cudaMemcpyAsync(&nt, surf_toff_.p + nc, sizeof nt, cudaMemcpyDeviceToHost, stream_), "D2H");
      sync();
      if (nt == 0) continue;
      grow(surf_vtx_, (size_t)nv * 6);
      grow(surf_idx_, (size_t)nt * 3);
      launch("surface_vertices", k_surf_vertices, blocks(3 * np), dim3(kBlock), L, 3 * np,
             (const double*)surf_phi_.p, (const uint32_t*)surf_vid_.p, surf_vtx_.p);
      launch("surface_triangles", k_surf_triangles, blocks(nc), dim3(kBlock), L, nc, (const double*)surf_phi_.p,
             cases, (const uint32_t*)surf_toff_.p, (const uint32_t*)surf_vid_.p, surf_idx_.p);
      launch("surface_normals", k_surf_normals, blocks(nt), dim3(kBlock), (long long)nt,
             (const uint32_t*)surf_idx_.p, surf_vtx_.p);
      launch("surface_normals", k_surf_normalize, blocks(nv), dim3(kBlock), (long long)nv, surf_vtx_.p);
      SurfaceMeshOut mo;
      mo.fluid_id = group;
      mo.vertices = fetch(surf_vtx_.p, (size_t)nv * 6);
      mo.indices = fetch(surf_idx_.p, (size_t)nt * 3);
      out.push_back(std::move(mo));
    }
  }

  int fluid_neighbors(uint64_t* off, uint32_t* idx, size_t cap, size_t* total) override {
    std::vector<uint32_t> ref = fetch(ref_.p, n_), cnt = fetch(ncnt_.p, n_);
    std::vector<uint16_t> nb = fetch(nbr_.p, (size_t)K_ * np_);
    std::vector<uint32_t> hidx = fetch(halo_idx_.p, (size_t)blocks_for((long long)cap_) * (size_t)hcap_);
    auto slot = [&](size_t i, size_t k) {
      return (((i >> 5) * (size_t)(K_ >> 2) + (k >> 2)) * 32 + (i & 31)) * 4 + (k & 3);
    };
    size_t tot = 0;
    for (size_t d = 0; d < n_; ++d) tot += 1 + std::min<size_t>(cnt[d], (size_t)K_);
    *total = tot;
    if (!off || !idx || cap < tot) return SPH_ERR_CAPACITY;
    std::vector<uint64_t> rowlen(n_);
    for (size_t d = 0; d < n_; ++d) rowlen[ref[d]] = 1 + std::min<size_t>(cnt[d], (size_t)K_);
    off[0] = 0;
    for (size_t r = 0; r < n_; ++r) off[r + 1] = off[r] + rowlen[r];
    for (size_t d = 0; d < n_; ++d) {
      const size_t r = ref[d];
      uint32_t* row = idx + off[r];
      const size_t c = std::min<size_t>(cnt[d], (size_t)K_);
      row[0] = ref[d];
      const uint32_t* h = hidx.data() + (d / kBlock) * (size_t)hcap_;
      for (size_t k = 0; k < c; ++k) row[1 + k] = ref[h[nb[slot(d, k)]]];
      std::sort(row, row + c + 1);
    }
    return SPH_OK;
  }

  int boundary_neighbors(int bi, uint64_t* off, uint32_t* idx, size_t cap, size_t* total) override;
  void boundary_volumes(int bi, double* out) override {
    if (boundary_kind_ != 1 || bi < 0 || bi >= (int)sample_counts_.size())
      throw Error(SPH_ERR_INVALID, "not a sample boundary");
    std::vector<R4<R>> x = fetch(xb_.p, ns_);
    std::vector<uint32_t> o = fetch(sorig_.p, ns_);
    for (size_t s = 0; s < ns_; ++s) {
      const size_t g = o[s];
      if (g >= sample_offsets_[bi] && g < sample_offsets_[bi] + sample_counts_[bi])
        out[g - sample_offsets_[bi]] = (double)x[s].w;
    }
  }
  void boundary_positions(int bi, double* out) override {
    if (boundary_kind_ != 1 || bi < 0 || bi >= (int)sample_counts_.size())
      throw Error(SPH_ERR_INVALID, "not a sample boundary");
    std::vector<R4<R>> x = fetch(xb_.p, ns_);
    std::vector<uint32_t> o = fetch(sorig_.p, ns_);
    for (size_t s = 0; s < ns_; ++s) {
      const size_t g = o[s];
      if (g >= sample_offsets_[bi] && g < sample_offsets_[bi] + sample_counts_[bi]) {
        double* d = out + 3 * (g - sample_offsets_[bi]);
        d[0] = (double)x[s].x; d[1] = (double)x[s].y; d[2] = (double)x[s].z;
      }
    }
  }
  void vm_samples(int bi, uint8_t* has, double* xbo, double* vbo, double* vol) override {
    if (boundary_kind_ != 2 || bi < 0 || bi >= (int)fields_.size())
      throw Error(SPH_ERR_INVALID, "not a volume-map boundary");
    std::vector<uint32_t> ref = fetch(ref_.p, n_);
    std::vector<R4<R>> x = fetch(vmx_.p + (size_t)bi * np_, n_), v = fetch(vmv_.p + (size_t)bi * np_, n_);
    for (size_t d = 0; d < n_; ++d) {
      const size_t r = ref[d];
      has[r] = v[d].w != R(0) ? 1 : 0;
      for (int c = 0; c < 3; ++c) {
        xbo[3 * r + c] = has[r] ? (double)(&x[d].x)[c] : 0.0;
        vbo[3 * r + c] = has[r] ? (double)(&v[d].x)[c] : 0.0;
      }
      vol[r] = has[r] ? (double)x[d].w : 0.0;
    }
  }
  void rigid_state(int bi, double* out) override {
    if (bi < 0 || bi >= nbodies_) throw Error(SPH_ERR_INVALID, "bad boundary index");
    Body b;
    cuda_check(cudaMemcpyAsync(&b, bodies_d_.p + bi, sizeof(Body), cudaMemcpyDeviceToHost, stream_), "memcpy");
    sync();
    if (!b.dynamic) throw Error(SPH_ERR_INVALID, "static boundary has no rigid state");
    const double v[19] = {b.com[0], b.com[1], b.com[2], b.q[0], b.q[1], b.q[2], b.q[3],
                          b.v[0], b.v[1], b.v[2], b.L[0], b.L[1], b.L[2],
                          b.F[0], b.F[1], b.F[2], b.T[0], b.T[1], b.T[2]};
    std::memcpy(out, v, sizeof v);
  }
  void set_rigid_state(int bi, const double* in) override;

  uint64_t hash_collisions() override;
  void restore(uint64_t steps, double time, size_t n, const double* x, const double* v,
               const double* m, const uint32_t* fid, const double* xi, const double* vi) override;

  int step_host(uint32_t nsteps, const double* xi, const double* vi, double* xo, double* vo) override {
    if (!initialized_) throw Error(SPH_ERR_STATE, "initialize before stepping");
    const size_t n3 = 3 * n_;
    const int nb = blocks_for((long long)n_);
    if (!io_stream_) {
      cuda_check(cudaStreamCreateWithFlags(&io_stream_, cudaStreamNonBlocking), "cudaStreamCreate");
      cuda_check(cudaEventCreateWithFlags(&io_ready_, cudaEventDisableTiming), "cudaEventCreate");
    }
    if (xi || vi) {
      stage_x_.alloc(std::max<size_t>(n3, 3));
      stage_v_.alloc(std::max<size_t>(n3, 3));
      // positions and velocities travel on two streams, so two copy engines
      // can carry them at once
      if (xi) cuda_check(cudaMemcpyAsync(stage_x_.p, xi, n3 * sizeof(double), cudaMemcpyHostToDevice, stream_), "H2D");
      if (vi) {
        cuda_check(cudaMemcpyAsync(stage_v_.p, vi, n3 * sizeof(double), cudaMemcpyHostToDevice, io_stream_), "H2D");
        cuda_check(cudaEventRecord(io_ready_, io_stream_), "event");
        cuda_check(cudaStreamWaitEvent(stream_, io_ready_, 0), "event");
      }
      launch("state_io", k_state_in<R>, dim3(nb), dim3(kBlock), (int)n_, (const uint32_t*)ref_.p,
             (const double*)(xi ? stage_x_.p : nullptr), (const double*)(vi ? stage_v_.p : nullptr), pos_.p, vel_.p);
      // the positions the step integrates from live in xv too
      if (xi) cuda_check(cudaMemcpyAsync(xv_.p, pos_.p, n_ * sizeof(R4<R>), cudaMemcpyDeviceToDevice, stream_), "D2D");
    }
    // The state a step returns is final once its update has sorted the
    // integrated particles, so the last step's readback is issued right
    // there on a copy stream and overlaps the rest of that update (neighbor
    // search, solve). Graph-captured stepping, and an update that disabled
    // particles (which renumbers them afterwards), read back at the end.
    int st = SPH_OK;
    early_done_ = false;
    if ((xo || vo) && nsteps > 0) {
      if (nsteps > 1) st = step(nsteps - 1);
      stage_x_.alloc(std::max<size_t>(n3, 3));
      stage_v_.alloc(std::max<size_t>(n3, 3));
      early_xo_ = xo;
      early_vo_ = vo;
      const size_t n_before = n_;
      int st1;
      try {
        st1 = step(1);
      } catch (...) {
        early_xo_ = early_vo_ = nullptr;
        if (early_done_) cudaStreamSynchronize(io_stream_);
        throw;
      }
      early_xo_ = early_vo_ = nullptr;
      if (st == SPH_OK) st = st1;
      if (early_done_) cuda_check(cudaStreamSynchronize(io_stream_), "readback");
      if (early_done_ && n_ == n_before) return st;
    } else {
      st = step(nsteps);
    }
    if (xo || vo) {
      stage_x_.alloc(std::max<size_t>(n3, 3));
      stage_v_.alloc(std::max<size_t>(n3, 3));
      launch("state_io", k_state_out<R>, dim3(blocks_for((long long)n_)), dim3(kBlock), (int)n_,
             (const uint32_t*)ref_.p, (const R4<R>*)xv_.p, (const R4<R>*)vel_.p, xo ? stage_x_.p : nullptr,
             vo ? stage_v_.p : nullptr);
      if (xo) cuda_check(cudaMemcpyAsync(xo, stage_x_.p, 3 * n_ * sizeof(double), cudaMemcpyDeviceToHost, stream_), "D2H");
      if (vo) cuda_check(cudaMemcpyAsync(vo, stage_v_.p, 3 * n_ * sizeof(double), cudaMemcpyDeviceToHost, stream_), "D2H");
      sync();
    }
    return st;
  }
  void* stream() const override { return (void*)stream_; }
  void step_stats(sph_step_stats* o) const override {
    std::memset(o, 0, sizeof *o);
    o->particles = n_;
    o->solver_iterations = (uint32_t)h_sc_->iterations;
    o->solver_iterations_first = (uint32_t)h_sc_->iterations_eqs1;
    o->max_neighbors = (uint32_t)h_sc_->max_nbrs;
    o->max_boundary_neighbors = (uint32_t)h_sc_->max_bnbrs;
    o->predicted_density_error = h_sc_->err;
    o->time_increment = h_sc_->dt;
    o->average_density = h_sc_->avg_density;
    o->not_converged = h_sc_->status == 2;
  }
  uint64_t launches() const override { return launches_; }
  void set_profiling(bool on) override { profiling_ = on; }
  bool kernel_time(const std::string& name, double* ms, uint64_t* count) override {
    collect_profile();
    if (name == "*") {  // every timed launch of the handle
      *ms = 0.0;
      *count = 0;
      for (const auto& kv : prof_) {
        *ms += kv.second.ms;
        *count += kv.second.count;
      }
      return !prof_.empty();
    }
    auto it = prof_.find(name);
    if (it == prof_.end()) return false;
    *ms = it->second.ms;
    *count = it->second.count;
    return true;
  }
  size_t device_bytes() const override {
    size_t b = d_sc_.bytes() + d_meas_.bytes();
    for (const auto* d : {&pos_, &pos2_, &vel_, &vel2_, &xv_, &acc_, &vstar_, &xq_, &xu_, &TA_, &TB_, &xint_, &vint_, &bG_, &bGu_,
                          &xb_, &xb2_, &vb_, &vb2_, &xbody_, &vmx_, &vmv_, &snap_pos_, &snap_vel_, &snap_acc_,
                          &snap_xint_, &snap_vint_})
      b += d->bytes();
    for (const auto* d : {&press_, &s_, &aii_, &bW_, &rho_pred_}) b += d->bytes();
    b += uu_.bytes() + SA_.bytes();
    b += nbr_.bytes();
    for (const auto* d : {&ref_, &ref2_, &fid_, &fid2_, &key_, &slot_, &perm_, &halo_idx_, &halo_n_, &vm_near_, &ncnt_,
                          &count_, &start_,
                          &tile_sums_, &sbid_, &sbid2_, &sorig_, &sorig2_, &skey_, &sslot_, &sperm_, &scount_,
                          &sstart_, &snap_ref_, &snap_fid_})
      b += d->bytes();
    b += partials_.bytes() + body_partials_.bytes() + stage_x_.bytes() + stage_v_.bytes();
    b += eval_pos_.bytes() + eval_out_.bytes();
    b += surf_vol_.bytes() + surf_phi_.bytes() + surf_vtx_.bytes() + surf_flag_.bytes() + surf_vid_.bytes() +
         surf_tris_.bytes() + surf_toff_.bytes() + surf_idx_.bytes() + surf_tiles_.bytes() + surf_bounds_.bytes();
    b += contact_pairs_.bytes() + contact_cells_.bytes() + contact_state_.bytes() + contact_idx_.bytes() +
         contact_scalars_.bytes();
    b += bodies_d_.bytes() + snap_bodies_.bytes() + snap_sc_.bytes() + ns_d_.bytes() + vms_.bytes();
    for (const auto& f : fields_) b += f->sdf.bytes() + f->vm.bytes();
    return b;
  }

 private:
  friend SystemBase* make_system_copy(const SystemBase*);
  struct FieldPair {
    sph_grid_desc sdf_desc, vm_desc;
    DBuf<double> sdf, vm;
    bool has_aabb = false;  // mesh bounding box (body frame) for rigid-rigid contact
    double aabb_c[3] = {0, 0, 0}, aabb_h[3] = {0, 0, 0};
  };
  struct ProfEntry {
    double ms = 0;
    uint64_t count = 0;
    std::vector<std::pair<cudaEvent_t, cudaEvent_t>> pool;
    size_t used = 0;
  };

  sph_config cfg_;
  cudaStream_t stream_ = nullptr;
  uint32_t contact_fixed_sweeps_ = 0;  // 0: the reference's merit test
  // sph_step_host's overlapped readback of the last step
  cudaStream_t io_stream_ = nullptr;
  cudaEvent_t io_ready_ = nullptr;
  double* early_xo_ = nullptr;
  double* early_vo_ = nullptr;
  bool early_done_ = false;
  Scalars* h_sc_ = nullptr;
  double* h_meas_ = nullptr;
  DBuf<Scalars> d_sc_;
  DBuf<double> d_meas_;
  StepParams<R> P_{};
  size_t n_ = 0, cap_ = 0, np_ = 0;
  int K_ = 64;
  uint32_t T_ = 64, mask_ = 3;
  bool fluid_uploaded_ = false, initialized_ = false;
  uint64_t steps_ = 0;
  double current_time_ = 0, time_offset_ = 0, wall_ = 0, avg_density_ = 0;
  uint64_t time_offset_steps_ = 0;
  int last_iters_ = 3;
  int nb_ = 4;  // neighbor gather batch (prefetch width) of the neighbor passes
  // Neighbor lists in ascending stencil-key order (1) or in stencil order (0,
  // the default: neighbor records come from the block's staged halo, so list
  // order no longer matters for memory locality, and stencil order lets the
  // search skip buckets whose cell lies beyond the support radius).
  bool sorted_lists_ = false;
  bool pdl_ = true;       // programmatic dependent launch between the sweep passes
  bool prefetch_ = true;  // sweep passes prefetch the next wave's streams into L2
  std::map<std::pair<const void*, size_t>, int> resident_;
  uint64_t launches_ = 0;
  bool profiling_ = false;
  std::map<std::string, ProfEntry> prof_;
  struct Pending { std::string name; size_t idx; };
  std::vector<Pending> pending_;

  // particle state
  DBuf<R4<R>> pos_, pos2_, vel_, vel2_, xv_, acc_, vstar_, xint_, vint_, bG_, bGu_;
  DBuf<R4<R>> xq_, xu_;      // IISPH sweep records {x, V p}, {x, V a_x}
  DBuf<R4<R>> TA_, TB_;      // IISPH per-solve constants of the two sweep passes
  DBuf<R2<R>> uu_, SA_;      // IISPH sweep records {V a_y, V a_z}; {s, a_ii}
  DBuf<R> press_, s_, aii_, bW_, rho_pred_;
  DBuf<uint32_t> ref_, ref2_, fid_, fid2_, key_, slot_, perm_, ncnt_, halo_idx_, halo_n_;
  DBuf<uint16_t> nbr_;
  int hcap_ = 8192;   // halo table capacity per block (grows on overflow, at most 65535)
  int hs_ = sizeof(R) == 4 ? 1536 : 1024;  // halo records staged in shared memory per block
  // the same for the IISPH sweep passes (f32: 1792 x 24 B lets five pass-B
  // blocks share an SM's shared memory)
  int sweep_hs_ = sizeof(R) == 4 ? 1792 : 1024;
  DBuf<uint32_t> count_, start_, tile_sums_;
  DBuf<double> partials_, body_partials_, stage_x_, stage_v_;
  // boundaries
  std::vector<Body> bodies_;
  DBuf<Body> bodies_d_;
  int nbodies_ = 0;
  bool any_dynamic_ = false;
  int boundary_kind_ = 0;
  std::vector<double> h_sample_x_;
  std::vector<uint32_t> h_sample_bid_;
  std::vector<size_t> sample_offsets_, sample_counts_;
  size_t ns_ = 0;
  DBuf<R4<R>> xb_, xb2_, vb_, vb2_, xbody_;
  DBuf<uint32_t> sbid_, sbid2_, sorig_, sorig2_, skey_, sslot_, sperm_, scount_, sstart_;
  DBuf<int> ns_d_;
  std::vector<std::unique_ptr<FieldPair>> fields_;
  DBuf<VMDesc> vms_;
  // rigid-rigid contact of volume-map bodies
  bool contact_ = false;
  int contact_task_cap_ = 0;
  ContactGL contact_gl_{};
  DBuf<ContactPair> contact_pairs_;
  DBuf<ContactCell> contact_cells_;
  DBuf<ContactState> contact_state_;
  DBuf<int> contact_idx_;
  DBuf<ContactScalars> contact_scalars_;
  DBuf<R4<R>> vmx_, vmv_;
  DBuf<uint32_t> vm_near_;  // particles near a volume map this step
  DBuf<float> eval_pos_, eval_out_;  // quantity evaluation positions and values
  // surface reconstruction scratch (grown on demand, render frames only)
  DBuf<double> surf_vol_, surf_phi_, surf_vtx_;
  DBuf<uint32_t> surf_flag_, surf_vid_, surf_tris_, surf_toff_, surf_idx_, surf_tiles_;
  DBuf<unsigned long long> surf_bounds_;
  // bounding box of the scene (cells chosen from it)
  struct BBox {
    double mn[3], mx[3];
    bool any = false;
    void clear() { any = false; }
  } bbox_;
  BBox& host_bbox_ = bbox_;

  // ---- helpers ---------------------------------------------------------------
  void bbox_add(double x, double y, double z) {
    const double p[3] = {x, y, z};
    if (!bbox_.any) {
      for (int d = 0; d < 3; ++d) bbox_.mn[d] = bbox_.mx[d] = p[d];
      bbox_.any = true;
      return;
    }
    for (int d = 0; d < 3; ++d) {
      bbox_.mn[d] = std::min(bbox_.mn[d], p[d]);
      bbox_.mx[d] = std::max(bbox_.mx[d], p[d]);
    }
  }
  template <class T>
  void copy_h2d(T* dst, const T* src, size_t n) {
    if (n == 0) return;
    cuda_check(cudaMemcpyAsync(dst, src, n * sizeof(T), cudaMemcpyHostToDevice, stream_), "cudaMemcpy H2D");
    sync();
  }
  template <class T>
  std::vector<T> fetch(const T* src, size_t n) {
    std::vector<T> h(n);
    if (n) {
      cuda_check(cudaMemcpyAsync(h.data(), src, n * sizeof(T), cudaMemcpyDeviceToHost, stream_), "cudaMemcpy D2H");
      sync();
    }
    return h;
  }
  void sync() { cuda_check(cudaStreamSynchronize(stream_), "cudaStreamSynchronize"); }
  void need_iisph() {
    if (cfg_.pressure_solver != SPH_IISPH && cfg_.pressure_solver != SPH_IISPH_W_OST)
      throw Error(SPH_ERR_INVALID, "field only exists for IISPH solvers");
  }
  void ensure_partials(size_t n) {
    if (partials_.n < n) partials_.alloc(n);
  }

  Body make_body(const sph_rigid_init* r) {
    Body b{};
    if (!r) {
      b.dynamic = 0;
      b.mass = 1;
      b.q[0] = 1;
      return b;
    }
    if (!(r->mass != 0.0)) throw Error(SPH_ERR_INVALID, "Rigid body mass cannot be zero.");
    b.dynamic = 1;
    b.mass = r->mass;
    std::memcpy(b.inv_inertia_body, r->inertia_inv_body, sizeof b.inv_inertia_body);
    std::memcpy(b.com, r->center_of_mass, sizeof b.com);
    std::memcpy(b.q, r->orientation, sizeof b.q);
    std::memcpy(b.v, r->linear_velocity, sizeof b.v);
    // L = (R I_body R^T) omega ; derived: I^-1_world, omega (rigid_body_motion.rs:39-77)
    double Rm[9];
    host_rot(b.q, Rm);
    double Iw[9];
    host_sandwich(Rm, r->inertia_body, Iw);
    for (int i = 0; i < 3; ++i)
      b.L[i] = (Iw[i * 3] * r->angular_velocity[0] + Iw[i * 3 + 1] * r->angular_velocity[1]) +
               Iw[i * 3 + 2] * r->angular_velocity[2];
    host_sandwich(Rm, b.inv_inertia_body, b.inv_inertia_world);
    for (int i = 0; i < 3; ++i)
      b.omega[i] = (b.inv_inertia_world[i * 3] * b.L[0] + b.inv_inertia_world[i * 3 + 1] * b.L[1]) +
                   b.inv_inertia_world[i * 3 + 2] * b.L[2];
    return b;
  }
  static void host_rot(const double q[4], double R_[9]) {
    const double ww = q[0] * q[0], ii = q[1] * q[1], jj = q[2] * q[2], kk = q[3] * q[3];
    const double ij = q[1] * q[2] * 2.0, wk = q[0] * q[3] * 2.0, wj = q[0] * q[2] * 2.0;
    const double ik = q[1] * q[3] * 2.0, jk = q[2] * q[3] * 2.0, wi = q[0] * q[1] * 2.0;
    R_[0] = ww + ii - jj - kk; R_[1] = ij - wk; R_[2] = wj + ik;
    R_[3] = wk + ij; R_[4] = ww - ii + jj - kk; R_[5] = jk - wi;
    R_[6] = ik - wj; R_[7] = wi + jk; R_[8] = ww - ii - jj + kk;
  }
  static void host_sandwich(const double R_[9], const double M[9], double out[9]) {
    double t[9];
    for (int r = 0; r < 3; ++r)
      for (int c = 0; c < 3; ++c)
        t[r * 3 + c] = (R_[r * 3] * M[c] + R_[r * 3 + 1] * M[3 + c]) + R_[r * 3 + 2] * M[6 + c];
    for (int r = 0; r < 3; ++r)
      for (int c = 0; c < 3; ++c)
        out[r * 3 + c] = (t[r * 3] * R_[c * 3] + t[r * 3 + 1] * R_[c * 3 + 1]) + t[r * 3 + 2] * R_[c * 3 + 2];
  }

  void alloc_particles() {
    const size_t c = cap_;
    pos_.alloc(c); pos2_.alloc(c); vel_.alloc(c); vel2_.alloc(c); xv_.alloc(c); acc_.alloc(c);
    ref_.alloc(c); ref2_.alloc(c); fid_.alloc(c); fid2_.alloc(c);
    key_.alloc(c); slot_.alloc(c); perm_.alloc(c); ncnt_.alloc(c);
    press_.alloc(c);
    bW_.alloc(c); bG_.alloc(c); bGu_.alloc(c);
    const bool needs_vstar = cfg_.pressure_solver != SPH_SESPH;
    if (needs_vstar) vstar_.alloc(c);
    if (cfg_.pressure_solver == SPH_IISPH || cfg_.pressure_solver == SPH_IISPH_W_OST) {
      s_.alloc(c); aii_.alloc(c); xq_.alloc(c); xu_.alloc(c); uu_.alloc(c); TA_.alloc(c); TB_.alloc(c); SA_.alloc(c);
    }
    if (cfg_.pressure_solver == SPH_SESPH_W_SPLITTING) rho_pred_.alloc(c);
    if (cfg_.integration_scheme == SPH_TAKE_PREDICTED) { xint_.alloc(c); vint_.alloc(c); }
    K_ = (int)round_up(cfg_.neighbor_capacity ? cfg_.neighbor_capacity : 128, 4);
    nbr_.alloc((size_t)K_ * np_);
    halo_n_.alloc((size_t)blocks_for((long long)c));
    halo_idx_.alloc((size_t)blocks_for((long long)c) * (size_t)hcap_);
    ensure_partials(2 * (size_t)blocks_for((long long)c));
    press_.zero(stream_);
    bW_.zero(stream_); bG_.zero(stream_); bGu_.zero(stream_);
  }

  void choose_grid() {
    // Morton buckets: 2^(3m) with 2^m >= the scene extent in cells (so that
    // cells only share a bucket when they are 2^m cells apart), m in [2, 8].
    const double h = cfg_.kernel_support_radius;
    for (size_t s = 0; s < h_sample_x_.size() / 3; ++s)
      bbox_add(h_sample_x_[3 * s], h_sample_x_[3 * s + 1], h_sample_x_[3 * s + 2]);
    double ext = 4;
    if (bbox_.any)
      for (int d = 0; d < 3; ++d) ext = std::max(ext, (bbox_.mx[d] - bbox_.mn[d]) / h + 3.0);
    int m = 2;
    while (m < 8 && (double)(1u << m) < ext) ++m;
    mask_ = (1u << m) - 1u;
    T_ = 1u << (3 * m);
    count_.alloc(T_ + 2);
    start_.alloc(T_ + 2);
    count_.zero(stream_);
    tile_sums_.alloc((size_t)((T_ + 2 + kScanTile - 1) / kScanTile) + 1);
  }

  void setup_params() {
    const double h = cfg_.kernel_support_radius, sp = cfg_.rest_density_grid_spacing;
    P_.k = make_kernel_const<R>(h);
    P_.range = h;
    const double band = sizeof(R) == 4 ? 1e-5 : 1e-12;
    P_.range2_lo = (R)(h * h * (1.0 - band));
    P_.range2_hi = (R)(h * h * (1.0 + band));
    P_.spacing = sp;
    P_.V0 = (R)(sp * sp * sp);
    P_.visc_f = (R)(cfg_.fluid_viscosity * 2.0 * (3.0 + 2.0));
    P_.visc_b = (R)(cfg_.boundary_viscosity * 2.0 * (3.0 + 2.0));
    P_.eps_visc = (R)(0.01 * sp * sp);
    P_.gamma_p = (R)cfg_.boundary_pressure_acceleration_weighting;
    P_.gravity_mode = cfg_.gravity_mode;
    for (int d = 0; d < 3; ++d) P_.gc[d] = (R)cfg_.gravity_center[d];
    P_.disable_below = cfg_.disable_particles_below;
    P_.mask = mask_;
    P_.T = T_;
    P_.K = K_;
    P_.Np = (int)np_;
    P_.cfl = cfg_.cfl_time_step;
    P_.dt_fixed = cfg_.time_increment;
    P_.dt_max = cfg_.max_time_increment;
    P_.cfl_number = cfg_.cfl_number;
    P_.stiffness = (R)cfg_.stiffness;
    P_.omega = (R)cfg_.relaxation_factor;
    P_.min_diag = (R)cfg_.min_diagonal_element;
    P_.tde = cfg_.target_density_error;
    P_.iteration_cap = (int)cfg_.max_solver_iterations;
    P_.sorted_lists = sorted_lists_ ? 1 : 0;
  }

  // ---- launches ---------------------------------------------------------------
  template <class F>
  void with_nb(F&& f) {
    switch (nb_) {
      case 4: f(std::integral_constant<int, 4>{}); break;
      default: f(std::integral_constant<int, 8>{}); break;
    }
  }
  template <class Kern, class... Args>
  void launch(const char* name, Kern kernel, dim3 g, dim3 b, Args... args) {
    launch_s(name, kernel, g, b, 0, args...);
  }
  // dynamic shared memory of a halo-staging pass: nvec R4 and nscal R arrays
  size_t smem_of(int nvec, int nscal) const {
    return (size_t)hs_ * ((size_t)nvec * sizeof(R4<R>) + (size_t)nscal * sizeof(R));
  }
  NbrArgs nargs() const {
    NbrArgs N;
    N.nbr = nbr_.p;
    N.ncnt = ncnt_.p;
    N.hidx = halo_idx_.p;
    N.hn = halo_n_.p;
    N.K = K_;
    N.hcap = hcap_;
    N.hs = hs_;
    return N;
  }
  template <class Kern, class... Args>
  void launch_s(const char* name, Kern kernel, dim3 g, dim3 b, size_t smem, Args... args) {
    launch_impl(false, name, kernel, g, b, smem, args...);
  }
  // A launch that may overlap the end of the kernel before it (programmatic
  // dependent launch): only for kernels that call grid_dep_wait() before
  // reading what that kernel writes. Timed (profiling) runs launch plainly so
  // that the events around each kernel bracket it alone.
  bool dep_launch() const { return pdl_ && !profiling_; }
  template <class Kern, class... Args>
  void launch_dep(const char* name, Kern kernel, dim3 g, dim3 b, size_t smem, Args... args) {
    launch_impl(dep_launch(), name, kernel, g, b, smem, args...);
  }
  template <class Kern, class... Args>
  void launch_impl(bool dep, const char* name, Kern kernel, dim3 g, dim3 b, size_t smem, Args... args) {
    if (smem) allow_smem((const void*)kernel, smem);
    cudaEvent_t e1 = nullptr;
    if (profiling_ && !capturing_) {
      ProfEntry& pe = prof_[name];
      if (pe.used == pe.pool.size()) {
        cudaEvent_t a, c;
        cuda_check(cudaEventCreate(&a), "event");
        cuda_check(cudaEventCreate(&c), "event");
        pe.pool.push_back({a, c});
      }
      auto& pr = pe.pool[pe.used];
      pending_.push_back({name, pe.used});
      ++pe.used;
      cuda_check(cudaEventRecord(pr.first, stream_), "event");
      e1 = pr.second;
    }
    if (dep) {
      cudaLaunchConfig_t lc{};
      lc.gridDim = g;
      lc.blockDim = b;
      lc.dynamicSmemBytes = smem;
      lc.stream = stream_;
      cudaLaunchAttribute at[1];
      at[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
      at[0].val.programmaticStreamSerializationAllowed = 1;
      lc.attrs = at;
      lc.numAttrs = 1;
      cuda_check(cudaLaunchKernelEx(&lc, kernel, args...), name);
    } else {
      kernel<<<g, b, smem, stream_>>>(args...);
    }
    cuda_check(cudaGetLastError(), name);
    if (!capturing_) ++launches_;
    else if (!in_loop_body_) ++capture_kernels_;
    if (e1) cuda_check(cudaEventRecord(e1, stream_), "event");
  }
  void collect_profile() {
    if (pending_.empty()) return;
    sync();
    for (auto& p : pending_) {
      ProfEntry& pe = prof_[p.name];
      float ms = 0;
      cudaEventElapsedTime(&ms, pe.pool[p.idx].first, pe.pool[p.idx].second);
      pe.ms += ms;
      pe.count += 1;
    }
    pending_.clear();
    for (auto& kv : prof_) kv.second.used = 0;
  }

  // exclusive scan of count[0..m) into out, clearing count
  void scan(uint32_t* count, uint32_t m, uint32_t* out) {
    const int tiles = (int)((m + kScanTile - 1) / kScanTile);
    launch("scan", k_scan_tiles, dim3(tiles), dim3(kBlock), (const uint32_t*)count, (int)m, tile_sums_.p);
    launch("scan", k_scan_tile_sums, dim3(1), dim3(1024), tile_sums_.p, tiles);
    launch("scan", k_scan_apply, dim3(tiles), dim3(kBlock), count, (int)m, (const uint32_t*)tile_sums_.p, out);
  }

  void sort_particles() {
    const int nb = blocks_for((long long)n_);
    const int* dn = &d_sc_.p->n;
    scan(count_.p, T_ + 2, start_.p);
    launch("sort", k_scatter, dim3(nb), dim3(kBlock), dn, (const uint32_t*)key_.p, (const uint32_t*)slot_.p,
           (const uint32_t*)start_.p, perm_.p);
    launch("sort", k_bucket_order, dim3(nb), dim3(kBlock), dn, (const uint32_t*)key_.p, (const uint32_t*)start_.p,
           (const uint32_t*)ref_.p, perm_.p);
    launch("sort", k_gather_particles<R>, dim3(nb), dim3(kBlock), dn, (const uint32_t*)perm_.p,
           (const R4<R>*)pos_.p, (const R4<R>*)vel_.p, (const uint32_t*)ref_.p, (const uint32_t*)fid_.p,
           pos2_.p, vel2_.p, ref2_.p, fid2_.p);
    swap_particle_buffers();
  }
  void swap_particle_buffers() {
    std::swap(pos_.p, pos2_.p);
    std::swap(vel_.p, vel2_.p);
    std::swap(ref_.p, ref2_.p);
    std::swap(fid_.p, fid2_.p);
  }
  void swap_sample_buffers() {
    std::swap(xb_.p, xb2_.p);
    std::swap(vb_.p, vb2_.p);
    std::swap(sbid_.p, sbid2_.p);
    std::swap(sorig_.p, sorig2_.p);
  }

  void sort_samples() {
    const int nb = blocks_for((long long)ns_);
    const int* dn = ns_d_.p;
    launch("sample_sort", k_sample_key<R>, dim3(nb), dim3(kBlock), dn, (const R4<R>*)xb_.p, skey_.p, sslot_.p,
           scount_.p, P_.range, mask_);
    scan(scount_.p, T_ + 2, sstart_.p);
    launch("sample_sort", k_scatter, dim3(nb), dim3(kBlock), dn, (const uint32_t*)skey_.p, (const uint32_t*)sslot_.p,
           (const uint32_t*)sstart_.p, sperm_.p);
    launch("sample_sort", k_bucket_order, dim3(nb), dim3(kBlock), dn, (const uint32_t*)skey_.p,
           (const uint32_t*)sstart_.p, (const uint32_t*)sorig_.p, sperm_.p);
    launch("sample_sort", k_gather_samples<R>, dim3(nb), dim3(kBlock), dn, (const uint32_t*)sperm_.p,
           (const R4<R>*)xb_.p, (const R4<R>*)vb_.p, (const uint32_t*)sbid_.p, (const uint32_t*)sorig_.p,
           xb2_.p, vb2_.p, sbid2_.p, sorig2_.p);
    swap_sample_buffers();
  }

  SampleGrid<R> sample_grid() const {
    SampleGrid<R> G;
    G.xb = xb_.p; G.vb = vb_.p; G.bid = sbid_.p; G.orig = sorig_.p; G.start = sstart_.p; G.mask = mask_;
    return G;
  }

  void init_sample_boundaries() {
    ns_ = h_sample_bid_.size();
    xb_.alloc(ns_); xb2_.alloc(ns_); vb_.alloc(ns_); vb2_.alloc(ns_); xbody_.alloc(ns_);
    sbid_.alloc(ns_); sbid2_.alloc(ns_); sorig_.alloc(ns_); sorig2_.alloc(ns_);
    skey_.alloc(ns_); sslot_.alloc(ns_); sperm_.alloc(ns_);
    scount_.alloc(T_ + 2); sstart_.alloc(T_ + 2);
    scount_.zero(stream_);
    ns_d_.alloc(1);
    const int nsi = (int)ns_;
    copy_h2d(ns_d_.p, &nsi, 1);
    std::vector<R4<R>> hx(ns_), hb(ns_);
    std::vector<uint32_t> ho(ns_);
    for (size_t s = 0; s < ns_; ++s) {
      hx[s] = R4<R>{(R)h_sample_x_[3 * s], (R)h_sample_x_[3 * s + 1], (R)h_sample_x_[3 * s + 2], R(0)};
      hb[s] = hx[s];
      ho[s] = (uint32_t)s;
    }
    copy_h2d(xb_.p, hx.data(), ns_);
    copy_h2d(xbody_.p, hb.data(), ns_);
    copy_h2d(sbid_.p, h_sample_bid_.data(), ns_);
    copy_h2d(sorig_.p, ho.data(), ns_);
    vb_.zero(stream_);
    const int nb = blocks_for((long long)ns_);
    // dynamic boundaries: world positions from the initial pose
    // (StaticSampleBoundary::initialize -> update_positions_and_velocities)
    if (any_dynamic_)
      launch("body_samples", k_body_samples<R>, dim3(nb), dim3(kBlock), (const int*)ns_d_.p,
             (const Body*)bodies_d_.p, (const R4<R>*)xbody_.p, (const uint32_t*)sorig_.p,
             (const uint32_t*)sbid_.p, xb_.p, vb_.p);
    sort_samples();
    launch("sample_volumes", k_sample_volumes<R>, dim3(nb), dim3(kBlock), (const int*)ns_d_.p, sample_grid(),
           xb2_.p, cfg_.boundary_rest_volume_weighting, P_);
    // the volumes were written into the spare buffer; carry the other lanes over
    std::vector<R4<R>> vols = fetch(xb2_.p, ns_);
    std::vector<R4<R>> cur = fetch(xb_.p, ns_);
    for (size_t s = 0; s < ns_; ++s) cur[s].w = vols[s].w;
    copy_h2d(xb_.p, cur.data(), ns_);
  }

  void set_volume_map_aabb(int bi, const double* c, const double* hext) override {
    if (initialized_) throw Error(SPH_ERR_STATE, "bounding boxes are set before initialize");
    if (bi < 0 || bi >= (int)fields_.size()) throw Error(SPH_ERR_INVALID, "not a volume-map boundary");
    for (int d = 0; d < 3; ++d)
      if (!std::isfinite(c[d]) || !std::isfinite(hext[d]) || hext[d] < 0.0)
        throw Error(SPH_ERR_INVALID, "bad bounding box");
    FieldPair& f = *fields_[bi];
    f.has_aabb = true;
    for (int d = 0; d < 3; ++d) {
      f.aabb_c[d] = c[d];
      f.aabb_h[d] = hext[d];
    }
  }

  // Contact runs when some pair of boxed boundaries has a dynamic body. Its
  // task capacity bounds the sub-cells of every such pair: an overlap is no
  // wider than either box, and a rotated box no wider than twice the norm of
  // its half extents.
  void init_contacts() {
    const int nb = (int)fields_.size();
    const double target = cfg_.kernel_support_radius * 0.5;  // CONTACT_CELL_SIZE_FACTOR (:60)
    double total = 0.0;
    for (int i = 0; i < nb; ++i)
      for (int j = i + 1; j < nb; ++j) {
        const FieldPair &a = *fields_[i], &b = *fields_[j];
        if (!a.has_aabb || !b.has_aabb || (!bodies_[i].dynamic && !bodies_[j].dynamic)) continue;
        const double ra = 2.0 * std::sqrt(a.aabb_h[0] * a.aabb_h[0] + a.aabb_h[1] * a.aabb_h[1] + a.aabb_h[2] * a.aabb_h[2]);
        const double rb = 2.0 * std::sqrt(b.aabb_h[0] * b.aabb_h[0] + b.aabb_h[1] * b.aabb_h[1] + b.aabb_h[2] * b.aabb_h[2]);
        double cnt = 1.0;
        for (int d = 0; d < 3; ++d) {
          const double ea = bodies_[i].dynamic ? ra : 2.0 * a.aabb_h[d];
          const double eb = bodies_[j].dynamic ? rb : 2.0 * b.aabb_h[d];
          cnt *= std::floor(std::min(ea, eb) / target) + 2.0;
        }
        total += cnt;
      }
    contact_ = total > 0.0;
    if (!contact_) return;
    if (total > 4.0e6) throw Error(SPH_ERR_CAPACITY, "rigid-rigid contact would need more than 4M sub-cells");
    contact_task_cap_ = (int)total;
    contact_pairs_.alloc((size_t)kMaxBodies * (kMaxBodies - 1) / 2);
    contact_cells_.alloc((size_t)contact_task_cap_);
    contact_state_.alloc((size_t)contact_task_cap_);
    contact_idx_.alloc((size_t)contact_task_cap_);
    contact_scalars_.alloc(1);
    contact_scalars_.zero(stream_);
    std::vector<double> gx, gw;
    gauss_legendre_nodes(kContactQuad, gx, gw);
    for (int k = 0; k < kContactQuad; ++k) {
      contact_gl_.x[k] = gx[k];
      contact_gl_.w[k] = gw[k];
    }
  }

  // VolumeMapBoundary::step_forward_in_time (volume_map_boundary.rs:1440-1453):
  // contact forces first; the body step that follows integrates them.
  void issue_contacts() {
    if (!contact_) return;
    const double h = cfg_.kernel_support_radius;
    launch("contact_tasks", k_contact_tasks, dim3(1), dim3(32), (const VMDesc*)vms_.p, (const Body*)bodies_d_.p,
           nbodies_, h * 0.5, contact_pairs_.p, contact_scalars_.p, contact_task_cap_);
    launch("contact_build", k_contact_build, dim3(std::min(contact_task_cap_, 2 * 148)), dim3(kContactThreads),
           (const VMDesc*)vms_.p, (const Body*)bodies_d_.p, (const ContactPair*)contact_pairs_.p,
           (const ContactScalars*)contact_scalars_.p, contact_cells_.p, contact_gl_, h, (const Scalars*)d_sc_.p);
    launch("contact_solve", k_contact_solve, dim3(1), dim3(kContactSolveThreads), bodies_d_.p, nbodies_,
           (const ContactCell*)contact_cells_.p, contact_scalars_.p, contact_idx_.p, contact_state_.p,
           (const Scalars*)d_sc_.p, kContactSweepCap, (int)contact_fixed_sweeps_);
  }

  void set_dependent_launch(bool on) override {
    if (chunk_steps_) throw Error(SPH_ERR_STATE, "a chunk of graph steps is in flight");
    if (pdl_ == on) return;
    pdl_ = on;
    destroy_graphs();  // the captured launches carry the old setting
  }
  void set_contact_sweeps(uint32_t fixed) override {
    if (chunk_steps_) throw Error(SPH_ERR_STATE, "a chunk of graph steps is in flight");
    if (fixed > (uint32_t)kContactSweepCap) throw Error(SPH_ERR_INVALID, "more contact sweeps than the cap");
    if (fixed == contact_fixed_sweeps_) return;
    contact_fixed_sweeps_ = fixed;
    destroy_graphs();  // the captured contact solve carries the old count
  }
  uint32_t contact_sweeps() const override { return contact_fixed_sweeps_; }
  void contact_stats(uint32_t* out) override {
    ContactScalars c{};
    if (contact_) c = fetch(contact_scalars_.p, 1)[0];
    out[0] = (uint32_t)c.ncells;
    out[1] = (uint32_t)c.iterations;
    out[2] = (uint32_t)c.overflow;
    out[3] = (uint32_t)c.capped;
  }

  void init_volume_maps() {
    const int nvm = (int)fields_.size();
    std::vector<VMDesc> h(nvm);
    for (int b = 0; b < nvm; ++b) {
      auto fill = [](DevField& F, const sph_grid_desc& g, const double* nodes) {
        for (int d = 0; d < 3; ++d) {
          F.xmin[d] = g.x_min[d];
          F.xmax[d] = g.x_max[d];
          F.n[d] = (int)g.n[d];
        }
        F.dx = g.dx;
        F.NX = 3 * g.n[0] + 1;
        F.NY = 3 * g.n[1] + 1;
        F.nodes = nodes;
      };
      fill(h[b].sdf, fields_[b]->sdf_desc, fields_[b]->sdf.p);
      fill(h[b].vm, fields_[b]->vm_desc, fields_[b]->vm.p);
      h[b].body = bodies_[b].dynamic ? b : -1;
      h[b].has_aabb = fields_[b]->has_aabb ? 1 : 0;
      for (int d = 0; d < 3; ++d) {
        h[b].aabb_c[d] = fields_[b]->aabb_c[d];
        h[b].aabb_h[d] = fields_[b]->aabb_h[d];
      }
    }
    vms_.alloc(nvm);
    copy_h2d(vms_.p, h.data(), (size_t)nvm);
    vmx_.alloc((size_t)nvm * np_);
    vmv_.alloc((size_t)nvm * np_);
    vm_near_.alloc(std::max<size_t>(cap_, 1));
    vmv_.zero(stream_);
  }

  BoundaryArgs<R> bargs() {
    BoundaryArgs<R> B{};
    B.kind = boundary_kind_;
    if (boundary_kind_ == 1) B.grid = sample_grid();
    B.vmx = vmx_.p;
    B.vmv = vmv_.p;
    B.vms = vms_.p;
    B.nvm = (int)fields_.size();
    B.bodies = bodies_d_.p;
    B.any_dynamic = any_dynamic_ ? 1 : 0;
    B.bW = bW_.p;
    B.bG = bG_.p;
    B.bGu = bGu_.p;
    B.body_partials = body_partials_.p;
    B.nbodies = nbodies_;
    return B;
  }

  void body_reduce(int producer_blocks) {
    if (!any_dynamic_) return;
    launch("body_reduce", k_body_reduce, dim3(nbodies_), dim3(kBlock), bodies_d_.p, nbodies_,
           (const double*)body_partials_.p, producer_blocks);
  }

  // One Jacobi iteration: pressure accelerations of the current pressures, then
  // the pressure update with the residual reduction.
  // first: the solve's first sweep, whose pass A follows the source pass
  // (which writes TA) and so must not overlap it.
  void iisph_iteration(int after, bool first) {
    const int nb = blocks_for((long long)n_);
    NbrArgs N = nargs();
    N.hs = sweep_hs_;
    const size_t sm_a = (size_t)sweep_hs_ * sizeof(R4<R>);
    const size_t sm_b = (size_t)sweep_hs_ * (sizeof(R4<R>) + sizeof(R2<R>));
    N.ahead = resident_blocks((const void*)k_sweep_accel<R>, sm_a);
    launch_impl(!first && dep_launch(), "iisph_pressure_accel", k_sweep_accel<R>, dim3(nb), dim3(kBlock),
             sm_a, (const Scalars*)d_sc_.p, (const R*)press_.p, (const R4<R>*)TA_.p, (const R4<R>*)xq_.p, N,
             xu_.p, uu_.p, P_, (R4<R>*)nullptr, (const R4<R>*)nullptr);
    N.ahead = resident_blocks((const void*)k_sweep_jacobi<R>, sm_b);
    launch_dep("iisph_jacobi", k_sweep_jacobi<R>, dim3(nb), dim3(kBlock), sm_b, d_sc_.p, (const R4<R>*)TB_.p,
             (const R2<R>*)SA_.p, (const R4<R>*)xu_.p, (const R2<R>*)uu_.p, N, press_.p, xq_.p, partials_.p,
             after, P_);
  }
  // The distance, in blocks, of a sweep pass's L2 prefetch (0 when it is
  // off): half the blocks resident on the whole GPU at once, so a block's
  // lines arrive about half a block lifetime ahead (on the 1M scene a whole
  // wave ahead measured 2 % slower, two waves 10 %).
  int resident_blocks(const void* fn, size_t smem) {
    if (!prefetch_) return 0;
    auto it = resident_.find({fn, smem});
    if (it != resident_.end()) return it->second;
    allow_smem(fn, smem);
    int per_sm = 0, sms = 0;
    cuda_check(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, fn, kBlock, smem), "occupancy");
    cuda_check(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device), "attribute");
    const int r = std::max(0, per_sm * sms / 2);
    resident_[{fn, smem}] = r;
    return r;
  }

  // The pressure acceleration after a solve (a13 with the solved pressures;
  // OUT 1: +=, OUT 2: overwrite) as one more sweep pass A: the per-solve
  // constants and the {x, V p} records of the last sweep are still current.
  // Only without reaction forces onto dynamic bodies.
  template <int OUT>
  void final_pressure_accel() {
    const int nb = blocks_for((long long)n_);
    NbrArgs N = nargs();
    N.hs = sweep_hs_;
    launch_s("pressure_accel", k_sweep_accel<R, OUT>, dim3(nb), dim3(kBlock), (size_t)sweep_hs_ * sizeof(R4<R>),
             (const Scalars*)d_sc_.p, (const R*)press_.p, (const R4<R>*)TA_.p, (const R4<R>*)xq_.p, N,
             (R4<R>*)nullptr, (R2<R>*)nullptr, P_, acc_.p, (const R4<R>*)TB_.p);
  }

  // resolve_pressure_globally's loop (iisph.rs:419-550). Sweeps run on the
  // device and stop themselves once converged; the host only checks the flag
  // after a batch sized by the previous solve.
  void solve_loop(int after) {
    if (capturing_ && after < 0) {
      solve_loop_graph();
      return;
    }
    int batch = after >= 0 ? after + 1 : std::max(3, last_iters_);
    if (after < 0 && cfg_.max_solver_iterations) batch = std::min(batch, (int)cfg_.max_solver_iterations);
    // Timed (profiling) solves run one sweep per host check, so that every
    // timed sweep launch does a sweep's work (no launch that finds the loop
    // converged and returns); the results are the same either way.
    if (profiling_ && after < 0) batch = 1;
    for (int k = 0; k < batch; ++k) iisph_iteration(after, k == 0);
    if (after >= 0) return;
    int launched = batch;
    for (;;) {
      cuda_check(cudaMemcpyAsync(&h_sc_->converged, &d_sc_.p->converged, sizeof(int), cudaMemcpyDeviceToHost, stream_), "memcpy");
      sync();
      if (h_sc_->converged) break;
      const int more = profiling_ ? 1 : launched < 16 ? 2 : 4;
      for (int k = 0; k < more; ++k) iisph_iteration(after, false);
      launched += more;
    }
  }

  void calc_acceleration() {
    const int nb = blocks_for((long long)n_);
    if (any_dynamic_)
      launch("body_gravity", k_body_gravity, dim3(1), dim3(32), bodies_d_.p, nbodies_, cfg_.gravity_mode,
             cfg_.gravity_center[0], cfg_.gravity_center[1], cfg_.gravity_center[2]);
    const Scalars* csc = d_sc_.p;
    const auto xv = (const R4<R>*)xv_.p;
    const auto vel = (const R4<R>*)vel_.p;
    const NbrArgs nbr = nargs();
    const size_t sm_xv = smem_of(2, 0), sm_xp = smem_of(1, 1);
    with_nb([&](auto NBc) {
    constexpr int NB = decltype(NBc)::value;
    switch (cfg_.pressure_solver) {
      case SPH_SESPH:
        launch_s("accel_sesph", k_accel<R, 1>, dim3(nb), dim3(kBlock), sm_xv, csc, xv, vel, nbr, bargs(), acc_.p,
               vstar_.p, press_.p, 0, P_);
        body_reduce(nb);
        break;
      case SPH_SESPH_W_SPLITTING:
        launch_s("accel_nonpressure", k_accel<R, 0>, dim3(nb), dim3(kBlock), sm_xv, csc, xv, vel, nbr, bargs(),
               acc_.p, vstar_.p, press_.p, 1, P_);
        body_reduce(nb);
        launch_s("split_density", k_split_density<R, NB>, dim3(nb), dim3(kBlock), sm_xv, csc, xv, vel,
               (const R4<R>*)vstar_.p, nbr, bargs(), press_.p, rho_pred_.p, P_);
        launch_s("pressure_accel", k_pressure_accel<R, 1>, dim3(nb), dim3(kBlock), sm_xp, csc, xv, vel,
               (const R*)press_.p, nbr, bargs(), acc_.p, 1, P_);
        body_reduce(nb);
        break;
      case SPH_IISPH:
        launch_s("accel_nonpressure", k_accel<R, 0>, dim3(nb), dim3(kBlock), sm_xv, csc, xv, vel, nbr, bargs(),
               acc_.p, vstar_.p, press_.p, 1, P_);
        body_reduce(nb);
        launch_s("iisph_source_diag", k_iisph_source_diag<R, 1>, dim3(nb), dim3(kBlock), sm_xv, csc, xv, vel,
               (const R4<R>*)vstar_.p, nbr, bargs(), s_.p, aii_.p, press_.p, TA_.p, TB_.p, SA_.p, xq_.p, P_);
        solve_loop(-1);
        if (any_dynamic_) {
          launch_s("pressure_accel", k_pressure_accel<R, 1>, dim3(nb), dim3(kBlock), sm_xp, csc, xv, vel,
                 (const R*)press_.p, nbr, bargs(), acc_.p, 1, P_);
          body_reduce(nb);
        } else {
          final_pressure_accel<1>();
        }
        break;
      case SPH_IISPH_W_OST:
        launch_s("accel_nonpressure", k_accel<R, 0>, dim3(nb), dim3(kBlock), sm_xv, csc, xv, vel, nbr, bargs(),
               acc_.p, vstar_.p, press_.p, 1, P_);
        launch_s("iisph_source_diag", k_iisph_source_diag<R, 0>, dim3(nb), dim3(kBlock), sm_xv, csc, xv, vel,
               (const R4<R>*)vstar_.p, nbr, bargs(), s_.p, aii_.p, press_.p, TA_.p, TB_.p, SA_.p, xq_.p, P_);
        solve_loop(3);
        final_pressure_accel<2>();  // IISPHwOST takes no dynamic boundaries
        launch("ost_predict", k_ost_predict<R>, dim3(nb), dim3(kBlock), d_sc_.p, (const R4<R>*)acc_.p, vstar_.p);
        launch_s("iisph_source_diag", k_iisph_source_diag<R, 1>, dim3(nb), dim3(kBlock), sm_xv, csc, xv, vel,
               (const R4<R>*)vstar_.p, nbr, bargs(), s_.p, aii_.p, press_.p, TA_.p, TB_.p, SA_.p, xq_.p, P_);
        solve_loop(-1);
        final_pressure_accel<2>();
        launch("ost_commit", k_ost_commit<R>, dim3(nb), dim3(kBlock), csc, xv, vel, (const R4<R>*)vstar_.p,
               (const R4<R>*)acc_.p, xint_.p, vint_.p);
        break;
    }
    });
  }

 public:
  // System::update (sph/mod.rs:674-731); mode 0/1 integrate first (EulerCromer
  // / TakePredicted, euler_cromer.rs:12-25 / take_predicted.rs:14-27), 2 not.
  void update(int mode) {
    issue_update(mode);
    cuda_check(cudaMemcpyAsync(h_sc_, d_sc_.p, sizeof(Scalars), cudaMemcpyDeviceToHost, stream_), "memcpy");
    sync();
    collect_profile();
    avg_density_ = h_sc_->avg_density;
    if (h_sc_->iterations > 0) last_iters_ = h_sc_->iterations;
    if (h_sc_->max_nbrs > K_ || h_sc_->max_halo > hcap_) {
      // Neighbor or halo capacity exceeded: grow it and redo the update on
      // the same (already integrated) state. Reaction forces gathered so far
      // are discarded first; they are rebuilt by the redo.
      grow_capacity(h_sc_->max_nbrs, h_sc_->max_halo);
      zero_body_forces();
      finish_disable();
      update(2);
      return;
    }
    finish_disable();
  }

 private:
  // The kernels of one update, from integration to the average density.
  void issue_update(int mode) {
    const int nb = blocks_for((long long)n_);
    const bool sample_dyn = boundary_kind_ == 1 && any_dynamic_;
    launch("integrate_key", k_integrate_key<R>, dim3(nb), dim3(kBlock), d_sc_.p, pos_.p, vel_.p,
           (const R4<R>*)acc_.p, (const R4<R>*)xint_.p, (const R4<R>*)vint_.p, mode, key_.p, slot_.p,
           count_.p, P_);
    launch("prologue", k_prologue<R>, dim3(1), dim3(1), d_sc_.p, P_,
           (capturing_ && cfg_.cfl_time_step) ? 1 : 0);
    sort_particles();
    if ((early_xo_ || early_vo_) && !capturing_ && !early_done_) issue_early_readback();
    if (sample_dyn) {
      const int sb = blocks_for((long long)ns_);
      launch("body_samples", k_body_samples<R>, dim3(sb), dim3(kBlock), (const int*)ns_d_.p,
             (const Body*)bodies_d_.p, (const R4<R>*)xbody_.p, (const uint32_t*)sorig_.p,
             (const uint32_t*)sbid_.p, xb_.p, vb_.p);
      sort_samples();
    }
    if (boundary_kind_ == 1)
      launch("boundary_samples", k_sample_aggregate<R>, dim3(nb), dim3(kBlock), d_sc_.p, (const R4<R>*)pos_.p,
             sample_grid(), bW_.p, bG_.p, bGu_.p, P_);
    else if (boundary_kind_ == 2) {
      launch("vm_near", k_vm_near<R>, dim3(nb), dim3(kBlock), d_sc_.p, (const R4<R>*)pos_.p,
             (const VMDesc*)vms_.p, (int)fields_.size(), (const Body*)bodies_d_.p, vm_near_.p, vmx_.p, vmv_.p,
             bW_.p, bG_.p, bGu_.p, P_);
      launch("boundary_samples", k_vm_sample<R>, dim3(nb), dim3(kBlock), d_sc_.p, (const uint32_t*)vm_near_.p,
             (const R4<R>*)pos_.p, (const VMDesc*)vms_.p, (int)fields_.size(), (const Body*)bodies_d_.p, vmx_.p,
             vmv_.p, bW_.p, bG_.p, bGu_.p, P_);
    }
    launch_s("neighbors_density", k_neighbors_density<R>, dim3(nb), dim3(kBlock), kSearchSmem, d_sc_.p,
             (const R4<R>*)pos_.p, (const uint32_t*)start_.p, xv_.p, nbr_.p, ncnt_.p, halo_idx_.p, halo_n_.p,
             (const R*)bW_.p, boundary_kind_ ? 1 : 0, hcap_, P_);
    // IISPH in f32 re-reads the lists in every sweep pass: order them for
    // shared-memory banks once per update
    if (sizeof(R) == 4 && (cfg_.pressure_solver == SPH_IISPH || cfg_.pressure_solver == SPH_IISPH_W_OST))
      launch_s("order_lists", k_order_lists<64, kOrderResidues>, dim3(nb), dim3(kBlock),
               order_lists_smem(64, kOrderResidues), (const Scalars*)d_sc_.p, nbr_.p, (const uint32_t*)ncnt_.p, K_);
    calc_acceleration();
    launch("avg_density", k_avg_density<R>, dim3(nb), dim3(kBlock), d_sc_.p, (const R4<R>*)xv_.p,
           (const R4<R>*)vel_.p, partials_.p, P_);
  }

  // sph_step_host's readback of the sorted, integrated state in reference
  // order: scatter on the engine's stream, copy on the copy stream.
  void issue_early_readback() {
    launch("state_io", k_state_out<R>, dim3(blocks_for((long long)n_)), dim3(kBlock), (int)n_,
           (const uint32_t*)ref_.p, (const R4<R>*)pos_.p, (const R4<R>*)vel_.p, early_xo_ ? stage_x_.p : nullptr,
           early_vo_ ? stage_v_.p : nullptr);
    cuda_check(cudaEventRecord(io_ready_, stream_), "event");
    cuda_check(cudaStreamWaitEvent(io_stream_, io_ready_, 0), "event");
    if (early_xo_)
      cuda_check(cudaMemcpyAsync(early_xo_, stage_x_.p, 3 * n_ * sizeof(double), cudaMemcpyDeviceToHost, io_stream_),
                 "D2H");
    if (early_vo_)
      cuda_check(cudaMemcpyAsync(early_vo_, stage_v_.p, 3 * n_ * sizeof(double), cudaMemcpyDeviceToHost, io_stream_),
                 "D2H");
    early_done_ = true;
  }

  // Grows the neighbor-list and halo capacities past the counts a step
  // needed (with headroom: compressing scenes raise them step after step).
  // Returns whether anything grew.
  bool grow_capacity(int max_nbrs, int max_halo) {
    bool grew = false;
    if (max_nbrs > K_) {
      K_ = (int)round_up((size_t)max_nbrs * 3 / 2 + 8, 8);  // multiple of 4 (64-bit groups)
      P_.K = K_;
      nbr_.alloc((size_t)K_ * np_);
      grew = true;
    }
    if (max_halo > hcap_) {
      if (max_halo > 65535)
        throw Error(SPH_ERR_CAPACITY, "a block's neighborhood holds more than 65535 particles");
      hcap_ = (int)std::min<size_t>(65535, round_up((size_t)max_halo * 3 / 2, 256));
      halo_idx_.alloc((size_t)blocks_for((long long)cap_) * (size_t)hcap_);
      grew = true;
    }
    return grew;
  }

  void zero_body_forces() {
    if (!any_dynamic_) return;
    std::vector<Body> hb = fetch(bodies_d_.p, (size_t)nbodies_);
    for (auto& b : hb) for (int c = 0; c < 3; ++c) { b.F[c] = 0; b.T[c] = 0; }
    copy_h2d(bodies_d_.p, hb.data(), hb.size());
  }

  // Reference-order bookkeeping after disabling particles below the threshold:
  // Fluid::disable swaps each removed particle with the last active one
  // (fluid.rs:159-210), which renumbers the survivors. The device already
  // moved the removed particles behind the active range; replay the swaps on
  // the reference indices here.
  void finish_disable() {
    const int below = h_sc_->n_below;
    const size_t n_old = (size_t)h_sc_->n;
    const size_t n_new = (size_t)h_sc_->n_active;
    // set up the scalars for the next update
    Scalars next = *h_sc_;
    next.n = (int)n_new;
    next.n_below = 0;
    next.max_speed = 0;
    if (below > 0) {
      std::vector<uint32_t> ref_all = fetch(ref_.p, n_old);
      std::vector<char> is_below(n_old, 0);
      for (size_t d = n_new; d < n_old; ++d) is_below[ref_all[d]] = 1;
      std::vector<uint32_t> cur(n_old);
      for (size_t k = 0; k < n_old; ++k) cur[k] = (uint32_t)k;
      size_t id = 0, nact = n_old;
      while (id < nact) {
        if (is_below[cur[id]]) {
          --nact;
          std::swap(cur[id], cur[nact]);
        } else {
          ++id;
        }
      }
      std::vector<uint32_t> newref(n_old, 0);
      for (size_t k = 0; k < n_new; ++k) newref[cur[k]] = (uint32_t)k;
      for (size_t d = 0; d < n_new; ++d) ref_all[d] = newref[ref_all[d]];
      copy_h2d(ref_.p, ref_all.data(), n_new);
      n_ = n_new;
    }
    copy_h2d(d_sc_.p, &next, 1);
    *h_sc_ = next;
  }

  // ---- graph-captured stepping --------------------------------------------------
  // One step (body step, update, epilogue) is captured into a CUDA graph; the
  // IISPH Jacobi loop inside it is a conditional while-node whose body (two
  // sweep kernels and a condition kernel) repeats until the sweep kernel sets
  // `converged`. The particle sort ping-pongs between two buffer sets, so two
  // graphs are captured, one per starting set. A chunk of graph launches
  // ends with one copy of the step scalars; when any step of it needed host
  // work the per-step path would have done (neighbor overflow, disabled
  // particles, a loop that hit its limit), the chunk's starting state is put
  // back from a device snapshot and the chunk is replayed on that path.
 public:
  void set_step_graphs(uint32_t chunk) override {
    if (chunk_steps_) throw Error(SPH_ERR_STATE, "a chunk of graph steps is in flight");
    graph_chunk_ = chunk;
    if (!chunk) destroy_graphs();
    else if (initialized_) prepare_graphs();
  }
  uint32_t step_graph_chunk() const override { return graph_chunk_; }
  uint64_t graph_replays() const override { return graph_replays_; }

  void get_tuning(sph_tuning* out) const override {
    out->gather_batch = (uint32_t)nb_;
    out->halo_stage = (uint32_t)hs_;
    out->sweep_stage = (uint32_t)sweep_hs_;
  }
  void set_tuning(const sph_tuning& t) override {
    if (chunk_steps_) throw Error(SPH_ERR_STATE, "a chunk of graph steps is in flight");
    if (t.gather_batch != 4 && t.gather_batch != 8) throw Error(SPH_ERR_INVALID, "gather batch must be 4 or 8");
    // the widest staged record is {x, v, m} of the source/diagonal pass
    const size_t record = 2 * sizeof(R4<R>) + sizeof(R);
    if (t.halo_stage > 65535u || (size_t)t.halo_stage * record + kStaticSmemReserve > kMaxSmemPerBlock)
      throw Error(SPH_ERR_INVALID, "halo stage exceeds a block's shared memory");
    // the sweep's widest staging is pass B's {x, V a_x} and {V a_y, V a_z}
    const size_t sweep_record = sizeof(R4<R>) + sizeof(R2<R>);
    if (t.sweep_stage > 65535u || (size_t)t.sweep_stage * sweep_record + kStaticSmemReserve > kMaxSmemPerBlock)
      throw Error(SPH_ERR_INVALID, "sweep stage exceeds a block's shared memory");
    if ((int)t.gather_batch == nb_ && (int)t.halo_stage == hs_ && (int)t.sweep_stage == sweep_hs_) return;
    nb_ = (int)t.gather_batch;
    hs_ = (int)t.halo_stage;
    sweep_hs_ = (int)t.sweep_stage;
    destroy_graphs();  // the captured launches carry the old parameters
  }

  void chunk_begin(uint32_t c) override {
    if (!initialized_) throw Error(SPH_ERR_STATE, "initialize before stepping");
    if (chunk_steps_) throw Error(SPH_ERR_STATE, "a chunk of graph steps is in flight");
    if (c == 0) return;
    prepare_graphs();
    take_snapshot();
    chunk_start_sc_ = *h_sc_;
    chunk_t0_ = std::chrono::steady_clock::now();
    launch("chunk_begin", k_chunk_begin, dim3(1), dim3(1), d_sc_.p, current_time_);
    for (uint32_t k = 0; k < c; ++k) {
      StepGraph& g = graphs_[0].key == (const void*)pos_.p ? graphs_[0] : graphs_[1];
      if (g.key != (const void*)pos_.p) throw Error(SPH_ERR_STATE, "step graph does not match the buffers");
      swap_particle_buffers();
      if (boundary_kind_ == 1 && any_dynamic_) swap_sample_buffers();
      cuda_check(cudaGraphLaunch(g.exec, stream_), "cudaGraphLaunch");
    }
    cuda_check(cudaMemcpyAsync(h_chunk_sc_, d_sc_.p, sizeof(Scalars), cudaMemcpyDeviceToHost, stream_), "memcpy");
    cuda_check(cudaEventRecord(chunk_event_, stream_), "cudaEventRecord");
    chunk_steps_ = c;
  }

  bool chunk_ready() override {
    if (!chunk_steps_) return true;
    return cudaEventQuery(chunk_event_) != cudaErrorNotReady;
  }

  ChunkOutcome chunk_finish() override {
    ChunkOutcome o;
    if (!chunk_steps_) return o;
    const uint32_t c = chunk_steps_;
    chunk_steps_ = 0;
    cuda_check(cudaEventSynchronize(chunk_event_), "chunk");
    const Scalars s = *h_chunk_sc_;
    o.steps = c;
    if (s.trouble) {
      restore_snapshot();
      *h_sc_ = chunk_start_sc_;
      ++graph_replays_;
      o.replayed = true;
      if (s.trouble == 1u && grow_capacity(s.chunk_max_nbrs, s.chunk_max_halo)) {
        // only the neighbor or halo capacity ran out: grow it past what the
        // chunk needed and run the chunk again as graphs (recaptured)
        chunk_begin(c);
        return chunk_finish();
      }
      o.status = step_plain(c);
      return o;
    }
    *h_sc_ = s;
    steps_ += c;
    if (cfg_.cfl_time_step) current_time_ = s.time_acc;
    avg_density_ = s.avg_density;
    if (s.iterations > 0) last_iters_ = s.iterations;
    launches_ += (uint64_t)c * graphs_[0].kernels + 3ull * s.loop_sweeps;
    wall_ = std::chrono::duration<double>(std::chrono::steady_clock::now() - chunk_t0_).count() / c;
    o.status = s.status_any == 2 ? SPH_NOT_CONVERGED : SPH_OK;
    return o;
  }

 private:
  struct StepGraph {
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t exec = nullptr;
    const void* key = nullptr;  // position buffer the captured step starts from
    uint64_t kernels = 0;       // kernel nodes outside the solver loops
  };
  static constexpr int kGraphSweepLimit = 10000;  // while-node bound without a sweep cap
  StepGraph graphs_[2];
  uint32_t graph_chunk_ = 0, chunk_steps_ = 0;
  size_t graph_n_ = 0;
  int graph_K_ = 0, graph_hcap_ = 0;
  bool capturing_ = false, in_loop_body_ = false;
  uint64_t capture_kernels_ = 0, graph_replays_ = 0;
  cudaStream_t body_stream_ = nullptr;
  cudaEvent_t chunk_event_ = nullptr;
  Scalars* h_chunk_sc_ = nullptr;
  Scalars chunk_start_sc_{};
  std::chrono::steady_clock::time_point chunk_t0_;
  DBuf<R4<R>> snap_pos_, snap_vel_, snap_acc_, snap_xint_, snap_vint_;
  DBuf<uint32_t> snap_ref_, snap_fid_;
  DBuf<Body> snap_bodies_;
  DBuf<Scalars> snap_sc_;

  void destroy_graphs() {
    for (auto& g : graphs_) {
      if (g.exec) cudaGraphExecDestroy(g.exec);
      if (g.graph) cudaGraphDestroy(g.graph);
      g = StepGraph{};
    }
    graph_n_ = 0;
    graph_K_ = 0;
  }

  void prepare_graphs() {
    if (graphs_[0].exec && graph_n_ == n_ && graph_K_ == K_ && graph_hcap_ == hcap_) return;
    destroy_graphs();
    if (!body_stream_) cuda_check(cudaStreamCreateWithFlags(&body_stream_, cudaStreamNonBlocking), "cudaStreamCreate");
    if (!chunk_event_) cuda_check(cudaEventCreateWithFlags(&chunk_event_, cudaEventDisableTiming), "cudaEventCreate");
    if (!h_chunk_sc_) cuda_check(cudaMallocHost((void**)&h_chunk_sc_, sizeof(Scalars)), "cudaMallocHost");
    alloc_snapshot();
    // capturing swaps the host-side buffer pointers as a launch would; two
    // captures in a row bring them back to where they started
    capture_step(graphs_[0]);
    capture_step(graphs_[1]);
    if (graphs_[0].key != (const void*)pos_.p) throw Error(SPH_ERR_STATE, "step graphs out of phase");
    graph_n_ = n_;
    graph_K_ = K_;
    graph_hcap_ = hcap_;
  }

  void capture_step(StepGraph& g) {
    g.key = (const void*)pos_.p;
    capture_kernels_ = 0;
    cuda_check(cudaStreamBeginCapture(stream_, cudaStreamCaptureModeThreadLocal), "cudaStreamBeginCapture");
    capturing_ = true;
    try {
      issue_contacts();
      if (any_dynamic_)
        launch("body_step", k_body_step, dim3(1), dim3(32), bodies_d_.p, nbodies_, (const Scalars*)d_sc_.p);
      issue_update(cfg_.integration_scheme == SPH_TAKE_PREDICTED ? 1 : 0);
      const int loop = cfg_.pressure_solver == SPH_IISPH || cfg_.pressure_solver == SPH_IISPH_W_OST;
      launch("step_epilogue", k_step_epilogue, dim3(1), dim3(1), d_sc_.p, K_, hcap_, loop);
    } catch (...) {
      capturing_ = false;
      in_loop_body_ = false;
      cudaGraph_t junk = nullptr;
      cudaStreamEndCapture(stream_, &junk);
      if (junk) cudaGraphDestroy(junk);
      cudaGetLastError();
      throw;
    }
    capturing_ = false;
    cuda_check(cudaStreamEndCapture(stream_, &g.graph), "cudaStreamEndCapture");
    cuda_check(cudaGraphInstantiate(&g.exec, g.graph, 0), "cudaGraphInstantiate");
    g.kernels = capture_kernels_;
  }

  // resolve_pressure_globally's loop (iisph.rs:419-550) as a while-node.
  void solve_loop_graph() {
    cudaStreamCaptureStatus st;
    cudaGraph_t graph = nullptr;
    const cudaGraphNode_t* deps = nullptr;
    size_t nd = 0;
    cuda_check(cudaStreamGetCaptureInfo(stream_, &st, nullptr, &graph, &deps, &nd), "cudaStreamGetCaptureInfo");
    cudaGraphConditionalHandle handle;
    cuda_check(cudaGraphConditionalHandleCreate(&handle, graph, 1, cudaGraphCondAssignDefault),
               "cudaGraphConditionalHandleCreate");
    cudaGraphNodeParams np{};
    np.type = cudaGraphNodeTypeConditional;
    np.conditional.handle = handle;
    np.conditional.type = cudaGraphCondTypeWhile;
    np.conditional.size = 1;
    cudaGraphNode_t node;
    cuda_check(cudaGraphAddNode(&node, graph, deps, nd, &np), "cudaGraphAddNode");
    cudaGraph_t body = np.conditional.phGraph_out[0];
    cuda_check(cudaStreamBeginCaptureToGraph(body_stream_, body, nullptr, nullptr, 0, cudaStreamCaptureModeThreadLocal),
               "cudaStreamBeginCaptureToGraph");
    const int limit = P_.iteration_cap > 0 ? P_.iteration_cap : kGraphSweepLimit;
    std::swap(stream_, body_stream_);
    in_loop_body_ = true;
    try {
      iisph_iteration(-1, true);
      launch_dep("solve_loop", k_loop_cond, dim3(1), dim3(1), 0, handle, (const Scalars*)d_sc_.p, limit);
    } catch (...) {
      in_loop_body_ = false;
      std::swap(stream_, body_stream_);
      cudaGraph_t junk = nullptr;
      cudaStreamEndCapture(body_stream_, &junk);
      throw;
    }
    in_loop_body_ = false;
    std::swap(stream_, body_stream_);
    cudaGraph_t captured = nullptr;
    cuda_check(cudaStreamEndCapture(body_stream_, &captured), "cudaStreamEndCapture");
    cuda_check(cudaStreamUpdateCaptureDependencies(stream_, &node, 1, cudaStreamSetCaptureDependencies),
               "cudaStreamUpdateCaptureDependencies");
  }

  // State that a chunk of steps reads from the step before it.
  template <class T>
  void d2d(T* dst, const T* src, size_t n) {
    if (n) cuda_check(cudaMemcpyAsync(dst, src, n * sizeof(T), cudaMemcpyDeviceToDevice, stream_), "D2D");
  }
  void alloc_snapshot() {
    const bool tp = cfg_.integration_scheme == SPH_TAKE_PREDICTED;
    if (snap_pos_.n < n_ || !snap_pos_.p) {
      const size_t c = std::max<size_t>(n_, 1);
      snap_pos_.alloc(c); snap_vel_.alloc(c); snap_acc_.alloc(c); snap_ref_.alloc(c); snap_fid_.alloc(c);
      if (tp) { snap_xint_.alloc(c); snap_vint_.alloc(c); }
    }
    if (!snap_sc_.p) snap_sc_.alloc(1);
    if (nbodies_ && snap_bodies_.n < (size_t)nbodies_) snap_bodies_.alloc((size_t)nbodies_);
  }
  void take_snapshot() {
    const bool tp = cfg_.integration_scheme == SPH_TAKE_PREDICTED;
    d2d(snap_pos_.p, pos_.p, n_); d2d(snap_vel_.p, vel_.p, n_); d2d(snap_acc_.p, acc_.p, n_);
    d2d(snap_ref_.p, ref_.p, n_); d2d(snap_fid_.p, fid_.p, n_);
    if (tp) { d2d(snap_xint_.p, xint_.p, n_); d2d(snap_vint_.p, vint_.p, n_); }
    if (nbodies_) d2d(snap_bodies_.p, bodies_d_.p, (size_t)nbodies_);
    d2d(snap_sc_.p, d_sc_.p, 1);
  }
  void restore_snapshot() {
    const bool tp = cfg_.integration_scheme == SPH_TAKE_PREDICTED;
    d2d(pos_.p, snap_pos_.p, n_); d2d(vel_.p, snap_vel_.p, n_); d2d(acc_.p, snap_acc_.p, n_);
    d2d(ref_.p, snap_ref_.p, n_); d2d(fid_.p, snap_fid_.p, n_);
    if (tp) { d2d(xint_.p, snap_xint_.p, n_); d2d(vint_.p, snap_vint_.p, n_); }
    if (nbodies_) d2d(bodies_d_.p, snap_bodies_.p, (size_t)nbodies_);
    d2d(d_sc_.p, snap_sc_.p, 1);
    sync();
  }
};

// ---- pieces defined out of line ------------------------------------------------
template <class R>
SystemBase* System<R>::clone() const {
  throw Error(SPH_ERR_INVALID, "clone is provided by sph_clone through checkpoint replay");
}

template <class R>
void System<R>::set_rigid_state(int bi, const double* in) {
  if (bi < 0 || bi >= nbodies_) throw Error(SPH_ERR_INVALID, "bad boundary index");
  Body b = fetch(bodies_d_.p + bi, 1)[0];
  if (!b.dynamic) throw Error(SPH_ERR_INVALID, "static boundary has no rigid state");
  std::memcpy(b.com, in, 3 * sizeof(double));
  std::memcpy(b.q, in + 3, 4 * sizeof(double));
  std::memcpy(b.v, in + 7, 3 * sizeof(double));
  std::memcpy(b.L, in + 10, 3 * sizeof(double));
  std::memcpy(b.F, in + 13, 3 * sizeof(double));
  std::memcpy(b.T, in + 16, 3 * sizeof(double));
  double Rm[9];
  host_rot(b.q, Rm);
  host_sandwich(Rm, b.inv_inertia_body, b.inv_inertia_world);
  for (int i = 0; i < 3; ++i)
    b.omega[i] = (b.inv_inertia_world[i * 3] * b.L[0] + b.inv_inertia_world[i * 3 + 1] * b.L[1]) +
                 b.inv_inertia_world[i * 3 + 2] * b.L[2];
  copy_h2d(bodies_d_.p + bi, &b, 1);
  bodies_[bi] = b;
}

// Enumerates sample-boundary neighbors of every particle (count, then fill).
template <class R>
__global__ void k_export_sample_neighbors(const Scalars* __restrict__ sc, const R4<R>* __restrict__ pos,
                                          SampleGrid<R> G, uint32_t* __restrict__ counts,
                                          const uint64_t* __restrict__ offs, uint32_t* __restrict__ out,
                                          StepParams<R> P) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= sc->n_active) return;
  const R4<R> xi = pos[i];
  const int cx = cell_coord((double)xi.x, P.range), cy = cell_coord((double)xi.y, P.range),
            cz = cell_coord((double)xi.z, P.range);
  uint32_t c = 0;
  for (int dz = -1; dz <= 1; ++dz)
    for (int dy = -1; dy <= 1; ++dy)
      for (int dx = -1; dx <= 1; ++dx) {
        const uint32_t k = morton_key(cx + dx, cy + dy, cz + dz, G.mask);
        for (uint32_t s = G.start[k]; s < G.start[k + 1]; ++s) {
          if (!in_range(xi, G.xb[s], P.range, P.range2_lo, P.range2_hi)) continue;
          if (out) out[offs[i] + c] = G.orig[s];
          ++c;
        }
      }
  if (!out) counts[i] = c;
}

template <class R>
int System<R>::boundary_neighbors(int bi, uint64_t* off, uint32_t* idx, size_t cap, size_t* total) {
  if (boundary_kind_ != 1 || bi < 0 || bi >= (int)sample_counts_.size())
    throw Error(SPH_ERR_INVALID, "not a sample boundary");
  const int nb = blocks_for((long long)n_);
  DBuf<uint32_t> counts;
  counts.alloc(std::max<size_t>(n_, 1));
  launch("export", k_export_sample_neighbors<R>, dim3(nb), dim3(kBlock), (const Scalars*)d_sc_.p,
         (const R4<R>*)xv_.p, sample_grid(), counts.p, (const uint64_t*)nullptr, (uint32_t*)nullptr, P_);
  std::vector<uint32_t> hc = fetch(counts.p, n_);
  std::vector<uint64_t> hoff(n_ + 1, 0);
  for (size_t d = 0; d < n_; ++d) hoff[d + 1] = hoff[d] + hc[d];
  DBuf<uint64_t> doff;
  doff.alloc(n_ + 1);
  copy_h2d(doff.p, hoff.data(), n_ + 1);
  DBuf<uint32_t> dout;
  dout.alloc(std::max<uint64_t>(hoff[n_], 1));
  launch("export", k_export_sample_neighbors<R>, dim3(nb), dim3(kBlock), (const Scalars*)d_sc_.p,
         (const R4<R>*)xv_.p, sample_grid(), counts.p, (const uint64_t*)doff.p, dout.p, P_);
  std::vector<uint32_t> all = fetch(dout.p, hoff[n_]);
  std::vector<uint32_t> ref = fetch(ref_.p, n_);
  const size_t lo = sample_offsets_[bi], hi = lo + sample_counts_[bi];
  std::vector<std::vector<uint32_t>> rows(n_);
  for (size_t d = 0; d < n_; ++d)
    for (uint64_t k = hoff[d]; k < hoff[d + 1]; ++k)
      if (all[k] >= lo && all[k] < hi) rows[ref[d]].push_back((uint32_t)(all[k] - lo));
  size_t tot = 0;
  for (auto& r : rows) tot += r.size();
  *total = tot;
  if (!off || !idx || cap < tot) return SPH_ERR_CAPACITY;
  off[0] = 0;
  for (size_t r = 0; r < n_; ++r) {
    std::sort(rows[r].begin(), rows[r].end());
    std::copy(rows[r].begin(), rows[r].end(), idx + off[r]);
    off[r + 1] = off[r] + rows[r].size();
  }
  return SPH_OK;
}

// XOR-prime hash (spatial_hashing.rs:49-71) of the 27 stencil cells of every
// particle; counts particles whose stencil has two cells in one hash bucket,
// the only case where the reference's neighbor lists hold duplicates.
__device__ __forceinline__ unsigned long long ref_hash(int k, int l, int m) {
  auto u = [](int v) -> unsigned long long {
    return v >= 0 ? (unsigned long long)v * 2ull : (unsigned long long)(-(long long)v) * 2ull + 1ull;
  };
  return (u(k) * 73856093ull) ^ (u(l) * 19349663ull) ^ (u(m) * 83492791ull);
}
template <class R>
__global__ void k_hash_collisions(const Scalars* __restrict__ sc, const R4<R>* __restrict__ pos,
                                  unsigned long long* __restrict__ out, double range) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= sc->n_active) return;
  const R4<R> x = pos[i];
  const int cx = cell_coord((double)x.x, range), cy = cell_coord((double)x.y, range),
            cz = cell_coord((double)x.z, range);
  unsigned long long h[27];
  int a = 0;
  for (int dx = -1; dx <= 1; ++dx)
    for (int dy = -1; dy <= 1; ++dy)
      for (int dz = -1; dz <= 1; ++dz) h[a++] = ref_hash(cx + dx, cy + dy, cz + dz);
  for (int p = 0; p < 27; ++p)
    for (int q = p + 1; q < 27; ++q)
      if (h[p] == h[q]) {
        atomicAdd(out, 1ull);
        return;
      }
}

template <class R>
uint64_t System<R>::hash_collisions() {
  DBuf<unsigned long long> d;
  d.alloc(1);
  d.zero(stream_);
  launch("diagnostics", k_hash_collisions<R>, dim3(blocks_for((long long)n_)), dim3(kBlock),
         (const Scalars*)d_sc_.p, (const R4<R>*)xv_.p, d.p, P_.range);
  return fetch(d.p, 1)[0];
}

template <class R>
void System<R>::restore(uint64_t steps, double time, size_t n, const double* x, const double* v,
                        const double* m, const uint32_t* fid, const double* xi, const double* vi) {
  if (!initialized_) throw Error(SPH_ERR_STATE, "initialize before restoring a checkpoint");
  if (n > cap_) throw Error(SPH_ERR_INVALID, "checkpoint holds more particles than the system");
  n_ = n;
  std::vector<R4<R>> hp(n), hv(n), hxi(n), hvi(n);
  std::vector<uint32_t> hr(n), hf(n);
  for (size_t i = 0; i < n; ++i) {
    hp[i] = R4<R>{(R)x[3 * i], (R)x[3 * i + 1], (R)x[3 * i + 2], R(0)};
    hv[i] = R4<R>{(R)v[3 * i], (R)v[3 * i + 1], (R)v[3 * i + 2], (R)m[i]};
    hr[i] = (uint32_t)i;
    hf[i] = fid ? fid[i] : 0u;
    if (xi) hxi[i] = R4<R>{(R)xi[3 * i], (R)xi[3 * i + 1], (R)xi[3 * i + 2], R(0)};
    if (vi) hvi[i] = R4<R>{(R)vi[3 * i], (R)vi[3 * i + 1], (R)vi[3 * i + 2], (R)m[i]};
  }
  copy_h2d(pos_.p, hp.data(), n);
  copy_h2d(vel_.p, hv.data(), n);
  copy_h2d(ref_.p, hr.data(), n);
  copy_h2d(fid_.p, hf.data(), n);
  if (cfg_.integration_scheme == SPH_TAKE_PREDICTED) {
    if (xi) copy_h2d(xint_.p, hxi.data(), n); else xint_.zero(stream_);
    if (vi) copy_h2d(vint_.p, hvi.data(), n); else vint_.zero(stream_);
  }
  acc_.zero(stream_);
  steps_ = steps;
  if (cfg_.cfl_time_step) {
    current_time_ = time;
  }
  Scalars s = *h_sc_;
  s.n = (int)n;
  s.n_active = (int)n;
  s.n_below = 0;
  s.max_speed = 0;
  copy_h2d(d_sc_.p, &s, 1);
  *h_sc_ = s;
  update(2);  // continue_from_checkpoint (sph/mod.rs:362-378)
}

SystemBase* create_system(const sph_config& c) {
  if (c.precision == SPH_F64) return new System<double>(c);
  return new System<float>(c);
}

}  // namespace sph

// ===========================================================================
// C ABI
// ===========================================================================
using sph::Error;
using sph::SystemBase;

struct sph_system {
  std::unique_ptr<SystemBase> impl;
  sph_config cfg;
  // Replay log for sph_clone: the inputs that built the system.
  struct Fluid { std::vector<double> x, v, m; std::vector<uint32_t> fid; } fluid;
  struct SampleB { std::vector<double> x; bool dyn; sph_rigid_init rigid; };
  struct VMB {
    sph_grid_desc sd, vd;
    std::vector<double> sn, vn;
    bool dyn;
    sph_rigid_init rigid;
    bool has_aabb = false;
    double aabb[6] = {0, 0, 0, 0, 0, 0};
  };
  std::vector<int> order;  // 0 sample, 1 vm
  std::vector<SampleB> samples;
  std::vector<VMB> vms;
  bool initialized = false;
};

template <class F>
static int guarded(F&& f) {
  try {
    f();
    return SPH_OK;
  } catch (const Error& e) {
    sph::g_last_error = e.what();
    return e.code;
  } catch (const std::bad_alloc&) {
    sph::g_last_error = "host allocation failed";
    return SPH_ERR_OOM;
  } catch (const std::exception& e) {
    sph::g_last_error = e.what();
    return SPH_ERR_CUDA;
  }
}

static void set_device(const sph_system_t* h) { cudaSetDevice(h->cfg.device); }

extern "C" {

void sph_config_default(sph_config* c) {
  std::memset(c, 0, sizeof *c);
  c->kernel_fn = SPH_CUBIC_BSPLINE_3D;
  c->integration_scheme = SPH_EULER_CROMER;
  c->pressure_solver = SPH_IISPH;
  c->neighbor_search = SPH_SPATIAL_HASHING;
  c->boundary_handling = SPH_VOLUME_MAP_BOUNDARY;
  c->precision = SPH_F32;
  c->cfl_time_step = 0;
  c->gravity_mode = SPH_GRAVITY_UNIFORM;
  c->rest_density_grid_spacing = 0.8;
  c->kernel_support_radius = 1.6;
  c->disable_particles_below = -50.0;
  c->fluid_viscosity = 0.2;
  c->boundary_viscosity = 0.2;
  c->boundary_pressure_acceleration_weighting = 0.7;
  c->boundary_rest_volume_weighting = 1.0;
  c->stiffness = 15000000.0;
  c->target_density_error = 0.05;
  c->relaxation_factor = 0.5;
  c->min_diagonal_element = 1e-10;
  c->time_increment = 0.006;
  c->max_time_increment = 0.01;
  c->cfl_number = 0.4;
  c->max_solver_iterations = 0;
  c->neighbor_capacity = 128;
  c->device = 0;
}

int sph_create(const sph_config* cfg, sph_system_t** out) {
  return guarded([&] {
    if (!cfg || !out) throw Error(SPH_ERR_INVALID, "null argument");
    if (cfg->kernel_fn != SPH_CUBIC_BSPLINE_3D) throw Error(SPH_ERR_INVALID, "unknown kernel function");
    if (cfg->neighbor_search != SPH_SPATIAL_HASHING) throw Error(SPH_ERR_INVALID, "unknown neighbor search");
    if (cfg->integration_scheme < 0 || cfg->integration_scheme > 1)
      throw Error(SPH_ERR_INVALID, "integration scheme not supported by the GPU engine");
    if (cfg->pressure_solver < 0 || cfg->pressure_solver > 3) throw Error(SPH_ERR_INVALID, "unknown pressure solver");
    if (cfg->boundary_handling < 0 || cfg->boundary_handling > 1)
      throw Error(SPH_ERR_INVALID, "unknown boundary handling");
    if (!(cfg->kernel_support_radius > 0) || !(cfg->rest_density_grid_spacing > 0))
      throw Error(SPH_ERR_INVALID, "support radius and spacing must be positive");
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0)
      throw Error(SPH_ERR_CUDA, "no CUDA device available");
    if (cfg->device < 0 || cfg->device >= ndev) throw Error(SPH_ERR_INVALID, "device ordinal out of range");
    auto h = std::make_unique<sph_system>();
    h->cfg = *cfg;
    h->impl.reset(sph::create_system(*cfg));
    *out = h.release();
  });
}

void sph_destroy(sph_system_t* h) {
  if (!h) return;
  set_device(h);
  delete h;
}

int sph_upload_fluid(sph_system_t* h, size_t n, const double* x, const double* v, const double* m,
                     const uint32_t* fid) {
  return guarded([&] {
    if (!h || (n && (!x || !m))) throw Error(SPH_ERR_INVALID, "null argument");
    if (h->initialized) throw Error(SPH_ERR_STATE, "fluid is uploaded before initialize");
    set_device(h);
    h->impl->upload_fluid(n, x, v, m, fid);
    h->fluid.x.assign(x, x + 3 * n);
    h->fluid.v = v ? std::vector<double>(v, v + 3 * n) : std::vector<double>(3 * n, 0.0);
    h->fluid.m.assign(m, m + n);
    h->fluid.fid = fid ? std::vector<uint32_t>(fid, fid + n) : std::vector<uint32_t>(n, 0u);
  });
}

int sph_add_sample_boundary(sph_system_t* h, size_t nb, const double* x, const sph_rigid_init* rigid,
                            int* bi) {
  return guarded([&] {
    if (!h || (nb && !x)) throw Error(SPH_ERR_INVALID, "null argument");
    if (h->initialized) throw Error(SPH_ERR_STATE, "boundaries are added before initialize");
    set_device(h);
    const int idx = h->impl->add_sample_boundary(nb, x, rigid);
    if (bi) *bi = idx;
    sph_system::SampleB s;
    s.x.assign(x, x + 3 * nb);
    s.dyn = rigid != nullptr;
    if (rigid) s.rigid = *rigid;
    h->samples.push_back(std::move(s));
    h->order.push_back(0);
  });
}

int sph_add_volume_map_boundary(sph_system_t* h, const sph_grid_desc* sdf, const double* sn,
                                const sph_grid_desc* vm, const double* vn, const sph_rigid_init* rigid,
                                int* bi) {
  return guarded([&] {
    if (!h || !sdf || !sn || !vm || !vn) throw Error(SPH_ERR_INVALID, "null argument");
    if (h->initialized) throw Error(SPH_ERR_STATE, "boundaries are added before initialize");
    set_device(h);
    const int idx = h->impl->add_volume_map(*sdf, sn, *vm, vn, rigid);
    if (bi) *bi = idx;
    sph_system::VMB b;
    b.sd = *sdf;
    b.vd = *vm;
    auto cnt = [](const sph_grid_desc& g) {
      return (size_t)(3 * g.n[0] + 1) * (size_t)(3 * g.n[1] + 1) * (size_t)(3 * g.n[2] + 1);
    };
    b.sn.assign(sn, sn + cnt(*sdf));
    b.vn.assign(vn, vn + cnt(*vm));
    b.dyn = rigid != nullptr;
    if (rigid) b.rigid = *rigid;
    h->vms.push_back(std::move(b));
    h->order.push_back(1);
  });
}

int sph_set_volume_map_aabb(sph_system_t* h, int bi, const double* center, const double* half_extents) {
  return guarded([&] {
    if (!h || !center || !half_extents) throw Error(SPH_ERR_INVALID, "null argument");
    if (h->initialized) throw Error(SPH_ERR_STATE, "bounding boxes are set before initialize");
    set_device(h);
    h->impl->set_volume_map_aabb(bi, center, half_extents);
    // the replay log of sph_clone: boundary bi is the bi-th volume map
    int k = -1;
    for (size_t j = 0, seen = 0; j < h->order.size(); ++j)
      if (h->order[j] == 1) {
        if ((int)j == bi) k = (int)seen;
        ++seen;
      }
    if (k >= 0) {
      h->vms[(size_t)k].has_aabb = true;
      for (int d = 0; d < 3; ++d) {
        h->vms[(size_t)k].aabb[d] = center[d];
        h->vms[(size_t)k].aabb[3 + d] = half_extents[d];
      }
    }
  });
}

int sph_get_contact_stats(sph_system_t* h, uint32_t* out4) {
  return guarded([&] {
    if (!h || !out4) throw Error(SPH_ERR_INVALID, "null argument");
    if (!h->initialized) throw Error(SPH_ERR_STATE, "initialize first");
    set_device(h);
    h->impl->contact_stats(out4);
  });
}

int sph_set_contact_sweeps(sph_system_t* h, uint32_t fixed_sweeps) {
  return guarded([&] {
    if (!h) throw Error(SPH_ERR_INVALID, "null argument");
    set_device(h);
    h->impl->set_contact_sweeps(fixed_sweeps);
  });
}

int sph_initialize(sph_system_t* h) {
  return guarded([&] {
    if (!h) throw Error(SPH_ERR_INVALID, "null argument");
    if (h->initialized) throw Error(SPH_ERR_STATE, "already initialized");
    set_device(h);
    h->impl->initialize();
    h->initialized = true;
  });
}

int sph_step(sph_system_t* h, uint32_t n) {
  int st = SPH_OK;
  int rc = guarded([&] {
    if (!h) throw Error(SPH_ERR_INVALID, "null argument");
    set_device(h);
    st = h->impl->step(n);
  });
  return rc != SPH_OK ? rc : st;
}

int sph_step_host(sph_system_t* h, uint32_t n, const double* xi, const double* vi, double* xo, double* vo) {
  int st = SPH_OK;
  int rc = guarded([&] {
    if (!h) throw Error(SPH_ERR_INVALID, "null argument");
    set_device(h);
    st = h->impl->step_host(n, xi, vi, xo, vo);
  });
  return rc != SPH_OK ? rc : st;
}
int sph_get_step_stats(const sph_system_t* h, sph_step_stats* out) {
  return guarded([&] {
    if (!h || !out) throw Error(SPH_ERR_INVALID, "null argument");
    h->impl->step_stats(out);
  });
}
int sph_get_stream(const sph_system_t* h, void** stream) {
  return guarded([&] {
    if (!h || !stream) throw Error(SPH_ERR_INVALID, "null argument");
    *stream = h->impl->stream();
  });
}
int sph_time(const sph_system_t* h, double* out) {
  return guarded([&] {
    if (!h || !out) throw Error(SPH_ERR_INVALID, "null argument");
    *out = h->impl->time();
  });
}
int sph_time_steps_propagated(const sph_system_t* h, uint64_t* out) {
  return guarded([&] {
    if (!h || !out) throw Error(SPH_ERR_INVALID, "null argument");
    *out = h->impl->steps();
  });
}
int sph_take_measurement(sph_system_t* h, sph_measurement* out) {
  return guarded([&] {
    if (!h || !out) throw Error(SPH_ERR_INVALID, "null argument");
    if (!h->initialized) throw Error(SPH_ERR_STATE, "initialize first");
    set_device(h);
    h->impl->measurement(out);
  });
}
int sph_num_particles(const sph_system_t* h, size_t* out) {
  return guarded([&] {
    if (!h || !out) throw Error(SPH_ERR_INVALID, "null argument");
    *out = h->impl->num_particles();
  });
}
int sph_get_fluid_ids(sph_system_t* h, uint32_t* out) {
  return guarded([&] {
    if (!h || !out) throw Error(SPH_ERR_INVALID, "null argument");
    set_device(h);
    h->impl->fluid_ids(out);
  });
}
int sph_get_fluid_pos(sph_system_t* h, float* out) {
  return guarded([&] {
    if (!h || !out) throw Error(SPH_ERR_INVALID, "null argument");
    set_device(h);
    h->impl->fluid_pos(out);
  });
}
int sph_get_quantity_of_fluid_samples(sph_system_t* h, int q, float* out) {
  return guarded([&] {
    if (!h || !out) throw Error(SPH_ERR_INVALID, "null argument");
    if (!h->initialized) throw Error(SPH_ERR_STATE, "initialize first");
    set_device(h);
    h->impl->quantity(q, out);
  });
}
int sph_get_quantity_at_positions(sph_system_t* h, int q, size_t n, const float* positions, float* out) {
  return guarded([&] {
    if (!h || (n && (!positions || !out))) throw Error(SPH_ERR_INVALID, "null argument");
    if (!h->initialized) throw Error(SPH_ERR_STATE, "initialize first");
    set_device(h);
    h->impl->quantity_at(q, n, positions, out);
  });
}
int sph_download(sph_system_t* h, int field, double* out) {
  return guarded([&] {
    if (!h || !out) throw Error(SPH_ERR_INVALID, "null argument");
    if (!h->initialized) throw Error(SPH_ERR_STATE, "initialize first");
    set_device(h);
    h->impl->download(field, out);
  });
}
int sph_get_fluid_neighbors(sph_system_t* h, uint64_t* off, uint32_t* idx, size_t cap, size_t* total) {
  int st = SPH_OK;
  int rc = guarded([&] {
    if (!h || !total) throw Error(SPH_ERR_INVALID, "null argument");
    if (!h->initialized) throw Error(SPH_ERR_STATE, "initialize first");
    set_device(h);
    st = h->impl->fluid_neighbors(off, idx, cap, total);
  });
  return rc != SPH_OK ? rc : st;
}
int sph_get_boundary_neighbors(sph_system_t* h, int bi, uint64_t* off, uint32_t* idx, size_t cap,
                               size_t* total) {
  int st = SPH_OK;
  int rc = guarded([&] {
    if (!h || !total) throw Error(SPH_ERR_INVALID, "null argument");
    if (!h->initialized) throw Error(SPH_ERR_STATE, "initialize first");
    set_device(h);
    st = h->impl->boundary_neighbors(bi, off, idx, cap, total);
  });
  return rc != SPH_OK ? rc : st;
}
int sph_get_boundary_volumes(sph_system_t* h, int bi, double* out) {
  return guarded([&] {
    if (!h || !out) throw Error(SPH_ERR_INVALID, "null argument");
    if (!h->initialized) throw Error(SPH_ERR_STATE, "initialize first");
    set_device(h);
    h->impl->boundary_volumes(bi, out);
  });
}
int sph_get_boundary_positions(sph_system_t* h, int bi, double* out) {
  return guarded([&] {
    if (!h || !out) throw Error(SPH_ERR_INVALID, "null argument");
    if (!h->initialized) throw Error(SPH_ERR_STATE, "initialize first");
    set_device(h);
    h->impl->boundary_positions(bi, out);
  });
}
int sph_get_volume_map_samples(sph_system_t* h, int bi, uint8_t* has, double* xb, double* vb, double* vol) {
  return guarded([&] {
    if (!h || !has || !xb || !vb || !vol) throw Error(SPH_ERR_INVALID, "null argument");
    if (!h->initialized) throw Error(SPH_ERR_STATE, "initialize first");
    set_device(h);
    h->impl->vm_samples(bi, has, xb, vb, vol);
  });
}
int sph_get_rigid_state(sph_system_t* h, int bi, double* out) {
  return guarded([&] {
    if (!h || !out) throw Error(SPH_ERR_INVALID, "null argument");
    if (!h->initialized) throw Error(SPH_ERR_STATE, "initialize first");
    set_device(h);
    h->impl->rigid_state(bi, out);
  });
}
int sph_set_rigid_state(sph_system_t* h, int bi, const double* in) {
  return guarded([&] {
    if (!h || !in) throw Error(SPH_ERR_INVALID, "null argument");
    if (!h->initialized) throw Error(SPH_ERR_STATE, "initialize first");
    set_device(h);
    h->impl->set_rigid_state(bi, in);
  });
}
int sph_hash_collisions(sph_system_t* h, uint64_t* out) {
  return guarded([&] {
    if (!h || !out) throw Error(SPH_ERR_INVALID, "null argument");
    if (!h->initialized) throw Error(SPH_ERR_STATE, "initialize first");
    set_device(h);
    *out = h->impl->hash_collisions();
  });
}
int sph_continue_from_checkpoint(sph_system_t* h, uint64_t steps, double t, size_t n, const double* x,
                                 const double* v, const double* m, const uint32_t* fid, const double* xi,
                                 const double* vi) {
  return guarded([&] {
    if (!h || (n && (!x || !v || !m))) throw Error(SPH_ERR_INVALID, "null argument");
    set_device(h);
    h->impl->restore(steps, t, n, x, v, m, fid, xi, vi);
  });
}

// SystemCheckpoint::from_sph_system (sph/mod.rs:849-856): step counter,
// time, the fluid in reference order (fluid.rs:351-371, integrator slots
// included) and one entry per boundary (Some for dynamic ones).
int sph_get_checkpoint(sph_system_t* h, sph_checkpoint_t** out) {
  return guarded([&] {
    if (!h || !out) throw Error(SPH_ERR_INVALID, "null argument");
    if (!h->initialized) throw Error(SPH_ERR_STATE, "initialize first");
    set_device(h);
    SystemBase* s = h->impl.get();
    const size_t n = s->num_particles();
    sph::fmt::Checkpoint c;
    c.time_steps_propagated = s->steps();
    c.current_time = s->time();
    c.position.resize(3 * n);
    c.velocity.resize(3 * n);
    c.mass.resize(n);
    c.fluid_id.resize(n);
    s->download(SPH_FIELD_POSITION, c.position.data());
    s->download(SPH_FIELD_VELOCITY, c.velocity.data());
    s->download(SPH_FIELD_MASS, c.mass.data());
    s->fluid_ids(c.fluid_id.data());
    if (h->cfg.integration_scheme == SPH_TAKE_PREDICTED) {  // take_predicted.rs:9-10: one slot each
      c.integrator_position.emplace_back(3 * n);
      c.integrator_velocity.emplace_back(3 * n);
      s->download(SPH_FIELD_INTEGRATOR_POSITION, c.integrator_position[0].data());
      s->download(SPH_FIELD_INTEGRATOR_VELOCITY, c.integrator_velocity[0].data());
    }
    size_t si = 0, vi = 0;
    for (size_t b = 0; b < h->order.size(); ++b) {
      const bool dyn = h->order[b] == 0 ? h->samples[si++].dyn : h->vms[vi++].dyn;
      sph::fmt::RigidState r;
      if (dyn) {
        s->rigid_state((int)b, r.s.data());
        r.dynamic = true;
      }
      c.boundaries.push_back(r);
    }
    *out = sph::fmt::new_checkpoint(std::move(c));
  });
}

// SPHSystem::continue_from_checkpoint (sph/mod.rs:362-378). As in the
// reference, the integrator slots start from zero (Fluid::resize_slots,
// fluid.rs:113-129, replaces them) and are rewritten by the update; the
// boundary entries are applied only when their count matches the system's
// boundaries, each only where both sides are dynamic
// (static_sample_boundary.rs:263-277, :561-572).
int sph_restore_checkpoint(sph_system_t* h, const sph_checkpoint_t* ck) {
  return guarded([&] {
    if (!h || !ck) throw Error(SPH_ERR_INVALID, "null argument");
    if (!h->initialized) throw Error(SPH_ERR_STATE, "initialize first");
    const sph::fmt::Checkpoint& c = ck->c;
    c.check();
    set_device(h);
    if (c.boundaries.size() == h->order.size()) {
      size_t si = 0, vi = 0;
      for (size_t b = 0; b < h->order.size(); ++b) {
        const bool dyn = h->order[b] == 0 ? h->samples[si++].dyn : h->vms[vi++].dyn;
        if (dyn && c.boundaries[b].dynamic) h->impl->set_rigid_state((int)b, c.boundaries[b].s.data());
      }
    }
    const size_t n = c.n();
    h->impl->restore(c.time_steps_propagated, c.current_time, n, c.position.data(), c.velocity.data(),
                     c.mass.data(), c.fluid_id.data(), nullptr, nullptr);
  });
}

// TimeStepInfo::from_system (render_info.rs:83-92, :110-158, :179-194) and
// the boundary's Samples visualization (static_sample_boundary.rs:221-249;
// a volume-map system has no samples and reports an empty, uniformly
// colored set, volume_map_boundary.rs:1484-1490), encoded as bincode.
int sph_encode_time_step_info(sph_system_t* h, const sph_frame_selector* sel, sph_bytes_t** out) {
  return guarded([&] {
    if (!h || !sel || !out) throw Error(SPH_ERR_INVALID, "null argument");
    if (!h->initialized) throw Error(SPH_ERR_STATE, "initialize first");
    set_device(h);
    SystemBase* s = h->impl.get();
    sph_frame_view f;
    std::memset(&f, 0, sizeof f);
    f.time_step_number = s->steps();
    s->measurement(&f.measurement);
    f.fluid = sel->fluid;
    f.fluid_coloring = sel->fluid_coloring;
    f.quantity = sel->quantity;
    std::vector<float> pos, data;
    std::vector<uint32_t> ids;
    std::vector<sph_sensor_plane> planes;
    std::vector<std::vector<float>> plane_data;
    sph_meshes meshes;
    if (sel->fluid == SPH_FLUID_TRIANGLE_MESH) {  // render_info.rs:128-133
      s->reconstruct_surfaces(meshes.m);
      f.meshes = &meshes;
      const size_t n = s->num_particles();
      std::vector<uint32_t> all(n);
      if (n) s->fluid_ids(all.data());
      for (uint32_t id : all) f.max_fluid_id = std::max(f.max_fluid_id, id);
    } else if (sel->fluid == SPH_FLUID_SAMPLES) {
      const size_t n = s->num_particles();
      pos.resize(3 * n);
      s->fluid_pos(pos.data());
      f.n = n;
      f.fluid_positions = pos.data();
      if (sel->fluid_coloring == SPH_COLORING_ID) {
        ids.resize(n);
        s->fluid_ids(ids.data());
        f.fluid_ids = ids.data();
      } else if (sel->fluid_coloring == SPH_COLORING_QUANTITY) {
        data.resize(n);
        s->quantity(sel->quantity, data.data());
        f.fluid_data = data.data();
      }
    } else if (sel->fluid == SPH_FLUID_SENSOR_PLANE) {
      if (sel->num_planes && !sel->planes) throw Error(SPH_ERR_INVALID, "null planes");
      planes.resize(sel->num_planes);
      plane_data.resize(sel->num_planes);
      for (size_t k = 0; k < sel->num_planes; ++k) {
        const sph_sensor_plane& p = sel->planes[k];
        const size_t np = p.rows * p.cols;
        if (np && !p.positions) throw Error(SPH_ERR_INVALID, "null plane positions");
        plane_data[k].resize(np);
        s->quantity_at(sel->quantity, np, p.positions, plane_data[k].data());
        planes[k] = sph_sensor_plane{p.positions, plane_data[k].data(), p.rows, p.cols};
      }
      f.num_planes = planes.size();
      f.planes = planes.data();
    }
    std::vector<float> bpos, poses;
    std::vector<uint32_t> bids;
    f.boundary_coloring = SPH_COLORING_UNIFORM;
    f.boundary_visualization = sel->boundary_visualization;
    if (sel->boundary_visualization == SPH_BOUNDARY_TRIANGLE_MESH) {
      // get_visualization (static_sample_boundary.rs:194-219, volume_map_boundary.rs:1459-1483):
      // each boundary's render mesh with its pose; BoundaryId lists the mesh id per sample for
      // sample boundaries and per boundary for volume maps
      const size_t nb = h->order.size();
      if (nb && !sel->render_meshes) throw Error(SPH_ERR_INVALID, "render meshes are needed for TriangleMesh");
      f.boundary_mesh_coloring = sel->boundary_mesh_coloring;
      f.num_boundary_meshes = nb;
      f.boundary_meshes = sel->render_meshes;
      poses.assign(7 * nb, 0.0f);
      size_t si = 0, vi = 0;
      for (size_t b = 0; b < nb; ++b) {
        const bool is_sample = h->order[b] == 0;
        const bool dyn = is_sample ? h->samples[si].dyn : h->vms[vi].dyn;
        const uint32_t id = sel->render_mesh_ids ? sel->render_mesh_ids[b] : (uint32_t)b;
        if (is_sample)
          bids.insert(bids.end(), h->samples[si].x.size() / 3, id);
        else
          bids.push_back(id);
        is_sample ? ++si : ++vi;
        float* P = &poses[7 * b];
        P[6] = 1.0f;  // RenderPose::IDENTITY
        if (dyn) {    // RenderPose::from(pose): translation, rotation (i, j, k, w)
          double st[19];
          s->rigid_state((int)b, st);
          P[0] = (float)st[0]; P[1] = (float)st[1]; P[2] = (float)st[2];
          P[3] = (float)st[4]; P[4] = (float)st[5]; P[5] = (float)st[6]; P[6] = (float)st[3];
        }
      }
      f.boundary_poses = poses.data();
      f.num_mesh_ids = bids.size();
      f.mesh_ids = bids.data();
    } else if (h->cfg.boundary_handling == SPH_STATIC_SAMPLE_BOUNDARY) {
      f.boundary_coloring = sel->boundary_coloring;
      size_t si = 0;
      for (size_t b = 0; b < h->order.size(); ++b) {
        if (h->order[b] != 0) continue;
        const size_t nb = h->samples[si++].x.size() / 3;
        std::vector<double> x(3 * nb);
        if (nb) s->boundary_positions((int)b, x.data());
        for (double v : x) bpos.push_back((float)v);
        bids.insert(bids.end(), nb, sel->render_mesh_ids ? sel->render_mesh_ids[b] : (uint32_t)b);
      }
      f.num_boundary_samples = bpos.size() / 3;
      f.boundary_positions = bpos.data();
      f.boundary_ids = bids.data();
    }
    *out = sph::fmt::new_bytes(sph::fmt::time_step_info_to_bincode(f));
  });
}

int sph_reconstruct_surfaces(sph_system_t* h, sph_meshes_t** out) {
  return guarded([&] {
    if (!h || !out) throw Error(SPH_ERR_INVALID, "null argument");
    if (!h->initialized) throw Error(SPH_ERR_STATE, "initialize first");
    set_device(h);
    auto m = std::make_unique<sph_meshes>();
    h->impl->reconstruct_surfaces(m->m);
    *out = m.release();
  });
}
int sph_meshes_count(const sph_meshes_t* m, size_t* out) {
  return guarded([&] {
    if (!m || !out) throw Error(SPH_ERR_INVALID, "null argument");
    *out = m->m.size();
  });
}
int sph_meshes_get(const sph_meshes_t* m, size_t k, uint32_t* fluid_id, size_t* nv, const double** vertices,
                   size_t* ni, const uint32_t** indices) {
  return guarded([&] {
    if (!m || !fluid_id || !nv || !vertices || !ni || !indices) throw Error(SPH_ERR_INVALID, "null argument");
    if (k >= m->m.size()) throw Error(SPH_ERR_INVALID, "mesh index out of range");
    const sph::SurfaceMeshOut& s = m->m[k];
    *fluid_id = s.fluid_id;
    *nv = s.vertices.size() / 6;
    *vertices = s.vertices.data();
    *ni = s.indices.size();
    *indices = s.indices.data();
  });
}
void sph_meshes_free(sph_meshes_t* m) { delete m; }

// Deep copy: rebuild from the recorded inputs, then restore the source's
// current dynamic state (fluid, rigid bodies, step counter and time).
int sph_clone(const sph_system_t* src, sph_system_t** out) {
  return guarded([&] {
    if (!src || !out) throw Error(SPH_ERR_INVALID, "null argument");
    if (!src->initialized) throw Error(SPH_ERR_STATE, "clone an initialized system");
    set_device(src);
    sph_system_t* h = nullptr;
    int rc = sph_create(&src->cfg, &h);
    if (rc) throw Error(rc, sph_last_error());
    std::unique_ptr<sph_system_t, void (*)(sph_system_t*)> guard(h, sph_destroy);
    const size_t n0 = src->fluid.m.size();
    rc = sph_upload_fluid(h, n0, src->fluid.x.data(), src->fluid.v.data(), src->fluid.m.data(),
                          src->fluid.fid.data());
    if (rc) throw Error(rc, sph_last_error());
    size_t si = 0, vi = 0;
    for (int kind : src->order) {
      if (kind == 0) {
        const auto& s = src->samples[si++];
        rc = sph_add_sample_boundary(h, s.x.size() / 3, s.x.data(), s.dyn ? &s.rigid : nullptr, nullptr);
      } else {
        const auto& b = src->vms[vi++];
        int bi = -1;
        rc = sph_add_volume_map_boundary(h, &b.sd, b.sn.data(), &b.vd, b.vn.data(), b.dyn ? &b.rigid : nullptr,
                                         &bi);
        if (rc == SPH_OK && b.has_aabb) rc = sph_set_volume_map_aabb(h, bi, b.aabb, b.aabb + 3);
      }
      if (rc) throw Error(rc, sph_last_error());
    }
    rc = sph_initialize(h);
    if (rc) throw Error(rc, sph_last_error());
    SystemBase* s = const_cast<SystemBase*>(src->impl.get());
    const size_t n = s->num_particles();
    std::vector<double> x(3 * n), v(3 * n), m(n), fidd(n), xi, vvi;
    s->download(SPH_FIELD_POSITION, x.data());
    s->download(SPH_FIELD_VELOCITY, v.data());
    s->download(SPH_FIELD_MASS, m.data());
    s->download(SPH_FIELD_FLUID_ID, fidd.data());
    std::vector<uint32_t> fid(n);
    for (size_t i = 0; i < n; ++i) fid[i] = (uint32_t)fidd[i];
    if (src->cfg.integration_scheme == SPH_TAKE_PREDICTED) {
      xi.resize(3 * n);
      vvi.resize(3 * n);
      s->download(SPH_FIELD_INTEGRATOR_POSITION, xi.data());
      s->download(SPH_FIELD_INTEGRATOR_VELOCITY, vvi.data());
    }
    for (int b = 0; b < (int)src->order.size(); ++b) {
      double st[19];
      bool dyn = false;
      try {
        s->rigid_state(b, st);
        dyn = true;
      } catch (const Error&) {
      }
      if (dyn) h->impl->set_rigid_state(b, st);
    }
    h->impl->restore(s->steps(), s->time(), n, x.data(), v.data(), m.data(), fid.data(),
                     xi.empty() ? nullptr : xi.data(), vvi.empty() ? nullptr : vvi.data());
    sph_tuning t;
    s->get_tuning(&t);
    h->impl->set_tuning(t);
    h->impl->set_contact_sweeps(s->contact_sweeps());
    h->impl->set_step_graphs(s->step_graph_chunk());
    *out = guard.release();
  });
}

int sph_launch_count(const sph_system_t* h, uint64_t* out) {
  return guarded([&] {
    if (!h || !out) throw Error(SPH_ERR_INVALID, "null argument");
    *out = h->impl->launches();
  });
}
int sph_get_tuning(const sph_system_t* h, sph_tuning* out) {
  return guarded([&] {
    if (!h || !out) throw Error(SPH_ERR_INVALID, "null argument");
    h->impl->get_tuning(out);
  });
}
int sph_set_tuning(sph_system_t* h, const sph_tuning* tuning) {
  return guarded([&] {
    if (!h || !tuning) throw Error(SPH_ERR_INVALID, "null argument");
    set_device(h);
    h->impl->set_tuning(*tuning);
  });
}
int sph_autotune(sph_system_t* h, uint32_t steps, sph_tuning* best, double* best_ms_per_step) {
  return guarded([&] {
    if (!h || !best) throw Error(SPH_ERR_INVALID, "null argument");
    if (!h->initialized) throw Error(SPH_ERR_STATE, "initialize before tuning");
    if (steps == 0) throw Error(SPH_ERR_INVALID, "tuning needs at least one timed step");
    set_device(h);
    const bool f32 = h->cfg.precision == SPH_F32;
    sph_tuning cur{};
    h->impl->get_tuning(&cur);
    std::vector<sph_tuning> cand;
    for (uint32_t nb : {4u, 8u})
      for (uint32_t hs : f32 ? std::vector<uint32_t>{1024, 1536, 2048} : std::vector<uint32_t>{512, 1024, 1536})
        cand.push_back(sph_tuning{nb, hs, cur.sweep_stage});
    cudaEvent_t e0 = nullptr, e1 = nullptr;
    sph::cuda_check(cudaEventCreate(&e0), "cudaEventCreate");
    std::unique_ptr<CUevent_st, cudaError_t (*)(cudaEvent_t)> g0(e0, cudaEventDestroy);
    sph::cuda_check(cudaEventCreate(&e1), "cudaEventCreate");
    std::unique_ptr<CUevent_st, cudaError_t (*)(cudaEvent_t)> g1(e1, cudaEventDestroy);
    auto advance = [](sph_system_t* k, uint32_t n) {
      const int rc = sph_step(k, n);
      if (rc != SPH_OK && rc != SPH_NOT_CONVERGED) throw Error(rc, sph_last_error());
    };
    double best_t = std::numeric_limits<double>::infinity();
    sph_tuning pick = cur;
    auto time_candidate = [&](const sph_tuning& c) {
      sph_system_t* k = nullptr;
      int rc = sph_clone(h, &k);
      if (rc) throw Error(rc, sph_last_error());
      std::unique_ptr<sph_system_t, void (*)(sph_system_t*)> guard(k, sph_destroy);
      k->impl->set_tuning(c);
      advance(k, 1);  // warm-up: graph capture and list capacity
      cudaStream_t st = (cudaStream_t)k->impl->stream();
      sph::cuda_check(cudaEventRecord(e0, st), "cudaEventRecord");
      advance(k, steps);
      sph::cuda_check(cudaEventRecord(e1, st), "cudaEventRecord");
      sph::cuda_check(cudaEventSynchronize(e1), "cudaEventSynchronize");
      float ms = 0.f;
      sph::cuda_check(cudaEventElapsedTime(&ms, e0, e1), "cudaEventElapsedTime");
      const double per = (double)ms / (double)steps;
      if (per < best_t) {
        best_t = per;
        pick = c;
      }
    };
    for (const sph_tuning& c : cand) time_candidate(c);
    // then the sweep passes' staging capacity, with the best of the above
    const sph_tuning base = pick;
    for (uint32_t ss : f32 ? std::vector<uint32_t>{1536, 1792, 2048} : std::vector<uint32_t>{1024, 1536})
      if (ss != base.sweep_stage) time_candidate(sph_tuning{base.gather_batch, base.halo_stage, ss});
    h->impl->set_tuning(pick);
    *best = pick;
    if (best_ms_per_step) *best_ms_per_step = best_t;
  });
}
int sph_set_step_graphs(sph_system_t* h, uint32_t chunk_steps) {
  return guarded([&] {
    if (!h) throw Error(SPH_ERR_INVALID, "null argument");
    set_device(h);
    h->impl->set_step_graphs(chunk_steps);
  });
}
int sph_graph_replays(const sph_system_t* h, uint64_t* out) {
  return guarded([&] {
    if (!h || !out) throw Error(SPH_ERR_INVALID, "null argument");
    *out = h->impl->graph_replays();
  });
}
int sph_set_profiling(sph_system_t* h, int enabled) {
  return guarded([&] {
    if (!h) throw Error(SPH_ERR_INVALID, "null argument");
    h->impl->set_profiling(enabled != 0);
  });
}
int sph_kernel_time(sph_system_t* h, const char* kernel, double* ms, uint64_t* launches) {
  return guarded([&] {
    if (!h || !kernel || !ms || !launches) throw Error(SPH_ERR_INVALID, "null argument");
    set_device(h);
    if (!h->impl->kernel_time(kernel, ms, launches)) throw Error(SPH_ERR_INVALID, "no timing for that kernel");
  });
}
int sph_device_bytes(const sph_system_t* h, size_t* out) {
  return guarded([&] {
    if (!h || !out) throw Error(SPH_ERR_INVALID, "null argument");
    *out = h->impl->device_bytes();
  });
}

const char* sph_last_error(void) { return sph::g_last_error.c_str(); }

}  // extern "C"

// ---- volume-map field construction ----------------------------------------------
static void mesh_aabb(const double* v, size_t nv, double mn[3], double mx[3]) {
  for (int d = 0; d < 3; ++d) { mn[d] = INFINITY; mx[d] = -INFINITY; }
  for (size_t i = 0; i < nv; ++i)
    for (int d = 0; d < 3; ++d) {
      mn[d] = std::min(mn[d], v[3 * i + d]);
      mx[d] = std::max(mx[d], v[3 * i + d]);
    }
}

extern "C" int sph_volume_map_grids(const double* verts, size_t nv, double dx, double r, sph_grid_desc* sg,
                         sph_grid_desc* vg) {
  return guarded([&] {
    if (!verts || nv == 0 || !sg || !vg || !(dx > 0) || !(r > 0)) throw Error(SPH_ERR_INVALID, "invalid argument");
    double mn[3], mx[3];
    mesh_aabb(verts, nv, mn, mx);
    const double pads[2] = {3.1 * r, 2.0 * r + dx / 6.0};
    sph_grid_desc* gs[2] = {sg, vg};
    for (int w = 0; w < 2; ++w) {
      for (int d = 0; d < 3; ++d) {
        gs[w]->x_min[d] = mn[d] - pads[w];
        gs[w]->x_max[d] = mx[d] + pads[w];
        gs[w]->n[d] = (int64_t)std::llround((gs[w]->x_max[d] - gs[w]->x_min[d]) / dx);
        if (gs[w]->n[d] < 1) throw Error(SPH_ERR_INVALID, "grid has no cells");
      }
      gs[w]->dx = dx;
    }
  });
}

static sph::LatticeDesc lattice_of(const sph_grid_desc& g) {
  sph::LatticeDesc L;
  for (int d = 0; d < 3; ++d) {
    L.xmin[d] = g.x_min[d];
    L.n[d] = g.n[d];
  }
  L.dx = g.dx;
  L.NX = 3 * g.n[0] + 1;
  L.NY = 3 * g.n[1] + 1;
  L.NZ = 3 * g.n[2] + 1;
  return L;
}

template <class T>
static T* dev_upload(const T* h, size_t n) {
  T* d = nullptr;
  sph::cuda_check(cudaMalloc((void**)&d, std::max<size_t>(n, 1) * sizeof(T)), "cudaMalloc");
  if (n) sph::cuda_check(cudaMemcpy(d, h, n * sizeof(T), cudaMemcpyHostToDevice), "cudaMemcpy");
  return d;
}

static void prune_and_download(const sph::LatticeDesc& L, double* raw, int has_lo, double lo, int has_hi,
                               double hi, double* out) {
  const long long total = L.NX * L.NY * L.NZ;
  const long long ncell = L.n[0] * L.n[1] * L.n[2];
  unsigned char* keep = nullptr;
  double* fin = nullptr;
  sph::cuda_check(cudaMalloc((void**)&keep, total), "cudaMalloc");
  sph::cuda_check(cudaMalloc((void**)&fin, total * sizeof(double)), "cudaMalloc");
  cudaMemset(keep, 0, total);
  sph::k_prune_cells<<<(unsigned)((ncell + 255) / 256), 256>>>(L, raw, has_lo, lo, has_hi, hi, keep);
  sph::k_apply_keep<<<(unsigned)((total + 255) / 256), 256>>>(total, raw, keep, fin);
  sph::cuda_check(cudaGetLastError(), "prune");
  sph::cuda_check(cudaMemcpy(out, fin, total * sizeof(double), cudaMemcpyDeviceToHost), "cudaMemcpy");
  cudaFree(keep);
  cudaFree(fin);
}

extern "C" {

int sph_build_sdf_field(const double* verts, size_t nv, const uint32_t* faces, size_t nf, const sph_grid_desc* g,
                        double r, double* out, int device) {
  return guarded([&] {
    if (!verts || !faces || !g || !out || nf == 0) throw Error(SPH_ERR_INVALID, "invalid argument");
    sph::cuda_check(cudaSetDevice(device), "cudaSetDevice");
    sph::upload_serendipity_tables();
    // per-triangle geometry and pseudo-normals
    auto V = [&](uint32_t i, int d) { return verts[3 * (size_t)i + d]; };
    std::vector<double> tri(9 * nf), fn(3 * nf), en(9 * nf, 0.0), vn(9 * nf, 0.0);
    for (size_t t = 0; t < nf; ++t) {
      for (int k = 0; k < 3; ++k)
        for (int d = 0; d < 3; ++d) {
          if (faces[3 * t + k] >= nv) throw Error(SPH_ERR_INVALID, "face index out of range");
          tri[9 * t + 3 * k + d] = V(faces[3 * t + k], d);
        }
      const double* a = &tri[9 * t];
      const double e1[3] = {a[3] - a[0], a[4] - a[1], a[5] - a[2]}, e2[3] = {a[6] - a[0], a[7] - a[1], a[8] - a[2]};
      const double n[3] = {e1[1] * e2[2] - e1[2] * e2[1], e1[2] * e2[0] - e1[0] * e2[2], e1[0] * e2[1] - e1[1] * e2[0]};
      const double nn = std::sqrt((n[0] * n[0] + n[1] * n[1]) + n[2] * n[2]);
      for (int d = 0; d < 3; ++d) fn[3 * t + d] = n[d] / nn;
    }
    auto angle_at = [&](size_t t, uint32_t vid) {
      const uint32_t i0 = faces[3 * t], i1 = faces[3 * t + 1], i2 = faces[3 * t + 2];
      uint32_t o1, o2;
      if (vid == i0) { o1 = i1; o2 = i2; } else if (vid == i1) { o1 = i2; o2 = i0; } else { o1 = i0; o2 = i1; }
      double e1[3], e2[3];
      for (int d = 0; d < 3; ++d) { e1[d] = V(o1, d) - V(vid, d); e2[d] = V(o2, d) - V(vid, d); }
      double cs = ((e1[0] * e2[0] + e1[1] * e2[1]) + e1[2] * e2[2]) /
                  (std::sqrt((e1[0] * e1[0] + e1[1] * e1[1]) + e1[2] * e1[2]) *
                   std::sqrt((e2[0] * e2[0] + e2[1] * e2[1]) + e2[2] * e2[2]));
      cs = std::max(-1.0, std::min(1.0, cs));
      return std::acos(cs);
    };
    std::vector<std::vector<size_t>> incident(nv);
    for (size_t t = 0; t < nf; ++t)
      for (int k = 0; k < 3; ++k) incident[faces[3 * t + k]].push_back(t);
    for (size_t t = 0; t < nf; ++t) {
      for (int k = 0; k < 3; ++k) {
        const uint32_t vid = faces[3 * t + k];
        for (size_t u : incident[vid]) {
          const double ang = angle_at(u, vid);
          for (int d = 0; d < 3; ++d) vn[9 * t + 3 * k + d] += fn[3 * u + d] * ang;
        }
        const uint32_t ea = faces[3 * t + k], eb = faces[3 * t + (k + 1) % 3];
        for (size_t u : incident[ea]) {
          bool hb = false;
          for (int m = 0; m < 3; ++m) hb |= faces[3 * u + m] == eb;
          if (hb)
            for (int d = 0; d < 3; ++d) en[9 * t + 3 * k + d] += fn[3 * u + d];
        }
      }
    }
    sph::MeshDev M;
    double* dtri = dev_upload(tri.data(), tri.size());
    double* dfn = dev_upload(fn.data(), fn.size());
    double* den = dev_upload(en.data(), en.size());
    double* dvn = dev_upload(vn.data(), vn.size());
    M.tri = dtri; M.fn = dfn; M.en = den; M.vn = dvn; M.nt = (int)nf;
    const sph::LatticeDesc L = lattice_of(*g);
    const long long total = L.NX * L.NY * L.NZ;
    double* raw = nullptr;
    sph::cuda_check(cudaMalloc((void**)&raw, total * sizeof(double)), "cudaMalloc");
    sph::k_sdf_nodes<<<(unsigned)((total + 255) / 256), 256>>>(M, L, raw);
    sph::cuda_check(cudaGetLastError(), "k_sdf_nodes");
    const double pad = 3.1 * r;
    prune_and_download(L, raw, 1, -pad, 1, pad, out);
    cudaFree(raw); cudaFree(dtri); cudaFree(dfn); cudaFree(den); cudaFree(dvn);
  });
}

int sph_build_volume_map_field(const sph_grid_desc* sg, const double* sdf_nodes, const sph_grid_desc* vg, double r,
                               int degree, double* out, int device) {
  return guarded([&] {
    if (!sg || !sdf_nodes || !vg || !out || degree < 1 || degree > sph::kMaxGL)
      throw Error(SPH_ERR_INVALID, "invalid argument");
    sph::cuda_check(cudaSetDevice(device), "cudaSetDevice");
    sph::upload_serendipity_tables();
    std::vector<double> gx, gw;
    sph::gauss_legendre_nodes(degree, gx, gw);
    sph::cuda_check(cudaMemcpyToSymbol(sph::c_gl_x, gx.data(), degree * sizeof(double)), "gl nodes");
    sph::cuda_check(cudaMemcpyToSymbol(sph::c_gl_w, gw.data(), degree * sizeof(double)), "gl weights");
    const sph::LatticeDesc LS = lattice_of(*sg);
    const size_t ns = (size_t)(LS.NX * LS.NY * LS.NZ);
    double* dsdf = dev_upload(sdf_nodes, ns);
    sph::DevField F;
    for (int d = 0; d < 3; ++d) {
      F.xmin[d] = sg->x_min[d];
      F.xmax[d] = sg->x_max[d];
      F.n[d] = (int)sg->n[d];
    }
    F.dx = sg->dx;
    F.NX = LS.NX;
    F.NY = LS.NY;
    F.nodes = dsdf;
    const sph::LatticeDesc L = lattice_of(*vg);
    const long long total = L.NX * L.NY * L.NZ;
    double* raw = nullptr;
    sph::cuda_check(cudaMalloc((void**)&raw, total * sizeof(double)), "cudaMalloc");
    sph::k_volume_map_nodes<<<(unsigned)total, 256>>>(F, L, r, degree, raw);
    sph::cuda_check(cudaGetLastError(), "k_volume_map_nodes");
    prune_and_download(L, raw, 1, 0.0, 0, 0.0, out);
    cudaFree(raw);
    cudaFree(dsdf);
  });
}

}  // extern "C"
