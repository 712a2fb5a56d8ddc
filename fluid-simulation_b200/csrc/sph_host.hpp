// Host-side interface shared by the single-scene system (sph_system.cu) and
// the scene server (sph_server.cu): error type, CUDA status check and the
// precision-agnostic `SystemBase` that `System<float>` / `System<double>`
// implement.
#pragma once

#include <cuda_runtime.h>

#include <cstdint>
#include <stdexcept>
#include <string>
#include <vector>

#include "../../include/sphgpu.h"

namespace sph {

struct Error : std::runtime_error {
  int code;
  Error(int c, const std::string& m) : std::runtime_error(m), code(c) {}
};

extern thread_local std::string g_last_error;

inline void cuda_check(cudaError_t e, const char* what) {
  if (e == cudaSuccess) return;
  const int code = (e == cudaErrorMemoryAllocation) ? SPH_ERR_OOM : SPH_ERR_CUDA;
  throw Error(code, std::string(what) + ": " + cudaGetErrorString(e));
}

// Outcome of one asynchronous chunk of graph-captured steps.
struct ChunkOutcome {
  int status = SPH_OK;        // SPH_OK or SPH_NOT_CONVERGED
  uint32_t steps = 0;         // steps the chunk advanced
  bool replayed = false;      // the chunk was redone on the per-step path
};

// One reconstructed fluid surface: 6 doubles per vertex (position, normal).
struct SurfaceMeshOut {
  uint32_t fluid_id = 0;
  std::vector<double> vertices;
  std::vector<uint32_t> indices;
};

class SystemBase {
 public:
  virtual ~SystemBase() = default;
  virtual SystemBase* clone() const = 0;
  virtual void upload_fluid(size_t n, const double* x, const double* v, const double* m,
                            const uint32_t* fid) = 0;
  virtual int add_sample_boundary(size_t nb, const double* x, const sph_rigid_init* rigid) = 0;
  virtual int add_volume_map(const sph_grid_desc& sd, const double* sn, const sph_grid_desc& vd,
                             const double* vn, const sph_rigid_init* rigid) = 0;
  virtual void initialize() = 0;
  virtual int step(uint32_t n) = 0;
  virtual double time() const = 0;
  virtual uint64_t steps() const = 0;
  virtual void measurement(sph_measurement* m) = 0;
  virtual size_t num_particles() const = 0;
  virtual void download(int field, double* out) = 0;
  virtual void fluid_ids(uint32_t* out) = 0;
  virtual void fluid_pos(float* out) = 0;
  virtual void quantity(int q, float* out) = 0;
  virtual void quantity_at(int q, size_t n, const float* pos, float* out) = 0;
  virtual void reconstruct_surfaces(std::vector<SurfaceMeshOut>& out) = 0;
  virtual int fluid_neighbors(uint64_t* off, uint32_t* idx, size_t cap, size_t* total) = 0;
  virtual int boundary_neighbors(int bi, uint64_t* off, uint32_t* idx, size_t cap, size_t* total) = 0;
  virtual void boundary_volumes(int bi, double* out) = 0;
  virtual void boundary_positions(int bi, double* out) = 0;  // world frame, upload order
  virtual void vm_samples(int bi, uint8_t* has, double* xb, double* vb, double* vol) = 0;
  virtual void set_volume_map_aabb(int bi, const double* center, const double* half_extents) = 0;
  virtual void contact_stats(uint32_t* out4) = 0;  // cells, sweeps, overflow, capped of the last step
  virtual void set_contact_sweeps(uint32_t fixed) = 0;  // 0: merit test; n: exactly n sweeps
  // programmatic dependent launch between the sweep passes (on by default;
  // the scene server turns it off: its scenes share the SMs)
  virtual void set_dependent_launch(bool on) = 0;
  virtual uint32_t contact_sweeps() const = 0;
  virtual void rigid_state(int bi, double* out) = 0;
  virtual void set_rigid_state(int bi, const double* in) = 0;
  virtual uint64_t hash_collisions() = 0;
  virtual void restore(uint64_t steps, double time, size_t n, const double* x, const double* v,
                       const double* m, const uint32_t* fid, const double* xi, const double* vi) = 0;
  virtual int step_host(uint32_t n, const double* xi, const double* vi, double* xo, double* vo) = 0;
  virtual void* stream() const = 0;
  virtual void step_stats(sph_step_stats* out) const = 0;
  virtual uint64_t launches() const = 0;
  virtual void set_profiling(bool on) = 0;
  virtual bool kernel_time(const std::string& name, double* ms, uint64_t* count) = 0;
  virtual size_t device_bytes() const = 0;
  // Graph-captured stepping. `set_step_graphs(c)` with c > 0 makes `step`
  // advance in chunks of up to c graph launches with one host check per
  // chunk; 0 restores the per-step path. The chunk interface lets one host
  // thread keep many systems in flight: `chunk_begin` enqueues, `chunk_ready`
  // polls, `chunk_finish` checks (and replays the chunk on the per-step path
  // when a step needed host work: neighbor overflow, disabled particles or an
  // unconverged solve).
  virtual void set_step_graphs(uint32_t chunk) = 0;
  virtual uint32_t step_graph_chunk() const = 0;
  virtual void chunk_begin(uint32_t n) = 0;
  virtual bool chunk_ready() = 0;
  virtual ChunkOutcome chunk_finish() = 0;
  virtual uint64_t graph_replays() const = 0;
  // Result-invariant launch parameters of the neighbor passes (sph_tuning).
  virtual void get_tuning(sph_tuning* out) const = 0;
  virtual void set_tuning(const sph_tuning& t) = 0;
  int device = 0;
};

SystemBase* create_system(const sph_config& c);

}  // namespace sph

// The C ABI's owned mesh list (sph_reconstruct_surfaces).
struct sph_meshes {
  std::vector<sph::SurfaceMeshOut> m;
};
