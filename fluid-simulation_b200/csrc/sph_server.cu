// Scene server: the request-loop form of the reference's backend worker
// (sci-phi-backend/src/lib.rs:190-210 steps one Box<dyn SPHSystem> per
// worker). Many independent scenes share one GPU:
//
//  * a setup thread admits queued scenes in arrival order while the device
//    has a free slot and the scene's estimated device bytes fit the budget,
//    builds each one (upload, boundaries, first update, step graphs) on its
//    own stream, and later takes finished scenes' results and frees them;
//  * a scheduler thread keeps every admitted scene in flight: whenever a
//    scene's chunk of graph-captured steps has completed it checks the chunk
//    (replaying it per step if needed) and enqueues the next one, so the
//    kernels of all scenes overlap on the device.
//
// Scenes never share device data, and every kernel and reduction of a scene
// runs in a fixed order on its own stream, so a scene's result is the same
// alone and beside others.
#include <algorithm>
#include <atomic>
#include <chrono>
#include <cmath>
#include <condition_variable>
#include <cstring>
#include <deque>
#include <map>
#include <memory>
#include <mutex>
#include <set>
#include <thread>
#include <vector>

#include "sph_host.hpp"

namespace sph {

using Clock = std::chrono::steady_clock;

struct SceneJob {
  uint64_t ticket = 0;
  // deep copy of the request
  sph_config cfg{};
  std::vector<double> x, v, m;
  std::vector<uint32_t> fid;
  struct Samples {
    std::vector<double> x;
    bool dyn = false;
    sph_rigid_init rigid{};
  };
  struct VMap {
    sph_grid_desc sd{}, vd{};
    std::vector<double> sn, vn;
    bool dyn = false;
    sph_rigid_init rigid{};
  };
  std::vector<Samples> samples;
  std::vector<VMap> vmaps;
  uint32_t steps = 0;
  bool keep_state = false;
  uint64_t reserved = 0;
  // execution
  std::unique_ptr<SystemBase> sys;
  uint32_t done = 0;
  bool in_flight = false;
  int status = SPH_OK;
  std::string error;
  // result
  sph_scene_result result{};
  std::vector<double> xo, vo;
};

static size_t field_nodes(const sph_grid_desc& g) {
  return (size_t)(3 * g.n[0] + 1) * (size_t)(3 * g.n[1] + 1) * (size_t)(3 * g.n[2] + 1);
}

// Device bytes a scene will hold: the buffers System<R> allocates for its
// solver (at the default neighbor capacity plus growth room), the chunk
// snapshot, the Morton bucket arrays of its extent and its fields.
static uint64_t estimate_bytes(const SceneJob& j) {
  const double w = j.cfg.precision == SPH_F64 ? 8.0 : 4.0;
  const int ps = j.cfg.pressure_solver;
  const double K = std::max<double>(j.cfg.neighbor_capacity ? j.cfg.neighbor_capacity : 128, 128) * 1.5;
  double per = 4 * w * 8 + 4 * 8 + w * 2 + 2 * K + 4 * 8192.0 / 256;  // state, sort, p/bW, lists, halo table
  if (ps != SPH_SESPH) per += 4 * w;                    // predicted velocity
  if (ps == SPH_IISPH || ps == SPH_IISPH_W_OST) per += 2 * w + 18 * w;  // s, a_ii; sweep records xq, xu, uu, TA, TB, SA
  if (ps == SPH_SESPH_W_SPLITTING) per += w;
  if (j.cfg.integration_scheme == SPH_TAKE_PREDICTED) per += 2 * 4 * w * 2;
  per += 3 * 4 * w + 8;                                 // snapshot
  per += j.vmaps.size() * 2 * 4 * w;                    // volume-map samples
  size_t ns = 0;
  for (const auto& s : j.samples) ns += s.x.size() / 3;
  const size_t n = j.m.size();
  double bytes = per * (double)std::max<size_t>(n, 1) + (5 * 4 * w + 7 * 4) * (double)ns;
  // bucket count of System::choose_grid over the scene's bounding box
  double mn[3] = {INFINITY, INFINITY, INFINITY}, mx[3] = {-INFINITY, -INFINITY, -INFINITY};
  auto add = [&](const double* p) {
    for (int d = 0; d < 3; ++d) { mn[d] = std::min(mn[d], p[d]); mx[d] = std::max(mx[d], p[d]); }
  };
  for (size_t i = 0; i < n; ++i) add(&j.x[3 * i]);
  for (const auto& s : j.samples)
    for (size_t i = 0; i < s.x.size() / 3; ++i) add(&s.x[3 * i]);
  for (const auto& f : j.vmaps) {
    bytes += 8.0 * (double)(field_nodes(f.sd) + field_nodes(f.vd));
    if (!f.dyn) { add(f.sd.x_min); add(f.sd.x_max); add(f.vd.x_min); add(f.vd.x_max); }
  }
  double ext = 4;
  for (int d = 0; d < 3; ++d)
    if (mx[d] >= mn[d]) ext = std::max(ext, (mx[d] - mn[d]) / j.cfg.kernel_support_radius + 3.0);
  int mbits = 2;
  while (mbits < 8 && (double)(1u << mbits) < ext) ++mbits;
  const double T = (double)(1u << (3 * mbits)) + 2;
  bytes += T * 4 * (ns ? 4 : 2) + 2 * 8 * (double)(n / 256 + 1);
  return (uint64_t)(bytes * 1.1) + (4u << 20);
}

class Server {
 public:
  explicit Server(const sph_server_config& c) : cfg_(c) {
    if (cfg_.max_active == 0) cfg_.max_active = 64;
    if (cfg_.chunk_steps == 0) cfg_.chunk_steps = 25;
    cuda_check(cudaSetDevice(cfg_.device), "cudaSetDevice");
    size_t free_b = 0, total_b = 0;
    cuda_check(cudaMemGetInfo(&free_b, &total_b), "cudaMemGetInfo");
    budget_ = cfg_.memory_budget_bytes ? cfg_.memory_budget_bytes : (uint64_t)(0.9 * (double)free_b);
    t0_ = Clock::now();
    setup_thread_ = std::thread([this] { setup_loop(); });
    sched_thread_ = std::thread([this] { schedule_loop(); });
  }

  ~Server() {
    {
      std::lock_guard<std::mutex> lock(mu_);
      stop_ = true;
      stopping_.store(true);
      queue_.clear();
    }
    cv_.notify_all();
    sched_thread_.join();
    setup_thread_.join();
  }

  uint64_t submit(const sph_scene_request& r) {
    auto j = std::make_unique<SceneJob>();
    j->cfg = r.config;
    j->cfg.device = cfg_.device;
    if (r.n && (!r.position || !r.mass)) throw Error(SPH_ERR_INVALID, "null fluid arrays");
    j->x.assign(r.position, r.position + 3 * r.n);
    j->v = r.velocity ? std::vector<double>(r.velocity, r.velocity + 3 * r.n) : std::vector<double>(3 * r.n, 0.0);
    j->m.assign(r.mass, r.mass + r.n);
    j->fid = r.fluid_id ? std::vector<uint32_t>(r.fluid_id, r.fluid_id + r.n) : std::vector<uint32_t>(r.n, 0u);
    for (size_t b = 0; b < r.num_sample_sets; ++b) {
      const sph_sample_set& s = r.sample_sets[b];
      if (s.count && !s.positions) throw Error(SPH_ERR_INVALID, "null sample positions");
      SceneJob::Samples c;
      c.x.assign(s.positions, s.positions + 3 * s.count);
      c.dyn = s.rigid != nullptr;
      if (s.rigid) c.rigid = *s.rigid;
      j->samples.push_back(std::move(c));
    }
    for (size_t b = 0; b < r.num_volume_maps; ++b) {
      const sph_volume_map_set& f = r.volume_maps[b];
      if (!f.sdf || !f.sdf_nodes || !f.vm || !f.vm_nodes) throw Error(SPH_ERR_INVALID, "null volume map");
      SceneJob::VMap c;
      c.sd = *f.sdf;
      c.vd = *f.vm;
      c.sn.assign(f.sdf_nodes, f.sdf_nodes + field_nodes(*f.sdf));
      c.vn.assign(f.vm_nodes, f.vm_nodes + field_nodes(*f.vm));
      c.dyn = f.rigid != nullptr;
      if (f.rigid) c.rigid = *f.rigid;
      j->vmaps.push_back(std::move(c));
    }
    j->steps = r.steps;
    j->keep_state = r.keep_state != 0;
    j->reserved = estimate_bytes(*j);
    if (j->reserved > budget_) throw Error(SPH_ERR_CAPACITY, "scene exceeds the server's memory budget");
    j->result.submit_s = now();
    j->result.device_bytes_reserved = j->reserved;
    std::lock_guard<std::mutex> lock(mu_);
    if (stop_) throw Error(SPH_ERR_STATE, "server is stopping");
    j->ticket = ++next_ticket_;
    const uint64_t t = j->ticket;
    queue_.push_back(std::move(j));
    ++submitted_;
    cv_.notify_all();
    return t;
  }

  // true: finished (result copied); false: pending. Throws for unknown tickets.
  bool result(uint64_t t, double timeout_s, sph_scene_result* out) {
    std::unique_lock<std::mutex> lock(mu_);
    if (!known(t)) throw Error(SPH_ERR_INVALID, "unknown ticket");
    auto done = [&] { return finished_.count(t) != 0; };
    if (!done() && timeout_s != 0) {
      if (timeout_s < 0) done_cv_.wait(lock, done);
      else done_cv_.wait_for(lock, std::chrono::duration<double>(timeout_s), done);
    }
    auto it = finished_.find(t);
    if (it == finished_.end()) return false;
    if (out) *out = it->second->result;
    return true;
  }

  void fetch_state(uint64_t t, double* x, double* v) {
    std::lock_guard<std::mutex> lock(mu_);
    auto it = finished_.find(t);
    if (it == finished_.end()) throw Error(known(t) ? SPH_PENDING : SPH_ERR_INVALID, "scene not finished");
    const SceneJob& j = *it->second;
    if (!j.keep_state) throw Error(SPH_ERR_STATE, "scene was submitted without keep_state");
    if (x) std::copy(j.xo.begin(), j.xo.end(), x);
    if (v) std::copy(j.vo.begin(), j.vo.end(), v);
  }

  void release(uint64_t t) {
    std::lock_guard<std::mutex> lock(mu_);
    if (!finished_.erase(t)) throw Error(SPH_ERR_INVALID, "no finished scene with this ticket");
    released_.insert(t);
  }

  void stats(sph_server_stats* o) {
    std::lock_guard<std::mutex> lock(mu_);
    std::memset(o, 0, sizeof *o);
    o->submitted = submitted_;
    o->completed = completed_;
    o->queued = queue_.size();
    o->active = n_active_;
    o->peak_active = peak_active_;
    o->budget_bytes = budget_;
    o->reserved_bytes = reserved_;
    o->peak_reserved_bytes = peak_reserved_;
    o->graph_replays = replays_;
    o->kernel_launches = launches_;
  }

 private:
  sph_server_config cfg_;
  uint64_t budget_ = 0;
  Clock::time_point t0_;
  std::mutex mu_;
  std::condition_variable cv_, done_cv_;
  bool stop_ = false;
  std::atomic<bool> stopping_{false};
  uint64_t next_ticket_ = 0, submitted_ = 0, completed_ = 0, reserved_ = 0, peak_reserved_ = 0;
  uint64_t n_active_ = 0, peak_active_ = 0, replays_ = 0, launches_ = 0;
  std::deque<std::unique_ptr<SceneJob>> queue_;       // waiting for admission
  std::vector<std::unique_ptr<SceneJob>> ready_;      // built, not yet picked up by the scheduler
  std::vector<std::unique_ptr<SceneJob>> retiring_;   // stepped to the end, results not yet taken
  std::map<uint64_t, std::unique_ptr<SceneJob>> finished_;
  std::set<uint64_t> released_;
  std::thread setup_thread_, sched_thread_;

  double now() const { return std::chrono::duration<double>(Clock::now() - t0_).count(); }
  bool known(uint64_t t) const { return t >= 1 && t <= next_ticket_ && released_.count(t) == 0; }

  // Builds a scene's system exactly as the single-scene C ABI does.
  void build(SceneJob& j) {
    std::unique_ptr<SystemBase> s(create_system(j.cfg));
    s->upload_fluid(j.m.size(), j.x.data(), j.v.data(), j.m.data(), j.fid.data());
    for (const auto& b : j.samples) s->add_sample_boundary(b.x.size() / 3, b.x.data(), b.dyn ? &b.rigid : nullptr);
    for (const auto& f : j.vmaps)
      s->add_volume_map(f.sd, f.sn.data(), f.vd, f.vn.data(), f.dyn ? &f.rigid : nullptr);
    s->initialize();
    // concurrent scenes share the SMs: blocks of an early-launched dependent
    // kernel would hold SM resources another scene's kernels could use
    s->set_dependent_launch(false);
    s->set_step_graphs(cfg_.chunk_steps);
    j.sys = std::move(s);
    // the inputs are on the device now
    std::vector<double>().swap(j.x);
    std::vector<double>().swap(j.v);
    std::vector<double>().swap(j.m);
    std::vector<uint32_t>().swap(j.fid);
    j.samples.clear();
    j.vmaps.clear();
  }

  void take_result(SceneJob& j) {
    sph_scene_result& r = j.result;
    r.status = j.status;
    if (j.sys) {
      try {
        r.steps = j.sys->steps();
        r.time = j.sys->time();
        r.particles = j.sys->num_particles();
        j.sys->measurement(&r.measurement);
        r.graph_replays = j.sys->graph_replays();
        r.kernel_launches = j.sys->launches();
        if (j.keep_state && j.status != SPH_ERR_CUDA) {
          j.xo.resize(3 * r.particles);
          j.vo.resize(3 * r.particles);
          j.sys->download(SPH_FIELD_POSITION, j.xo.data());
          j.sys->download(SPH_FIELD_VELOCITY, j.vo.data());
        }
      } catch (const Error& e) {
        if (r.status == SPH_OK || r.status == SPH_NOT_CONVERGED) r.status = e.code;
        j.error = e.what();
      }
      j.sys.reset();
    }
    r.finish_s = now();
  }

  void setup_loop() {
    cudaSetDevice(cfg_.device);
    for (;;) {
      std::unique_ptr<SceneJob> job;
      std::vector<std::unique_ptr<SceneJob>> retired;
      {
        std::unique_lock<std::mutex> lock(mu_);
        auto admissible = [&] {
          return !queue_.empty() && n_active_ < cfg_.max_active && reserved_ + queue_.front()->reserved <= budget_;
        };
        cv_.wait(lock, [&] { return !retiring_.empty() || (stop_ && n_active_ == 0) || (!stop_ && admissible()); });
        retired.swap(retiring_);
        if (retired.empty() && stop_ && n_active_ == 0) break;
        if (!stop_ && admissible()) {
          job = std::move(queue_.front());
          queue_.pop_front();
          reserved_ += job->reserved;
          peak_reserved_ = std::max(peak_reserved_, reserved_);
          ++n_active_;
          peak_active_ = std::max(peak_active_, n_active_);
        }
      }
      for (auto& r : retired) {
        take_result(*r);
        std::lock_guard<std::mutex> lock(mu_);
        reserved_ -= r->reserved;
        --n_active_;
        ++completed_;
        replays_ += r->result.graph_replays;
        launches_ += r->result.kernel_launches;
        const uint64_t t = r->ticket;
        finished_[t] = std::move(r);
        done_cv_.notify_all();
        cv_.notify_all();
      }
      if (job) {
        job->result.start_s = now();
        try {
          build(*job);
        } catch (const Error& e) {
          job->status = e.code;
          job->error = e.what();
        } catch (const std::exception& e) {
          job->status = SPH_ERR_CUDA;
          job->error = e.what();
        }
        std::lock_guard<std::mutex> lock(mu_);
        if (job->status != SPH_OK || job->steps == 0) retiring_.push_back(std::move(job));
        else ready_.push_back(std::move(job));
        cv_.notify_all();
      }
    }
  }

  void schedule_loop() {
    cudaSetDevice(cfg_.device);
    std::vector<std::unique_ptr<SceneJob>> active;
    for (;;) {
      {
        std::lock_guard<std::mutex> lock(mu_);
        for (auto& j : ready_) active.push_back(std::move(j));
        ready_.clear();
        if (stop_ && active.empty() && n_active_ == 0) break;
      }
      bool progressed = false;
      for (size_t k = 0; k < active.size();) {
        SceneJob& j = *active[k];
        bool retire = false;
        try {
          if (j.in_flight) {
            if (!j.sys->chunk_ready()) {
              ++k;
              continue;
            }
            const ChunkOutcome o = j.sys->chunk_finish();
            j.in_flight = false;
            j.done += o.steps;
            if (o.status != SPH_OK && j.status == SPH_OK) j.status = o.status;
            progressed = true;
          }
          const bool stopping = stopping_.load();
          if (j.done >= j.steps || stopping) {
            if (stopping && j.done < j.steps && j.status == SPH_OK) {
              j.status = SPH_ERR_STATE;
              j.error = "server destroyed before the scene finished";
            }
            retire = true;
          } else {
            j.sys->chunk_begin(std::min(cfg_.chunk_steps, j.steps - j.done));
            j.in_flight = true;
            progressed = true;
          }
        } catch (const Error& e) {
          j.status = e.code;
          j.error = e.what();
          j.in_flight = false;
          retire = true;
        }
        if (retire) {
          std::lock_guard<std::mutex> lock(mu_);
          retiring_.push_back(std::move(active[k]));
          active.erase(active.begin() + (long)k);
          cv_.notify_all();
          progressed = true;
        } else {
          ++k;
        }
      }
      if (!progressed) {
        if (active.empty()) {
          std::unique_lock<std::mutex> lock(mu_);
          cv_.wait_for(lock, std::chrono::milliseconds(1), [&] { return !ready_.empty(); });
        } else {
          std::this_thread::sleep_for(std::chrono::microseconds(20));
        }
      }
    }
  }
};

}  // namespace sph

struct sph_server {
  std::unique_ptr<sph::Server> impl;
};

namespace {
template <class F>
int guarded_srv(F&& f) {
  try {
    return f();
  } catch (const sph::Error& e) {
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
}  // namespace

extern "C" {

int sph_server_create(const sph_server_config* cfg, sph_server_t** out) {
  return guarded_srv([&] {
    if (!cfg || !out) throw sph::Error(SPH_ERR_INVALID, "null argument");
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0)
      throw sph::Error(SPH_ERR_CUDA, "no CUDA device available");
    if (cfg->device < 0 || cfg->device >= ndev) throw sph::Error(SPH_ERR_INVALID, "device ordinal out of range");
    auto s = std::make_unique<sph_server>();
    s->impl = std::make_unique<sph::Server>(*cfg);
    *out = s.release();
    return (int)SPH_OK;
  });
}

int sph_server_submit(sph_server_t* s, const sph_scene_request* req, uint64_t* ticket) {
  return guarded_srv([&] {
    if (!s || !req || !ticket) throw sph::Error(SPH_ERR_INVALID, "null argument");
    *ticket = s->impl->submit(*req);
    return (int)SPH_OK;
  });
}

int sph_server_poll(sph_server_t* s, uint64_t ticket, sph_scene_result* out) {
  return guarded_srv([&] {
    if (!s) throw sph::Error(SPH_ERR_INVALID, "null argument");
    return s->impl->result(ticket, 0.0, out) ? (int)SPH_OK : (int)SPH_PENDING;
  });
}

int sph_server_wait(sph_server_t* s, uint64_t ticket, double timeout_s, sph_scene_result* out) {
  return guarded_srv([&] {
    if (!s) throw sph::Error(SPH_ERR_INVALID, "null argument");
    return s->impl->result(ticket, timeout_s, out) ? (int)SPH_OK : (int)SPH_PENDING;
  });
}

int sph_server_fetch_state(sph_server_t* s, uint64_t ticket, double* position, double* velocity) {
  return guarded_srv([&] {
    if (!s) throw sph::Error(SPH_ERR_INVALID, "null argument");
    s->impl->fetch_state(ticket, position, velocity);
    return (int)SPH_OK;
  });
}

int sph_server_release(sph_server_t* s, uint64_t ticket) {
  return guarded_srv([&] {
    if (!s) throw sph::Error(SPH_ERR_INVALID, "null argument");
    s->impl->release(ticket);
    return (int)SPH_OK;
  });
}

int sph_server_get_stats(sph_server_t* s, sph_server_stats* out) {
  return guarded_srv([&] {
    if (!s || !out) throw sph::Error(SPH_ERR_INVALID, "null argument");
    s->impl->stats(out);
    return (int)SPH_OK;
  });
}

void sph_server_destroy(sph_server_t* s) { delete s; }

}  // extern "C"
