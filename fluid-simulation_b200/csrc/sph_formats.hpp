// Readback formats either side of the step path: the system checkpoint
// (SerSystemCheckpoint, sph/mod.rs:883-915, written as RON by
// sci-phi-backend/src/recording.rs:37-61 and read back by the `--state` path
// of sph/setup/mod.rs:142-153; it also derives bincode Encode/Decode) and the
// recording frame (TimeStepInfo, render_info.rs:71-106, bincode).
//
// Both serializers are third-party crates in the reference (ron 0.12,
// bincode 2.0 with `config::standard()`); this file restates their published
// encodings for exactly the types above:
//   bincode standard: little endian; unsigned integers as varints (< 251 one
//     byte; else a marker 251/252/253 followed by u16/u32/u64), usize as u64;
//     f32/f64 as raw little-endian bytes; Vec/String as a varint length then
//     the elements; fixed arrays and tuples as their elements alone; Option as
//     a byte 0/1 then the value; enum variants as a u32 varint index then the
//     fields; structs as their fields in declaration order.
//   RON (ron::to_string, no pretty config): structs as `(field:value,...)`
//     without the struct name, sequences `[a,b]`, tuples and fixed arrays
//     `(a,b,c)`, `Some(v)` / `None`, integers in decimal, floats as Rust's
//     `Display` (shortest round-trip digits, never an exponent) with `.0`
//     appended to integral values.
#pragma once

#include <array>
#include <cstddef>
#include <cstdint>
#include <string>
#include <vector>

#include "../../include/sphgpu.h"

namespace sph {
namespace fmt {

// SerRigidBodyMotionCheckpoint (rigid_body_motion.rs:248-257) in the layout of
// sph_get_rigid_state: com[3], q[4] (w,i,j,k), v[3], L[3], F[3], T[3].
struct RigidState {
  bool dynamic = false;
  std::array<double, 19> s{};
};

// SystemCheckpoint / SerSystemCheckpoint (sph/mod.rs:833-915,
// fluid.rs:351-421, boundary_handling/mod.rs:135-170).
struct Checkpoint {
  uint64_t time_steps_propagated = 0;
  double current_time = 0;
  std::vector<uint32_t> fluid_id;
  std::vector<double> position, velocity, mass;          // 3n, 3n, n
  std::vector<std::vector<double>> integrator_position;  // slots x 3n
  std::vector<std::vector<double>> integrator_velocity;
  std::vector<RigidState> boundaries;
  size_t n() const { return mass.size(); }
  void check() const;  // array sizes agree
};

std::string checkpoint_to_ron(const Checkpoint& c);
Checkpoint checkpoint_from_ron(const char* text, size_t len);
std::vector<uint8_t> checkpoint_to_bincode(const Checkpoint& c);
Checkpoint checkpoint_from_bincode(const uint8_t* data, size_t len);

// TimeStepInfo (render_info.rs:71-81).
std::vector<uint8_t> time_step_info_to_bincode(const sph_frame_view& f);

// Rust's `Display` of an f64, the float syntax of RON's writer.
std::string rust_display(double v);

}  // namespace fmt
}  // namespace sph

// The C ABI's owned objects.
struct sph_bytes {
  std::vector<uint8_t> b;
};
struct sph_checkpoint {
  sph::fmt::Checkpoint c;
  // flat copies backing sph_checkpoint_view_of
  std::vector<double> xi, vi, rigid;
  std::vector<uint8_t> dyn;
};

namespace sph {
namespace fmt {
sph_bytes_t* new_bytes(std::vector<uint8_t>&& b);
sph_checkpoint_t* new_checkpoint(Checkpoint&& c);  // checks the array sizes
}  // namespace fmt
}  // namespace sph
