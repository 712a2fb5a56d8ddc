"""GPU-backed `SPHSystem` (reference: simulation_lib/src/sph/mod.rs:40-69).

`GpuSystem` mirrors the reference's object-safe system trait — `time`,
`time_steps_propagated`, `step_forward_in_time`, `take_measurement`,
`get_fluid_ids`, `get_fluid_pos`, `get_fluid_checkpoint`,
`get_quantity_of_fluid_samples`, `continue_from_checkpoint`, clone — over the
C ABI. Composition follows the reference's `Procedures` (sph/setup/input.rs:
101-134) and `Parameters` names; all state stays on the device between calls.
"""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass

import numpy as np

from . import _capi as A

PROCEDURES = {
    "kernel_function": {"CubicBSpline3D": A.CUBIC_BSPLINE_3D},
    "integration_scheme": {"EulerCromer": A.EULER_CROMER, "TakePredicted": A.TAKE_PREDICTED},
    "pressure_solver": {"SESPH": A.SESPH, "SESPHwSplitting": A.SESPH_W_SPLITTING, "IISPH": A.IISPH,
                        "IISPHwOST": A.IISPH_W_OST},
    "neighbor_search": {"SpatialHashing": A.SPATIAL_HASHING},
    "boundary_handling": {"StaticSampleBoundary": A.STATIC_SAMPLE_BOUNDARY,
                          "VolumeMapBoundary": A.VOLUME_MAP_BOUNDARY},
}

PARAMETER_KEYS = (
    "rest_density_grid_spacing", "kernel_support_radius", "disable_particles_below",
    "fluid_viscosity", "boundary_viscosity", "boundary_pressure_acceleration_weighting",
    "boundary_rest_volume_weighting", "stiffness", "target_density_error", "relaxation_factor",
    "min_diagonal_element", "time_increment", "max_time_increment", "cfl_number",
    "max_solver_iterations", "neighbor_capacity", "device",
)


def make_config(procedures: dict | None = None, parameters: dict | None = None,
                precision: str = "f32", cfl_time_step: bool = False,
                gravity: dict | None = None) -> A.SphConfig:
    """Build an `sph_config` from reference-style procedure names and parameters."""
    L = A.load()
    c = A.SphConfig()
    L.sph_config_default(C.byref(c))
    procedures = procedures or {}
    field_of = {"kernel_function": "kernel_fn", "integration_scheme": "integration_scheme",
                "pressure_solver": "pressure_solver", "neighbor_search": "neighbor_search",
                "boundary_handling": "boundary_handling"}
    for key, value in procedures.items():
        if key not in PROCEDURES:
            raise ValueError(f"unknown procedure {key!r}")
        if value not in PROCEDURES[key]:
            raise ValueError(f"unknown {key} variant {value!r}")
        setattr(c, field_of[key], PROCEDURES[key][value])
    for key, value in (parameters or {}).items():
        if key not in PARAMETER_KEYS:
            raise ValueError(f"unknown parameter {key!r}")
        setattr(c, key, value)
    c.precision = {"f32": A.F32, "f64": A.F64}[precision]
    c.cfl_time_step = 1 if cfl_time_step else 0
    if gravity:
        if gravity.get("type", "Uniform") == "Radial":
            c.gravity_mode = A.GRAVITY_RADIAL
            c.gravity_center[:] = gravity["center"]
        else:
            c.gravity_mode = A.GRAVITY_UNIFORM
    return c


@dataclass
class RigidInit:
    """Initial state of a dynamic boundary (RigidBodyMotion::new)."""
    mass: float
    inertia_body: np.ndarray
    center_of_mass: tuple
    orientation: tuple = (1.0, 0.0, 0.0, 0.0)  # w, i, j, k
    linear_velocity: tuple = (0.0, 0.0, 0.0)
    angular_velocity: tuple = (0.0, 0.0, 0.0)

    def to_c(self) -> A.SphRigidInit:
        r = A.SphRigidInit()
        I = np.asarray(self.inertia_body, np.float64).reshape(3, 3)
        r.mass = float(self.mass)
        r.inertia_body[:] = I.ravel().tolist()
        r.inertia_inv_body[:] = np.linalg.inv(I).ravel().tolist()
        r.center_of_mass[:] = list(self.center_of_mass)
        r.orientation[:] = list(self.orientation)
        r.linear_velocity[:] = list(self.linear_velocity)
        r.angular_velocity[:] = list(self.angular_velocity)
        return r

    def to_array32(self) -> np.ndarray:
        """The 32-double layout the oracle's rigid-body entry points take."""
        I = np.asarray(self.inertia_body, np.float64).reshape(3, 3)
        return np.concatenate([[self.mass], I.ravel(), np.linalg.inv(I).ravel(),
                               self.center_of_mass, self.orientation, self.linear_velocity,
                               self.angular_velocity]).astype(np.float64)


def grid_desc(x_min, x_max, dx, n) -> A.SphGridDesc:
    g = A.SphGridDesc()
    g.x_min[:] = [float(v) for v in x_min]
    g.x_max[:] = [float(v) for v in x_max]
    g.dx = float(dx)
    g.n[:] = [int(v) for v in n]
    return g


class GpuSystem:
    """A `System<K,I,P,N,B>` whose state lives on one GPU."""

    def __init__(self, config: A.SphConfig):
        self._L = A.load()
        self._cfg = config
        h = C.c_void_p()
        A.check(self._L.sph_create(C.byref(config), C.byref(h)))
        self._h = h
        self._boundaries = []

    # ---- lifetime --------------------------------------------------------------
    def close(self):
        if getattr(self, "_h", None):
            self._L.sph_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def clone(self) -> "GpuSystem":
        o = GpuSystem.__new__(GpuSystem)
        o._L, o._cfg, o._boundaries = self._L, self._cfg, list(self._boundaries)
        h = C.c_void_p()
        A.check(self._L.sph_clone(self._h, C.byref(h)))
        o._h = h
        return o

    # ---- setup -----------------------------------------------------------------
    def upload_fluid(self, position, velocity=None, mass=None, fluid_id=None):
        pos = np.ascontiguousarray(position, np.float64).reshape(-1, 3)
        n = pos.shape[0]
        vel = np.ascontiguousarray(np.zeros((n, 3)) if velocity is None else velocity,
                                   np.float64).reshape(-1, 3)
        m = np.ascontiguousarray(np.broadcast_to(mass, (n,)), np.float64)
        fid = np.ascontiguousarray(np.zeros(n) if fluid_id is None else fluid_id, np.uint32)
        A.check(self._L.sph_upload_fluid(self._h, n, pos.ravel(), vel.ravel(), m, fid))

    def add_sample_boundary(self, positions, rigid: RigidInit | None = None) -> int:
        p = np.ascontiguousarray(positions, np.float64).reshape(-1, 3)
        bi = C.c_int()
        r = C.byref(rigid.to_c()) if rigid is not None else None
        A.check(self._L.sph_add_sample_boundary(self._h, p.shape[0], p.ravel(), r, C.byref(bi)))
        self._boundaries.append(("samples", p.shape[0]))
        return bi.value

    def add_volume_map_boundary(self, sdf, vm, rigid: RigidInit | None = None, aabb=None) -> int:
        """sdf / vm: objects with x_min, x_max, dx, n, nodes (dense lattice, NaN absent).
        aabb: (center, half_extents) of the mesh in the body frame; boundaries
        with one take part in rigid-rigid contact."""
        bi = C.c_int()
        r = C.byref(rigid.to_c()) if rigid is not None else None
        sd = grid_desc(sdf.x_min, sdf.x_max, sdf.dx, sdf.n)
        vd = grid_desc(vm.x_min, vm.x_max, vm.dx, vm.n)
        A.check(self._L.sph_add_volume_map_boundary(
            self._h, C.byref(sd), np.ascontiguousarray(sdf.nodes, np.float64).ravel(), C.byref(vd),
            np.ascontiguousarray(vm.nodes, np.float64).ravel(), r, C.byref(bi)))
        self._boundaries.append(("volume_map", 0))
        if aabb is not None:
            c = np.ascontiguousarray(aabb[0], np.float64).reshape(3)
            h = np.ascontiguousarray(aabb[1], np.float64).reshape(3)
            A.check(self._L.sph_set_volume_map_aabb(self._h, bi.value, c, h))
        return bi.value

    def set_contact_sweeps(self, fixed_sweeps: int):
        """0: the reference's merit test ends each contact solve; n > 0:
        exactly n sweeps after the first (sph_set_contact_sweeps)."""
        A.check(self._L.sph_set_contact_sweeps(self._h, int(fixed_sweeps)))

    def contact_stats(self) -> dict:
        """Rigid-rigid contact of the last step: cells, solver sweeps, whether
        sub-cells were dropped for capacity, whether the sweep cap stopped it."""
        out = np.zeros(4, np.uint32)
        A.check(self._L.sph_get_contact_stats(self._h, out))
        return dict(zip(("cells", "sweeps", "overflow", "capped"), out.tolist()))

    def initialize(self):
        A.check(self._L.sph_initialize(self._h))

    # ---- SPHSystem -------------------------------------------------------------
    def time(self) -> float:
        t = C.c_double()
        A.check(self._L.sph_time(self._h, C.byref(t)))
        return t.value

    def time_steps_propagated(self) -> int:
        s = C.c_uint64()
        A.check(self._L.sph_time_steps_propagated(self._h, C.byref(s)))
        return s.value

    def step_forward_in_time(self, n_steps: int = 1) -> int:
        """Advance n_steps; returns SPH_OK or SPH_NOT_CONVERGED (capped IISPH)."""
        return A.check(self._L.sph_step(self._h, int(n_steps)), allow=(A.SPH_NOT_CONVERGED,))

    def step_host(self, n_steps, position_in=None, velocity_in=None, position_out=None,
                  velocity_out=None) -> int:
        """sph_step_host: host arrays (reference order, float64 [n,3]) in and out;
        pinned arrays (e.g. torch pin_memory) make the copies fastest."""
        def ptr(a):
            if a is None:
                return None
            if hasattr(a, "data_ptr"):
                return C.c_void_p(a.data_ptr())
            return a.ctypes.data_as(C.c_void_p)
        return A.check(self._L.sph_step_host(self._h, int(n_steps), ptr(position_in), ptr(velocity_in),
                                             ptr(position_out), ptr(velocity_out)),
                       allow=(A.SPH_NOT_CONVERGED,))

    def step_stats(self) -> dict:
        """Scalars of the last update (no device work)."""
        st = A.SphStepStats()
        A.check(self._L.sph_get_step_stats(self._h, C.byref(st)))
        return {name: getattr(st, name) for name, _ in A.SphStepStats._fields_}

    def stream(self) -> int:
        """cudaStream_t of the handle as an integer (torch.cuda.ExternalStream)."""
        s = C.c_void_p()
        A.check(self._L.sph_get_stream(self._h, C.byref(s)))
        return s.value or 0

    def take_measurement(self) -> dict:
        m = A.SphMeasurement()
        A.check(self._L.sph_take_measurement(self._h, C.byref(m)))
        return {name: getattr(m, name) for name, _ in A.SphMeasurement._fields_}

    @property
    def n(self) -> int:
        s = C.c_size_t()
        A.check(self._L.sph_num_particles(self._h, C.byref(s)))
        return s.value

    def get_fluid_ids(self) -> np.ndarray:
        out = np.zeros(self.n, np.uint32)
        A.check(self._L.sph_get_fluid_ids(self._h, out))
        return out

    def get_fluid_pos(self) -> np.ndarray:
        out = np.zeros(3 * self.n, np.float32)
        A.check(self._L.sph_get_fluid_pos(self._h, out))
        return out.reshape(-1, 3)

    def get_quantity_of_fluid_samples(self, quantity: int) -> np.ndarray:
        out = np.zeros(self.n, np.float32)
        A.check(self._L.sph_get_quantity_of_fluid_samples(self._h, int(quantity), out))
        return out

    def get_quantity_at_positions(self, quantity: int, positions) -> np.ndarray:
        """SPHSystem::get_quantity_at_positions (sph/mod.rs:241-341): the
        quantity at arbitrary positions (n x 3, taken as f32 like the
        reference's `&[[f32; 3]]`), e.g. the points of a sensor plane."""
        pos = np.ascontiguousarray(positions, np.float32).reshape(-1, 3)
        out = np.zeros(pos.shape[0], np.float32)
        A.check(self._L.sph_get_quantity_at_positions(self._h, int(quantity), pos.shape[0],
                                                      pos.reshape(-1), out))
        return out

    def download(self, field: int) -> np.ndarray:
        n = self.n
        shape = (n, 3) if field in A.VECTOR_FIELDS else (n,)
        out = np.zeros(int(np.prod(shape)), np.float64)
        A.check(self._L.sph_download(self._h, int(field), out))
        return out.reshape(shape)

    def get_fluid_checkpoint(self) -> dict:
        """FluidCheckpoint (fluid.rs:352-447): ids, positions, velocities, masses."""
        ck = {"fluid_id": self.get_fluid_ids(), "position": self.download(A.FIELD_POSITION),
              "velocity": self.download(A.FIELD_VELOCITY), "mass": self.download(A.FIELD_MASS),
              "time_steps_propagated": self.time_steps_propagated(), "current_time": self.time()}
        if self._cfg.integration_scheme == A.TAKE_PREDICTED:
            ck["integrator_position"] = self.download(A.FIELD_INTEGRATOR_POSITION)
            ck["integrator_velocity"] = self.download(A.FIELD_INTEGRATOR_VELOCITY)
        return ck

    def continue_from_checkpoint(self, ck: dict):
        pos = np.ascontiguousarray(ck["position"], np.float64).reshape(-1, 3)
        n = pos.shape[0]
        vel = np.ascontiguousarray(ck["velocity"], np.float64).reshape(-1, 3)
        m = np.ascontiguousarray(ck["mass"], np.float64)
        fid = np.ascontiguousarray(ck["fluid_id"], np.uint32)
        xi = ck.get("integrator_position")
        vi = ck.get("integrator_velocity")
        xi = None if xi is None else np.ascontiguousarray(xi, np.float64).ravel()
        vi = None if vi is None else np.ascontiguousarray(vi, np.float64).ravel()
        A.check(self._L.sph_continue_from_checkpoint(
            self._h, int(ck["time_steps_propagated"]), float(ck["current_time"]), n, pos.ravel(),
            vel.ravel(), m, fid, None if xi is None else xi.ctypes.data_as(C.c_void_p),
            None if vi is None else vi.ctypes.data_as(C.c_void_p)))

    # ---- parity helpers ----------------------------------------------------------
    def fluid_neighbors(self):
        """(offsets[n+1], indices) in reference index space, rows sorted, self included."""
        total = C.c_size_t()
        rc = self._L.sph_get_fluid_neighbors(self._h, None, None, 0, C.byref(total))
        A.check(rc, allow=(A.SPH_ERR_CAPACITY,))
        off = np.zeros(self.n + 1, np.uint64)
        idx = np.zeros(max(total.value, 1), np.uint32)
        A.check(self._L.sph_get_fluid_neighbors(self._h, off.ctypes.data_as(C.c_void_p),
                                                idx.ctypes.data_as(C.c_void_p), idx.size,
                                                C.byref(total)))
        return off, idx[:total.value]

    def boundary_neighbors(self, bi: int):
        total = C.c_size_t()
        rc = self._L.sph_get_boundary_neighbors(self._h, bi, None, None, 0, C.byref(total))
        A.check(rc, allow=(A.SPH_ERR_CAPACITY,))
        off = np.zeros(self.n + 1, np.uint64)
        idx = np.zeros(max(total.value, 1), np.uint32)
        A.check(self._L.sph_get_boundary_neighbors(self._h, bi, off.ctypes.data_as(C.c_void_p),
                                                   idx.ctypes.data_as(C.c_void_p), idx.size,
                                                   C.byref(total)))
        return off, idx[:total.value]

    def boundary_volumes(self, bi: int, nb: int) -> np.ndarray:
        out = np.zeros(nb)
        A.check(self._L.sph_get_boundary_volumes(self._h, bi, out))
        return out

    def boundary_positions(self, bi: int, nb: int) -> np.ndarray:
        out = np.zeros(3 * nb)
        A.check(self._L.sph_get_boundary_positions(self._h, bi, out))
        return out.reshape(-1, 3)

    # ---- surfaces, checkpoints and recording frames ------------------------------
    def reconstruct_surfaces(self):
        """Fluid::reconstruct_surfaces (sph/fluid.rs:212-347): [(fluid_id,
        vertices (n, 6): position and unit normal, indices (3 per triangle))]."""
        h = C.c_void_p()
        A.check(self._L.sph_reconstruct_surfaces(self._h, C.byref(h)))
        try:
            cnt = C.c_size_t()
            A.check(self._L.sph_meshes_count(h, C.byref(cnt)))
            out = []
            for k in range(cnt.value):
                fid, nv, ni = C.c_uint32(), C.c_size_t(), C.c_size_t()
                vp, ip = C.POINTER(C.c_double)(), C.POINTER(C.c_uint32)()
                A.check(self._L.sph_meshes_get(h, k, C.byref(fid), C.byref(nv), C.byref(vp), C.byref(ni),
                                               C.byref(ip)))
                v = np.ctypeslib.as_array(vp, shape=(6 * nv.value,)).reshape(-1, 6).copy() if nv.value else \
                    np.zeros((0, 6))
                i = np.ctypeslib.as_array(ip, shape=(ni.value,)).copy() if ni.value else np.zeros(0, np.uint32)
                out.append((fid.value, v, i))
            return out
        finally:
            self._L.sph_meshes_free(h)

    # ---- checkpoints and recording frames ------------------------------------
    def get_checkpoint(self):
        """SystemCheckpoint::from_sph_system (sph/mod.rs:849-856)."""
        from .formats import _from_handle
        h = C.c_void_p()
        A.check(self._L.sph_get_checkpoint(self._h, C.byref(h)))
        try:
            return _from_handle(h)
        finally:
            self._L.sph_checkpoint_free(h)

    def restore_checkpoint(self, ck):
        """SPHSystem::continue_from_checkpoint (sph/mod.rs:362-378) from a
        `formats.Checkpoint` (fluid, rigid states, step counter and time)."""
        from .formats import _to_handle
        h = _to_handle(ck)
        try:
            A.check(self._L.sph_restore_checkpoint(self._h, h))
        finally:
            self._L.sph_checkpoint_free(h)

    def encode_time_step_info(self, fluid="samples", fluid_coloring="uniform", quantity=A.Q_SPEED,
                              planes=(), boundary_coloring="uniform", render_mesh_ids=None,
                              boundary="samples", render_meshes=None) -> bytes:
        """TimeStepInfo::from_system (render_info.rs:83-92) as bincode bytes.
        fluid: "samples", "sensor_plane" or "triangle_mesh"; fluid_coloring:
        "uniform", "id" or "quantity" (samples); planes: [(positions, rows,
        cols)]; boundary: "samples" (boundary_coloring "uniform" or "id") or
        "triangle_mesh" with render_meshes [(vertices (n, 6), indices)] per
        boundary (boundary_coloring "original", "uniform" or "id")."""
        from .formats import _bytes
        keep = []
        sel = A.SphFrameSelector()
        sel.fluid = {"samples": A.FLUID_SAMPLES, "sensor_plane": A.FLUID_SENSOR_PLANE,
                     "triangle_mesh": A.FLUID_TRIANGLE_MESH}[fluid]
        sel.fluid_coloring = {"uniform": A.COLORING_UNIFORM, "id": A.COLORING_ID,
                              "quantity": A.COLORING_QUANTITY}[fluid_coloring]
        sel.quantity = int(quantity)
        arr = (A.SphSensorPlane * max(1, len(planes)))()
        for k, (pos, rows, cols) in enumerate(planes):
            p = np.ascontiguousarray(np.asarray(pos, np.float32).reshape(-1))
            keep.append(p)
            arr[k].positions = p.ctypes.data if p.size else None
            arr[k].rows, arr[k].cols = int(rows), int(cols)
        sel.num_planes = len(planes)
        sel.planes = arr
        if boundary == "triangle_mesh":
            from .formats import render_meshes as _rm
            sel.boundary_visualization = A.BOUNDARY_TRIANGLE_MESH
            sel.boundary_mesh_coloring = {"original": A.MESH_ORIGINAL, "uniform": A.MESH_UNIFORM,
                                          "id": A.MESH_BOUNDARY_ID}[boundary_coloring]
            sel.render_meshes = _rm(render_meshes or [], keep)
        else:
            sel.boundary_coloring = A.COLORING_ID if boundary_coloring == "id" else A.COLORING_UNIFORM
        if render_mesh_ids is not None:
            ids = np.ascontiguousarray(render_mesh_ids, np.uint32)
            keep.append(ids)
            sel.render_mesh_ids = ids.ctypes.data
        out = C.c_void_p()
        A.check(self._L.sph_encode_time_step_info(self._h, C.byref(sel), C.byref(out)))
        return _bytes(out)

    def volume_map_samples(self, bi: int):
        n = self.n
        has = np.zeros(n, np.uint8)
        xb, vb, vol = np.zeros(3 * n), np.zeros(3 * n), np.zeros(n)
        A.check(self._L.sph_get_volume_map_samples(self._h, bi, has, xb, vb, vol))
        return has.astype(bool), xb.reshape(n, 3), vb.reshape(n, 3), vol

    def rigid_state(self, bi: int) -> np.ndarray:
        out = np.zeros(19)
        A.check(self._L.sph_get_rigid_state(self._h, bi, out))
        return out

    def set_rigid_state(self, bi: int, state19):
        A.check(self._L.sph_set_rigid_state(self._h, bi, np.ascontiguousarray(state19, np.float64)))

    def hash_collisions(self) -> int:
        out = C.c_uint64()
        A.check(self._L.sph_hash_collisions(self._h, C.byref(out)))
        return out.value

    # ---- instrumentation -----------------------------------------------------------
    def launch_count(self) -> int:
        out = C.c_uint64()
        A.check(self._L.sph_launch_count(self._h, C.byref(out)))
        return out.value

    def set_profiling(self, enabled: bool):
        A.check(self._L.sph_set_profiling(self._h, 1 if enabled else 0))

    def kernel_time(self, name: str):
        ms, cnt = C.c_double(), C.c_uint64()
        rc = self._L.sph_kernel_time(self._h, name.encode(), C.byref(ms), C.byref(cnt))
        if rc:
            return None
        return ms.value, cnt.value

    def device_bytes(self) -> int:
        out = C.c_size_t()
        A.check(self._L.sph_device_bytes(self._h, C.byref(out)))
        return out.value

    def set_step_graphs(self, chunk_steps: int):
        """Graph-captured stepping in chunks of `chunk_steps` (0: per-step path)."""
        A.check(self._L.sph_set_step_graphs(self._h, int(chunk_steps)))

    def graph_replays(self) -> int:
        out = C.c_uint64()
        A.check(self._L.sph_graph_replays(self._h, C.byref(out)))
        return out.value

    def tuning(self) -> dict:
        """Result-invariant launch parameters of the neighbor passes."""
        t = A.SphTuning()
        A.check(self._L.sph_get_tuning(self._h, C.byref(t)))
        return {"gather_batch": t.gather_batch, "halo_stage": t.halo_stage, "sweep_stage": t.sweep_stage}

    def set_tuning(self, gather_batch: int, halo_stage: int, sweep_stage: int | None = None):
        """sweep_stage None keeps the current staging capacity of the IISPH sweep passes."""
        if sweep_stage is None:
            sweep_stage = self.tuning()["sweep_stage"]
        t = A.SphTuning(int(gather_batch), int(halo_stage), int(sweep_stage))
        A.check(self._L.sph_set_tuning(self._h, C.byref(t)))

    def autotune(self, steps: int = 5) -> dict:
        """Times each candidate tuning on a clone, applies the fastest and
        returns it with its milliseconds per step; this system does not step."""
        t, ms = A.SphTuning(), C.c_double()
        A.check(self._L.sph_autotune(self._h, int(steps), C.byref(t), C.byref(ms)))
        return {"gather_batch": t.gather_batch, "halo_stage": t.halo_stage, "sweep_stage": t.sweep_stage,
                "ms_per_step": ms.value}


# ---- per-trait shims ------------------------------------------------------------------
def find_samples(search_range, positions, samples, device=0):
    """NeighborSearch::find_samples (SpatialHashing) on the GPU -> (offsets, indices)."""
    L = A.load()
    pos = np.ascontiguousarray(positions, np.float64).reshape(-1, 3)
    smp = np.ascontiguousarray(samples, np.float64).reshape(-1, 3)
    total = C.c_size_t()
    rc = L.sph_spatial_hashing_find_samples(float(search_range), pos.shape[0], pos.ravel(),
                                            smp.shape[0], smp.ravel(), None, None, 0,
                                            C.byref(total), device)
    A.check(rc, allow=(A.SPH_ERR_CAPACITY,))
    off = np.zeros(pos.shape[0] + 1, np.uint64)
    idx = np.zeros(max(total.value, 1), np.uint32)
    A.check(L.sph_spatial_hashing_find_samples(float(search_range), pos.shape[0], pos.ravel(),
                                               smp.shape[0], smp.ravel(),
                                               off.ctypes.data_as(C.c_void_p),
                                               idx.ctypes.data_as(C.c_void_p), idx.size,
                                               C.byref(total), device))
    return off, idx[:total.value]


def kernel_function(r, h, precision="f32", device=0):
    L = A.load()
    rr = np.ascontiguousarray(r, np.float64).reshape(-1, 3)
    out = np.zeros(rr.shape[0])
    A.check(L.sph_kernel_function(rr.shape[0], rr.ravel(), float(h), out,
                                  A.F64 if precision == "f64" else A.F32, device))
    return out


def kernel_gradient(r, h, precision="f32", device=0):
    L = A.load()
    rr = np.ascontiguousarray(r, np.float64).reshape(-1, 3)
    out = np.zeros(3 * rr.shape[0])
    A.check(L.sph_kernel_gradient(rr.shape[0], rr.ravel(), float(h), out,
                                  A.F64 if precision == "f64" else A.F32, device))
    return out.reshape(-1, 3)
