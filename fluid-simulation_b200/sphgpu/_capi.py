"""ctypes declarations of the engine's C ABI (include/sphgpu.h).

The shared library is built in-tree (`libsphgpu.so` next to this file). There
is no fallback: if the library or a CUDA device is missing, the calls fail
with an explicit error.
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "libsphgpu.so")

# status codes
SPH_OK, SPH_ERR_INVALID, SPH_ERR_OOM, SPH_ERR_CUDA = 0, 1, 2, 3
SPH_NOT_CONVERGED, SPH_ERR_STATE, SPH_ERR_CAPACITY, SPH_PENDING = 4, 5, 6, 7

# procedure variants
CUBIC_BSPLINE_3D = 0
EULER_CROMER, TAKE_PREDICTED = 0, 1
SESPH, SESPH_W_SPLITTING, IISPH, IISPH_W_OST = 0, 1, 2, 3
SPATIAL_HASHING = 0
STATIC_SAMPLE_BOUNDARY, VOLUME_MAP_BOUNDARY = 0, 1
F32, F64 = 0, 1
GRAVITY_UNIFORM, GRAVITY_RADIAL = 0, 1

# download fields
FIELD_POSITION, FIELD_VELOCITY, FIELD_ACCELERATION = 0, 1, 2
FIELD_MASS, FIELD_VOLUME, FIELD_PRESSURE, FIELD_FLUID_ID = 3, 4, 5, 6
FIELD_SOURCE_TERM, FIELD_DIAGONAL, FIELD_PREDICTED_VELOCITY = 8, 9, 10
FIELD_INTEGRATOR_POSITION, FIELD_INTEGRATOR_VELOCITY = 11, 12
VECTOR_FIELDS = {FIELD_POSITION, FIELD_VELOCITY, FIELD_ACCELERATION, FIELD_PREDICTED_VELOCITY,
                 FIELD_INTEGRATOR_POSITION, FIELD_INTEGRATOR_VELOCITY}

# scalar quantities (render_info ScalarQuantity)
Q_SPEED, Q_VOLUME, Q_DENSITY, Q_DENSITY_ERROR, Q_PRESSURE, Q_KINETIC_ENERGY = range(6)


class SphConfig(C.Structure):
    _fields_ = [
        ("kernel_fn", C.c_int), ("integration_scheme", C.c_int), ("pressure_solver", C.c_int),
        ("neighbor_search", C.c_int), ("boundary_handling", C.c_int), ("precision", C.c_int),
        ("cfl_time_step", C.c_int), ("gravity_mode", C.c_int),
        ("rest_density_grid_spacing", C.c_double), ("kernel_support_radius", C.c_double),
        ("disable_particles_below", C.c_double), ("fluid_viscosity", C.c_double),
        ("boundary_viscosity", C.c_double),
        ("boundary_pressure_acceleration_weighting", C.c_double),
        ("boundary_rest_volume_weighting", C.c_double), ("stiffness", C.c_double),
        ("target_density_error", C.c_double), ("relaxation_factor", C.c_double),
        ("min_diagonal_element", C.c_double), ("time_increment", C.c_double),
        ("max_time_increment", C.c_double), ("cfl_number", C.c_double),
        ("gravity_center", C.c_double * 3), ("max_solver_iterations", C.c_uint32),
        ("neighbor_capacity", C.c_uint32), ("device", C.c_int),
    ]


class SphRigidInit(C.Structure):
    _fields_ = [
        ("mass", C.c_double), ("inertia_body", C.c_double * 9),
        ("inertia_inv_body", C.c_double * 9), ("center_of_mass", C.c_double * 3),
        ("orientation", C.c_double * 4), ("linear_velocity", C.c_double * 3),
        ("angular_velocity", C.c_double * 3),
    ]


class SphGridDesc(C.Structure):
    _fields_ = [("x_min", C.c_double * 3), ("x_max", C.c_double * 3), ("dx", C.c_double),
                ("n", C.c_int64 * 3)]


class SphMeasurement(C.Structure):
    _fields_ = [
        ("time", C.c_double), ("density", C.c_double), ("density_error", C.c_double),
        ("kinetic_energy", C.c_double), ("stiffness", C.c_double),
        ("fluid_viscosity", C.c_double), ("boundary_viscosity", C.c_double),
        ("fluid_depth", C.c_double), ("rest_density_grid_spacing", C.c_double),
        ("kernel_support_radius", C.c_double), ("time_step_size", C.c_double),
        ("target_density_error", C.c_double), ("solver_iterations", C.c_uint32),
        ("relaxation_factor", C.c_double), ("time_step_wall_clock_time", C.c_double),
        ("predicted_density_error", C.c_double),
    ]


class SphStepStats(C.Structure):
    _fields_ = [("particles", C.c_uint64), ("solver_iterations", C.c_uint32),
                ("solver_iterations_first", C.c_uint32), ("max_neighbors", C.c_uint32),
                ("max_boundary_neighbors", C.c_uint32), ("predicted_density_error", C.c_double),
                ("time_increment", C.c_double), ("average_density", C.c_double),
                ("not_converged", C.c_int)]


class SphServerConfig(C.Structure):
    _fields_ = [("device", C.c_int), ("memory_budget_bytes", C.c_uint64), ("max_active", C.c_uint32),
                ("chunk_steps", C.c_uint32)]


class SphSampleSet(C.Structure):
    _fields_ = [("count", C.c_size_t), ("positions", C.c_void_p), ("rigid", C.POINTER(SphRigidInit))]


class SphVolumeMapSet(C.Structure):
    _fields_ = [("sdf", C.POINTER(SphGridDesc)), ("sdf_nodes", C.c_void_p), ("vm", C.POINTER(SphGridDesc)),
                ("vm_nodes", C.c_void_p), ("rigid", C.POINTER(SphRigidInit))]


class SphSceneRequest(C.Structure):
    _fields_ = [("config", SphConfig), ("n", C.c_size_t), ("position", C.c_void_p), ("velocity", C.c_void_p),
                ("mass", C.c_void_p), ("fluid_id", C.c_void_p), ("num_sample_sets", C.c_size_t),
                ("sample_sets", C.POINTER(SphSampleSet)), ("num_volume_maps", C.c_size_t),
                ("volume_maps", C.POINTER(SphVolumeMapSet)), ("steps", C.c_uint32), ("keep_state", C.c_int)]


class SphSceneResult(C.Structure):
    _fields_ = [("status", C.c_int), ("steps", C.c_uint64), ("time", C.c_double), ("particles", C.c_uint64),
                ("measurement", SphMeasurement), ("submit_s", C.c_double), ("start_s", C.c_double),
                ("finish_s", C.c_double), ("device_bytes_reserved", C.c_uint64),
                ("graph_replays", C.c_uint64), ("kernel_launches", C.c_uint64)]


class SphTuning(C.Structure):
    _fields_ = [("gather_batch", C.c_uint32), ("halo_stage", C.c_uint32), ("sweep_stage", C.c_uint32)]


class SphServerStats(C.Structure):
    _fields_ = [(k, C.c_uint64) for k in (
        "submitted", "completed", "queued", "active", "peak_active", "budget_bytes", "reserved_bytes",
        "peak_reserved_bytes", "graph_replays", "kernel_launches")]


# checkpoint / recording formats
FORMAT_RON, FORMAT_BINCODE = 0, 1
FLUID_TRIANGLE_MESH, FLUID_SAMPLES, FLUID_SENSOR_PLANE = 0, 1, 2
COLORING_UNIFORM, COLORING_ID, COLORING_QUANTITY = 0, 1, 2


class SphCheckpointView(C.Structure):
    _fields_ = [
        ("time_steps_propagated", C.c_uint64), ("current_time", C.c_double), ("n", C.c_size_t),
        ("fluid_id", C.c_void_p), ("position", C.c_void_p), ("velocity", C.c_void_p), ("mass", C.c_void_p),
        ("integrator_position_slots", C.c_size_t), ("integrator_position", C.c_void_p),
        ("integrator_velocity_slots", C.c_size_t), ("integrator_velocity", C.c_void_p),
        ("num_boundaries", C.c_size_t), ("dynamic", C.c_void_p), ("rigid_state", C.c_void_p),
    ]


BOUNDARY_SAMPLES, BOUNDARY_TRIANGLE_MESH = 0, 1
MESH_ORIGINAL, MESH_UNIFORM, MESH_BOUNDARY_ID = 0, 1, 2


class SphRenderMesh(C.Structure):
    _fields_ = [("vertices", C.c_void_p), ("num_vertices", C.c_size_t), ("indices", C.c_void_p),
                ("num_indices", C.c_size_t)]


class SphSensorPlane(C.Structure):
    _fields_ = [("positions", C.c_void_p), ("data", C.c_void_p), ("rows", C.c_size_t), ("cols", C.c_size_t)]


class SphFrameSelector(C.Structure):
    _fields_ = [
        ("fluid", C.c_int), ("fluid_coloring", C.c_int), ("quantity", C.c_int),
        ("num_planes", C.c_size_t), ("planes", C.POINTER(SphSensorPlane)),
        ("boundary_coloring", C.c_int), ("render_mesh_ids", C.c_void_p),
        ("boundary_visualization", C.c_int), ("boundary_mesh_coloring", C.c_int),
        ("render_meshes", C.POINTER(SphRenderMesh)),
    ]


class SphFrameView(C.Structure):
    _fields_ = [
        ("time_step_number", C.c_uint64), ("measurement", SphMeasurement),
        ("fluid", C.c_int), ("fluid_coloring", C.c_int), ("quantity", C.c_int),
        ("n", C.c_size_t), ("fluid_positions", C.c_void_p), ("fluid_ids", C.c_void_p), ("fluid_data", C.c_void_p),
        ("num_planes", C.c_size_t), ("planes", C.POINTER(SphSensorPlane)),
        ("boundary_coloring", C.c_int), ("num_boundary_samples", C.c_size_t),
        ("boundary_positions", C.c_void_p), ("boundary_ids", C.c_void_p),
        ("meshes", C.c_void_p), ("max_fluid_id", C.c_uint32),
        ("boundary_visualization", C.c_int), ("boundary_mesh_coloring", C.c_int),
        ("num_boundary_meshes", C.c_size_t), ("boundary_meshes", C.POINTER(SphRenderMesh)),
        ("boundary_poses", C.c_void_p), ("num_mesh_ids", C.c_size_t), ("mesh_ids", C.c_void_p),
    ]


class SPHError(RuntimeError):
    def __init__(self, code, msg):
        super().__init__(f"sphgpu error {code}: {msg}")
        self.code = code


# every exported symbol: name -> (restype, argtypes)
_vp = C.c_void_p
_dp = np.ctypeslib.ndpointer(np.float64, flags="C")
_fp = np.ctypeslib.ndpointer(np.float32, flags="C")
_u32p = np.ctypeslib.ndpointer(np.uint32, flags="C")
_u64p = np.ctypeslib.ndpointer(np.uint64, flags="C")
_u8p = np.ctypeslib.ndpointer(np.uint8, flags="C")
_sz = C.c_size_t
SIGNATURES = {
    "sph_config_default": (None, [C.POINTER(SphConfig)]),
    "sph_create": (C.c_int, [C.POINTER(SphConfig), C.POINTER(_vp)]),
    "sph_destroy": (None, [_vp]),
    "sph_clone": (C.c_int, [_vp, C.POINTER(_vp)]),
    "sph_upload_fluid": (C.c_int, [_vp, _sz, _dp, _dp, _dp, _u32p]),
    "sph_add_sample_boundary": (C.c_int, [_vp, _sz, _dp, C.POINTER(SphRigidInit), C.POINTER(C.c_int)]),
    "sph_add_volume_map_boundary": (C.c_int, [_vp, C.POINTER(SphGridDesc), _dp, C.POINTER(SphGridDesc),
                                              _dp, C.POINTER(SphRigidInit), C.POINTER(C.c_int)]),
    "sph_initialize": (C.c_int, [_vp]),
    "sph_step": (C.c_int, [_vp, C.c_uint32]),
    "sph_step_host": (C.c_int, [_vp, C.c_uint32, _vp, _vp, _vp, _vp]),
    "sph_get_stream": (C.c_int, [_vp, C.POINTER(_vp)]),
    "sph_get_step_stats": (C.c_int, [_vp, C.POINTER(SphStepStats)]),
    "sph_time": (C.c_int, [_vp, C.POINTER(C.c_double)]),
    "sph_time_steps_propagated": (C.c_int, [_vp, C.POINTER(C.c_uint64)]),
    "sph_take_measurement": (C.c_int, [_vp, C.POINTER(SphMeasurement)]),
    "sph_num_particles": (C.c_int, [_vp, C.POINTER(_sz)]),
    "sph_get_fluid_ids": (C.c_int, [_vp, _u32p]),
    "sph_get_fluid_pos": (C.c_int, [_vp, _fp]),
    "sph_get_quantity_of_fluid_samples": (C.c_int, [_vp, C.c_int, _fp]),
    "sph_get_quantity_at_positions": (C.c_int, [_vp, C.c_int, _sz, _fp, _fp]),
    "sph_download": (C.c_int, [_vp, C.c_int, _dp]),
    "sph_get_fluid_neighbors": (C.c_int, [_vp, _vp, _vp, _sz, C.POINTER(_sz)]),
    "sph_get_boundary_neighbors": (C.c_int, [_vp, C.c_int, _vp, _vp, _sz, C.POINTER(_sz)]),
    "sph_get_boundary_volumes": (C.c_int, [_vp, C.c_int, _dp]),
    "sph_get_volume_map_samples": (C.c_int, [_vp, C.c_int, _u8p, _dp, _dp, _dp]),
    "sph_get_rigid_state": (C.c_int, [_vp, C.c_int, _dp]),
    "sph_set_rigid_state": (C.c_int, [_vp, C.c_int, _dp]),
    "sph_hash_collisions": (C.c_int, [_vp, C.POINTER(C.c_uint64)]),
    "sph_continue_from_checkpoint": (C.c_int, [_vp, C.c_uint64, C.c_double, _sz, _dp, _dp, _dp, _u32p,
                                               _vp, _vp]),
    "sph_spatial_hashing_find_samples": (C.c_int, [C.c_double, _sz, _dp, _sz, _dp, _vp, _vp, _sz,
                                                   C.POINTER(_sz), C.c_int]),
    "sph_spatial_hashing_find_samples_noalloc": (C.c_int, [C.c_double, _sz, _vp, _sz, _vp, _vp, _vp, _sz,
                                                           C.POINTER(_sz), C.c_int]),
    "sph_kernel_function": (C.c_int, [_sz, _dp, C.c_double, _dp, C.c_int, C.c_int]),
    "sph_kernel_gradient": (C.c_int, [_sz, _dp, C.c_double, _dp, C.c_int, C.c_int]),
    "sph_volume_map_grids": (C.c_int, [_dp, _sz, C.c_double, C.c_double, C.POINTER(SphGridDesc),
                                       C.POINTER(SphGridDesc)]),
    "sph_build_sdf_field": (C.c_int, [_dp, _sz, _u32p, _sz, C.POINTER(SphGridDesc), C.c_double, _dp,
                                      C.c_int]),
    "sph_build_volume_map_field": (C.c_int, [C.POINTER(SphGridDesc), _dp, C.POINTER(SphGridDesc),
                                             C.c_double, C.c_int, _dp, C.c_int]),
    "sph_last_error": (C.c_char_p, []),
    "sph_launch_count": (C.c_int, [_vp, C.POINTER(C.c_uint64)]),
    "sph_set_profiling": (C.c_int, [_vp, C.c_int]),
    "sph_kernel_time": (C.c_int, [_vp, C.c_char_p, C.POINTER(C.c_double), C.POINTER(C.c_uint64)]),
    "sph_device_bytes": (C.c_int, [_vp, C.POINTER(_sz)]),
    "sph_set_step_graphs": (C.c_int, [_vp, C.c_uint32]),
    "sph_graph_replays": (C.c_int, [_vp, C.POINTER(C.c_uint64)]),
    "sph_get_tuning": (C.c_int, [_vp, C.POINTER(SphTuning)]),
    "sph_set_tuning": (C.c_int, [_vp, C.POINTER(SphTuning)]),
    "sph_autotune": (C.c_int, [_vp, C.c_uint32, C.POINTER(SphTuning), C.POINTER(C.c_double)]),
    "sph_server_create": (C.c_int, [C.POINTER(SphServerConfig), C.POINTER(_vp)]),
    "sph_server_submit": (C.c_int, [_vp, C.POINTER(SphSceneRequest), C.POINTER(C.c_uint64)]),
    "sph_server_poll": (C.c_int, [_vp, C.c_uint64, C.POINTER(SphSceneResult)]),
    "sph_server_wait": (C.c_int, [_vp, C.c_uint64, C.c_double, C.POINTER(SphSceneResult)]),
    "sph_server_fetch_state": (C.c_int, [_vp, C.c_uint64, _dp, _dp]),
    "sph_server_release": (C.c_int, [_vp, C.c_uint64]),
    "sph_server_get_stats": (C.c_int, [_vp, C.POINTER(SphServerStats)]),
    "sph_server_destroy": (None, [_vp]),
    "sph_get_boundary_positions": (C.c_int, [_vp, C.c_int, _dp]),
    "sph_set_volume_map_aabb": (C.c_int, [_vp, C.c_int, _dp, _dp]),
    "sph_reconstruct_surfaces": (C.c_int, [_vp, C.POINTER(_vp)]),
    "sph_meshes_count": (C.c_int, [_vp, C.POINTER(_sz)]),
    "sph_meshes_get": (C.c_int, [_vp, _sz, C.POINTER(C.c_uint32), C.POINTER(_sz),
                                 C.POINTER(C.POINTER(C.c_double)), C.POINTER(_sz),
                                 C.POINTER(C.POINTER(C.c_uint32))]),
    "sph_meshes_free": (None, [_vp]),
    "sph_get_contact_stats": (C.c_int, [_vp, _u32p]),
    "sph_set_contact_sweeps": (C.c_int, [_vp, C.c_uint32]),
    "sph_bytes_get": (C.c_int, [_vp, C.POINTER(C.POINTER(C.c_uint8)), C.POINTER(_sz)]),
    "sph_bytes_free": (None, [_vp]),
    "sph_checkpoint_from_view": (C.c_int, [C.POINTER(SphCheckpointView), C.POINTER(_vp)]),
    "sph_checkpoint_view_of": (C.c_int, [_vp, C.POINTER(SphCheckpointView)]),
    "sph_checkpoint_free": (None, [_vp]),
    "sph_checkpoint_encode": (C.c_int, [_vp, C.c_int, C.POINTER(_vp)]),
    "sph_checkpoint_decode": (C.c_int, [C.c_char_p, _sz, C.c_int, C.POINTER(_vp)]),
    "sph_get_checkpoint": (C.c_int, [_vp, C.POINTER(_vp)]),
    "sph_restore_checkpoint": (C.c_int, [_vp, _vp]),
    "sph_frame_encode": (C.c_int, [C.POINTER(SphFrameView), C.POINTER(_vp)]),
    "sph_encode_time_step_info": (C.c_int, [_vp, C.POINTER(SphFrameSelector), C.POINTER(_vp)]),
}

_lib = None


def load():
    """Load libsphgpu.so (raises if it was not built)."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise ImportError(
            f"{LIB_PATH} is missing: build it with `make -C fluid-simulation_b200/csrc` "
            "(or __graft_entry__.build()); the engine has no CPU fallback")
    L = C.CDLL(LIB_PATH)
    for name, (res, args) in SIGNATURES.items():
        fn = getattr(L, name)
        fn.restype = res
        fn.argtypes = args
    _lib = L
    return L


def check(rc, allow=()):
    if rc == SPH_OK or rc in allow:
        return rc
    msg = load().sph_last_error()
    raise SPHError(rc, msg.decode() if msg else "")
