"""ctypes binding of the SPH oracle (test infrastructure only).

The oracle is a CPU f64 restatement of the reference's SPH step path
(SammyMcFly/fluid-simulation, ``simulation_lib``). Only ``tests/``,
``__graft_entry__.smoke()`` and ``bench.py``'s CPU-baseline legs import this
module; the engine never does.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB_PATH = os.path.join(_HERE, "liboracle.so")
_lib = None

F_POSITION, F_VELOCITY, F_ACCELERATION, F_MASS, F_VOLUME, F_PRESSURE = 0, 1, 2, 3, 4, 5
F_FLUID_ID, F_ORIGIN, F_SOURCE, F_DIAGONAL, F_SOLVER_VEL = 6, 7, 8, 9, 10
F_INTEGRATOR_POS, F_INTEGRATOR_VEL = 11, 12
_VEC_FIELDS = {F_POSITION, F_VELOCITY, F_ACCELERATION, F_SOLVER_VEL, F_INTEGRATOR_POS,
               F_INTEGRATOR_VEL}

MEASUREMENT_FIELDS = (
    "time", "density", "density_error", "kinetic_energy", "stiffness", "fluid_viscosity",
    "boundary_viscosity", "fluid_depth", "rest_density_grid_spacing", "kernel_support_radius",
    "time_step_size", "target_density_error", "solver_iterations", "relaxation_factor",
    "time_step_wall_clock_time", "predicted_density_error")


class OracleConfig(C.Structure):
    _fields_ = [
        ("integration_scheme", C.c_int), ("pressure_solver", C.c_int),
        ("boundary_handling", C.c_int), ("cfl_time_step", C.c_int),
        ("rest_density_grid_spacing", C.c_double), ("kernel_support_radius", C.c_double),
        ("disable_particles_below", C.c_double), ("fluid_viscosity", C.c_double),
        ("boundary_viscosity", C.c_double),
        ("boundary_pressure_acceleration_weighting", C.c_double),
        ("boundary_rest_volume_weighting", C.c_double), ("stiffness", C.c_double),
        ("target_density_error", C.c_double), ("relaxation_factor", C.c_double),
        ("min_diagonal_element", C.c_double), ("time_increment", C.c_double),
        ("max_time_increment", C.c_double), ("cfl_number", C.c_double),
        ("gravity_mode", C.c_int), ("gravity_center", C.c_double * 3),
        ("max_solver_iterations", C.c_uint), ("contact_fixed_sweeps", C.c_uint),
    ]


def build():
    """Compile liboracle.so with the committed Makefile."""
    subprocess.run(["make", "-s", "-C", _HERE], check=True)


def lib():
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(_LIB_PATH):
        build()
    L = C.CDLL(_LIB_PATH)
    vp, d, sz, i = C.c_void_p, C.c_double, C.c_size_t, C.c_int
    dp = np.ctypeslib.ndpointer(np.float64, flags="C")
    u64p = np.ctypeslib.ndpointer(np.uint64, flags="C")
    u32p = np.ctypeslib.ndpointer(np.uint32, flags="C")
    i64p = np.ctypeslib.ndpointer(np.int64, flags="C")
    u8p = np.ctypeslib.ndpointer(np.uint8, flags="C")
    f32p = np.ctypeslib.ndpointer(np.float32, flags="C")
    sig = {
        "oracle_system_create": (vp, [C.POINTER(OracleConfig)]),
        "oracle_destroy": (None, [vp]),
        "oracle_clone": (vp, [vp]),
        "oracle_upload_fluid": (i, [vp, sz, dp, dp, dp, u32p]),
        "oracle_add_sample_boundary": (i, [vp, sz, dp, vp]),
        "oracle_add_volume_map_boundary": (i, [vp, dp, i64p, dp, dp, i64p, dp, vp]),
        "oracle_initialize": (i, [vp]),
        "oracle_set_vm_aabb": (i, [vp, sz, dp, dp]),
        "oracle_contact_probe": (i, [vp, d, dp, dp, C.POINTER(sz), C.POINTER(C.c_uint)]),
        "oracle_sesph_probe": (i, [dp, sz, dp, dp, dp, dp, i, sz, vp, vp, vp, dp, dp, dp]),
        "oracle_nonpressure_probe": (i, [dp, i, sz, dp, dp, dp, dp, dp, i, sz, vp, vp, vp, dp, dp]),
        "oracle_iisph_terms_probe": (i, [dp, i, sz, dp, dp, dp, dp, i, sz, vp, vp, dp, dp]),
        "oracle_surfaces_from": (vp, [sz, dp, u32p, dp, d, d, d]),
        "oracle_surfaces": (vp, [vp]),
        "oracle_surfaces_count": (sz, [vp]),
        "oracle_surface_sizes": (None, [vp, sz, C.POINTER(C.c_uint32), C.POINTER(sz), C.POINTER(sz)]),
        "oracle_surface_copy": (None, [vp, sz, dp, dp, u32p]),
        "oracle_surfaces_free": (None, [vp]),
        "oracle_surface_grid": (None, [sz, dp, d, d, i64p, i64p]),
        "oracle_splitting_probe": (i, [dp, sz, dp, dp, dp, dp, dp, i, sz, vp, vp, vp, dp, dp, dp, dp]),
        "oracle_iisph_initialize_probe": (i, [sz, dp, dp, d, d, i, dp]),
        "oracle_step": (i, [vp, i]),
        "oracle_num_particles": (sz, [vp]),
        "oracle_measure": (None, [vp, dp]),
        "oracle_time": (d, [vp]),
        "oracle_steps": (C.c_ulonglong, [vp]),
        "oracle_hash_duplicates": (sz, [vp]),
        "oracle_download": (i, [vp, i, dp]),
        "oracle_quantity_at_positions": (i, [vp, i, sz, f32p, f32p]),
        "oracle_fluid_neighbor_total": (sz, [vp]),
        "oracle_fluid_neighbors": (None, [vp, u64p, u64p]),
        "oracle_boundary_neighbor_total": (sz, [vp, sz]),
        "oracle_boundary_neighbors": (None, [vp, sz, u64p, u64p]),
        "oracle_boundary_volumes": (i, [vp, sz, dp]),
        "oracle_vm_samples": (i, [vp, sz, u8p, dp, dp, dp]),
        "oracle_rigid_state": (i, [vp, sz, dp]),
        "oracle_fluid_probe": (i, [sz, dp, dp, u32p, vp, sz, vp, i, dp, dp, u32p,
                                   np.ctypeslib.ndpointer(np.uintp, flags="C")]),
        "oracle_ssb_create": (vp, []),
        "oracle_ssb_free": (None, [vp]),
        "oracle_ssb_count": (sz, [vp]),
        "oracle_ssb_len": (sz, [vp, sz]),
        "oracle_ssb_add": (i, [vp, sz, dp, vp]),
        "oracle_ssb_initialize": (None, [vp, d, d]),
        "oracle_ssb_find": (None, [vp, d, sz, dp, d]),
        "oracle_ssb_neighbor_count": (sz, [vp, sz, sz]),
        "oracle_ssb_add_force": (None, [vp, sz, dp, dp]),
        "oracle_ssb_step": (None, [vp, d]),
        "oracle_ssb_samples": (i, [vp, sz, dp, dp, dp, dp]),
        "oracle_integrate_probe": (i, [i, sz, dp, dp, dp, vp, vp, d]),
        "oracle_rigid_probe": (i, [dp, vp, i, dp, dp, i, d, i, i, dp, dp]),
        "oracle_kernel_w": (d, [d]),
        "oracle_kernel_dqw": (d, [d]),
        "oracle_kernel_function": (d, [dp, d]),
        "oracle_kernel_gradient": (None, [dp, d, dp]),
        "oracle_map_int_to_uint": (C.c_ulonglong, [i]),
        "oracle_hash": (C.c_ulonglong, [i, i, i]),
        "oracle_get_cell": (None, [dp, d, np.ctypeslib.ndpointer(np.int32, flags="C")]),
        "oracle_find_samples": (vp, [d, d, sz, dp, sz, dp]),
        "oracle_nl_total": (sz, [vp]),
        "oracle_nl_duplicates": (sz, [vp]),
        "oracle_nl_copy": (None, [vp, u64p, u64p]),
        "oracle_nl_free": (None, [vp]),
        "oracle_gauss_legendre": (i, [i, dp, dp]),
        "oracle_mesh_signed_distance": (d, [dp, sz, u32p, sz, dp]),
        "oracle_build_fields": (vp, [dp, sz, u32p, sz, d, d, i]),
        "oracle_build_sdf_only": (vp, [dp, sz, u32p, sz, d, d]),
        "oracle_fields_free": (None, [vp]),
        "oracle_field_desc": (None, [vp, i, dp, i64p]),
        "oracle_field_nodes": (None, [vp, i, dp]),
        "oracle_serendipity_function": (i, [dp, i64p, dp, dp, dp]),
        "oracle_serendipity_gradient": (i, [dp, i64p, dp, dp, dp]),
        "oracle_volume_at": (i, [dp, i64p, dp, dp, d, i, dp]),
        "oracle_rigid_body_step": (i, [dp, dp, dp, i, d, i, dp]),
        "oracle_iisph_probe": (i, [dp, dp, d, d, d, d, d, d, d, d, vp, d, i, dp]),
        "oracle_iisph_solve_probe": (i, [dp, dp, d, d, dp, d, d, d, d, d, d, d, vp, d, vp, dp]),
        "oracle_num_threads": (i, []),
        "oracle_set_num_threads": (None, [i]),
    }
    for name, (res, args) in sig.items():
        fn = getattr(L, name)
        fn.restype = res
        fn.argtypes = args
    _lib = L
    return L


def _f64(a):
    return np.ascontiguousarray(a, dtype=np.float64)


# ---- free functions -------------------------------------------------------------
def kernel_w(q):
    return lib().oracle_kernel_w(float(q))


def kernel_dqw(q):
    return lib().oracle_kernel_dqw(float(q))


def kernel_function(r, h):
    return lib().oracle_kernel_function(_f64(r), float(h))


def kernel_gradient(r, h):
    out = np.zeros(3)
    lib().oracle_kernel_gradient(_f64(r), float(h), out)
    return out


def map_int_to_uint(k):
    return lib().oracle_map_int_to_uint(int(k))


def cell_hash(k, l, m):
    return lib().oracle_hash(int(k), int(l), int(m))


def get_cell(p, cell_size):
    out = np.zeros(3, np.int32)
    lib().oracle_get_cell(_f64(p), float(cell_size), out)
    return out


def find_samples(search_range, positions, samples, cell_size=None):
    """SpatialHashing::find_samples; returns (offsets, indices, duplicates)."""
    L = lib()
    pos = _f64(positions).reshape(-1, 3)
    smp = _f64(samples).reshape(-1, 3)
    h = L.oracle_find_samples(float(search_range), float(cell_size or search_range),
                              pos.shape[0], pos.ravel(), smp.shape[0], smp.ravel())
    try:
        tot = L.oracle_nl_total(h)
        off = np.zeros(pos.shape[0] + 1, np.uint64)
        idx = np.zeros(max(tot, 1), np.uint64)
        L.oracle_nl_copy(h, off, idx)
        return off, idx[:tot], L.oracle_nl_duplicates(h)
    finally:
        L.oracle_nl_free(h)


def gauss_legendre(deg):
    x, w = np.zeros(deg), np.zeros(deg)
    lib().oracle_gauss_legendre(deg, x, w)
    return x, w


def mesh_signed_distance(verts, faces, p):
    v = _f64(verts).reshape(-1, 3)
    f = np.ascontiguousarray(faces, np.uint32).reshape(-1, 3)
    return lib().oracle_mesh_signed_distance(v.ravel(), v.shape[0], f.ravel(), f.shape[0], _f64(p))


class Field:
    """A serendipity field in dense-lattice form (NaN = absent node)."""

    def __init__(self, x_min, x_max, dx, n, nodes):
        self.x_min = np.asarray(x_min, np.float64)
        self.x_max = np.asarray(x_max, np.float64)
        self.dx = float(dx)
        self.n = np.asarray(n, np.int64)
        self.nodes = np.ascontiguousarray(nodes, np.float64).ravel()

    @property
    def desc(self):
        return np.concatenate([self.x_min, self.x_max, [self.dx]]).astype(np.float64)

    def function(self, p):
        out = np.zeros(1)
        rc = lib().oracle_serendipity_function(self.desc, self.n, self.nodes, _f64(p), out)
        return None if rc else float(out[0])

    def gradient(self, p):
        out = np.zeros(3)
        rc = lib().oracle_serendipity_gradient(self.desc, self.n, self.nodes, _f64(p), out)
        return None if rc else out


def build_fields(verts, faces, dx, r, degree=30, sdf_only=False):
    """DiscretizedBoundaryFields::new on the CPU -> (sdf Field, vm Field or None)."""
    L = lib()
    v = _f64(verts).reshape(-1, 3)
    f = np.ascontiguousarray(faces, np.uint32).reshape(-1, 3)
    if sdf_only:
        h = L.oracle_build_sdf_only(v.ravel(), v.shape[0], f.ravel(), f.shape[0], float(dx), float(r))
    else:
        h = L.oracle_build_fields(v.ravel(), v.shape[0], f.ravel(), f.shape[0], float(dx), float(r),
                                  int(degree))
    try:
        out = []
        for which in (0, 1):
            if sdf_only and which == 1:
                out.append(None)
                continue
            desc, n = np.zeros(7), np.zeros(3, np.int64)
            L.oracle_field_desc(h, which, desc, n)
            nodes = np.zeros(int(np.prod(3 * n + 1)))
            L.oracle_field_nodes(h, which, nodes)
            out.append(Field(desc[:3], desc[3:6], desc[6], n, nodes))
        return out[0], out[1]
    finally:
        L.oracle_fields_free(h)


def volume_at(sdf: Field, p, r, degree=30):
    out = np.zeros(1)
    rc = lib().oracle_volume_at(sdf.desc, sdf.n, sdf.nodes, _f64(p), float(r), int(degree), out)
    return None if rc else float(out[0])


def rigid_body_step(init32, forces, locations, dt, n_steps=1):
    out = np.zeros(19)
    fr = _f64(forces).reshape(-1, 3)
    lc = _f64(locations).reshape(-1, 3)
    lib().oracle_rigid_body_step(_f64(init32), fr.ravel(), lc.ravel(), fr.shape[0], float(dt),
                                 int(n_steps), out)
    return out


def iisph_solve_probe(pos, vel, mass, volume, acc0, dt, h, spacing, gamma_p, omega, eps, tde, bpos=None,
                      bvol=0.0, com=None):
    """IISPH::solve_and_add_acceleration for one particle and at most one
    boundary sample (dynamic when `com` is given). Returns pressure,
    acceleration, sweeps, predicted density error, body force, body torque."""
    out = np.zeros(12)
    keep = [None if v is None else _f64(v) for v in (bpos, com)]
    rc = lib().oracle_iisph_solve_probe(_f64(pos), _f64(vel), float(mass), float(volume), _f64(acc0), float(dt),
                                        float(h), float(spacing), float(gamma_p), float(omega), float(eps),
                                        float(tde), None if keep[0] is None else keep[0].ctypes.data, float(bvol),
                                        None if keep[1] is None else keep[1].ctypes.data, out)
    assert rc == 0
    return out[0], out[1:4], int(out[4]), out[5], out[6:9], out[9:12]


def iisph_probe(pos, vel, mass, volume, dt, h, spacing, gamma_p, omega, eps, bpos, bvol, after):
    """Single particle + one boundary sample IISPH solve; returns
    (pressure, a_ff, s_f, sweeps)."""
    out = np.zeros(4)
    keep = None if bpos is None else _f64(bpos)
    lib().oracle_iisph_probe(_f64(pos), _f64(vel), float(mass), float(volume), float(dt), float(h),
                             float(spacing), float(gamma_p), float(omega), float(eps),
                             None if keep is None else keep.ctypes.data_as(C.c_void_p),
                             float(bvol), int(after), out)
    return out[0], out[1], out[2], int(out[3])


def sesph_probe(h, spacing, stiffness, weighting, pos, mass, vol, acc=None, fluid_neighbors=True,
                boundary_pos=None, boundary_vol=None, body_com=None):
    """SESPH pressure and pressure acceleration on given fluid volumes (the
    setting of the reference's SESPH unit tests): (pressure[n], acc[n,3],
    body force[3], body torque[3])."""
    pos = _f64(pos).reshape(-1, 3)
    n = pos.shape[0]
    acc = np.zeros((n, 3)) if acc is None else _f64(acc).reshape(-1, 3)
    bp = None if boundary_pos is None else _f64(boundary_pos).reshape(-1, 3)
    nb = 0 if bp is None else bp.shape[0]
    bv = None if boundary_vol is None else _f64(boundary_vol)
    com = None if body_com is None else _f64(body_com)
    p, a, ft = np.zeros(n), np.zeros(3 * n), np.zeros(6)
    lib().oracle_sesph_probe(_f64([h, spacing, stiffness, weighting]), n, pos.ravel(), _f64(mass), _f64(vol),
                             acc.ravel(), 1 if fluid_neighbors else 0, nb,
                             None if bp is None else bp.ctypes.data, None if bv is None else bv.ctypes.data,
                             None if com is None else com.ctypes.data, p, a, ft)
    return p, a.reshape(n, 3), ft[:3], ft[3:]


def nonpressure_probe(h, spacing, pos, vel, mass, vol, fluid_viscosity=0.0, boundary_viscosity=0.0,
                      gravity=None, viscosity=True, acc=None, fluid_neighbors=True, boundary_pos=None,
                      boundary_vol=None, body_com=None):
    """Gravity (gravity = "uniform" or a radial center) and/or viscosity
    accelerations on given fluid arrays: (acc[n,3], body force[3], torque[3])."""
    pos = _f64(pos).reshape(-1, 3)
    n = pos.shape[0]
    acc = np.zeros((n, 3)) if acc is None else _f64(acc).reshape(-1, 3)
    bp = None if boundary_pos is None else _f64(boundary_pos).reshape(-1, 3)
    nb = 0 if bp is None else bp.shape[0]
    bv = None if boundary_vol is None else _f64(boundary_vol)
    com = None if body_com is None else _f64(body_com)
    radial = gravity is not None and not isinstance(gravity, str)
    center = gravity if radial else (0.0, 0.0, 0.0)
    prm = _f64([h, spacing, fluid_viscosity, boundary_viscosity, 1.0 if radial else 0.0, *center])
    which = (1 if gravity is not None else 0) | (2 if viscosity else 0)
    a, ft = np.zeros(3 * n), np.zeros(6)
    lib().oracle_nonpressure_probe(prm, which, n, pos.ravel(), _f64(vel).reshape(-1), _f64(mass), _f64(vol),
                                   acc.ravel(), 1 if fluid_neighbors else 0, nb,
                                   None if bp is None else bp.ctypes.data, None if bv is None else bv.ctypes.data,
                                   None if com is None else com.ctypes.data, a, ft)
    return a.reshape(n, 3), ft[:3], ft[3:]


def iisph_terms_probe(h, spacing, dt, weighting, which, pos, vel, mass, vol, fluid_neighbors=True,
                      boundary_pos=None, boundary_vol=None):
    """IISPH source term (which "vde" or "vp") or diagonal ("diag") on given
    arrays, vel being the predicted velocities: (s_f[n], a_ff[n])."""
    pos = _f64(pos).reshape(-1, 3)
    n = pos.shape[0]
    bp = None if boundary_pos is None else _f64(boundary_pos).reshape(-1, 3)
    nb = 0 if bp is None else bp.shape[0]
    bv = None if boundary_vol is None else _f64(boundary_vol)
    code = {"vde": 1, "vp": 2, "diag": 4}[which]
    s_f, a_ff = np.zeros(n), np.zeros(n)
    lib().oracle_iisph_terms_probe(_f64([h, spacing, dt, weighting]), code, n, pos.ravel(), _f64(vel).reshape(-1),
                                   _f64(mass), _f64(vol), 1 if fluid_neighbors else 0, nb,
                                   None if bp is None else bp.ctypes.data, None if bv is None else bv.ctypes.data,
                                   s_f, a_ff)
    return s_f, a_ff


def _meshes(m):
    L = lib()
    try:
        out = []
        for k in range(L.oracle_surfaces_count(m)):
            fid, nv, ni = C.c_uint32(), C.c_size_t(), C.c_size_t()
            L.oracle_surface_sizes(m, k, C.byref(fid), C.byref(nv), C.byref(ni))
            pos, nrm = np.zeros(3 * nv.value), np.zeros(3 * nv.value)
            idx = np.zeros(max(ni.value, 1), np.uint32)
            L.oracle_surface_copy(m, k, pos, nrm, idx)
            out.append((fid.value, pos.reshape(-1, 3), nrm.reshape(-1, 3), idx[:ni.value]))
        return out
    finally:
        L.oracle_surfaces_free(m)


def reconstruct_surfaces(positions, fluid_ids, masses, spacing, rest_volume, h):
    """Fluid::reconstruct_surfaces on given particles: [(fluid_id, positions,
    normals, indices)] in ascending fluid id."""
    pos = _f64(positions).reshape(-1, 3)
    n = pos.shape[0]
    ids = np.ascontiguousarray(fluid_ids, np.uint32).reshape(n)
    return _meshes(lib().oracle_surfaces_from(n, pos.ravel(), ids, _f64(masses).reshape(n), float(spacing),
                                              float(rest_volume), float(h)))


def surface_grid(positions, h, cube):
    pos = _f64(positions).reshape(-1, 3)
    k0, n = np.zeros(3, np.int64), np.zeros(3, np.int64)
    lib().oracle_surface_grid(pos.shape[0], pos.ravel(), float(h), float(cube), k0, n)
    return k0, n


def splitting_probe(h, spacing, dt, stiffness, weighting, pos, vel, mass, vol=None, acc=None,
                    fluid_neighbors=True, boundary_pos=None, boundary_vol=None, body_com=None):
    """SESPHwSplitting on given arrays (the predicted velocities are
    vel + dt acc): (density_pred[n], pressure[n], acc[n,3], body force, torque)."""
    pos = _f64(pos).reshape(-1, 3)
    n = pos.shape[0]
    vol = np.full(n, spacing ** 3) if vol is None else _f64(vol)
    acc = np.zeros((n, 3)) if acc is None else _f64(acc).reshape(-1, 3)
    bp = None if boundary_pos is None else _f64(boundary_pos).reshape(-1, 3)
    nb = 0 if bp is None else bp.shape[0]
    bv = None if boundary_vol is None else _f64(boundary_vol)
    com = None if body_com is None else _f64(body_com)
    rho, p, a, ft = np.zeros(n), np.zeros(n), np.zeros(3 * n), np.zeros(6)
    lib().oracle_splitting_probe(_f64([h, spacing, dt, stiffness, weighting]), n, pos.ravel(),
                                 _f64(vel).reshape(-1), _f64(mass), vol, acc.ravel(), 1 if fluid_neighbors else 0,
                                 nb, None if bp is None else bp.ctypes.data, None if bv is None else bv.ctypes.data,
                                 None if com is None else com.ctypes.data, rho, p, a, ft)
    return rho, p, a.reshape(n, 3), ft[:3], ft[3:]


def iisph_initialize_probe(s_f, a_ff, omega, eps, clamp):
    s_f, a_ff = _f64(s_f), _f64(a_ff)
    p = np.zeros(s_f.shape[0])
    lib().oracle_iisph_initialize_probe(s_f.shape[0], s_f, a_ff, float(omega), float(eps), 1 if clamp else 0, p)
    return p


def fluid_probe(positions, masses, fluid_ids=None, disable=(), drop=False, slots=None):
    """The oracle's Fluid built from positions, masses and ids, then
    resize_slots(*slots), disable(id) for each id in turn and drop_inactive.
    Returns positions, masses and ids (total length), the active and total
    lengths, the four slot-pool counts and the slot length. A disable that
    fails the reference's `id < num_active` assertion raises IndexError."""
    x = _f64(np.reshape(positions, (-1, 3)))
    n = x.shape[0]
    m = _f64(np.broadcast_to(masses, (n,)))
    fid = np.ascontiguousarray(np.zeros(n) if fluid_ids is None else fluid_ids, np.uint32)
    sl = None if slots is None else np.ascontiguousarray(slots, np.int64)
    ids = np.ascontiguousarray(disable, np.int64)
    op, om, of = np.zeros(3 * n), np.zeros(n), np.zeros(n, np.uint32)
    lens = np.zeros(7, np.uintp)
    rc = lib().oracle_fluid_probe(n, x.ravel(), m, fid, None if sl is None else sl.ctypes.data, ids.size,
                                  ids.ctypes.data if ids.size else None, int(bool(drop)), op, om, of, lens)
    if rc == 1:
        raise IndexError("Fluid::disable: id >= num_active")
    total = int(lens[1])
    return {"position": op.reshape(n, 3)[:total], "mass": om[:total], "fluid_id": of[:total],
            "len": int(lens[0]), "total_len": total, "slot_counts": [int(v) for v in lens[2:6]],
            "slot_len": int(lens[6])}


class SampleBoundaries:
    """The oracle's StaticSampleBoundary on its own (no fluid, no system):
    add static boundaries (world-frame samples) and dynamic ones (body-frame
    samples and a 32-value rigid init), then initialize, find, add_force and
    step as the reference's boundary API does."""

    def __init__(self):
        self._h = lib().oracle_ssb_create()

    def __del__(self):
        if getattr(self, "_h", None):
            lib().oracle_ssb_free(self._h)
            self._h = None

    def __len__(self):
        return lib().oracle_ssb_count(self._h)

    def add(self, samples, rigid=None):
        x = _f64(np.reshape(samples, (-1, 3)))
        keep = None if rigid is None else _f64(rigid)
        assert lib().oracle_ssb_add(self._h, x.shape[0], x.ravel(), None if keep is None else keep.ctypes.data) == 0

    def initialize(self, h, rest_volume_weighting=1.0):
        lib().oracle_ssb_initialize(self._h, float(h), float(rest_volume_weighting))

    def find_boundary_samples(self, search_range, positions, spacing):
        x = _f64(np.reshape(positions, (-1, 3)))
        lib().oracle_ssb_find(self._h, float(search_range), x.shape[0], x.ravel(), float(spacing))

    def neighbor_count(self, bi, particle):
        return lib().oracle_ssb_neighbor_count(self._h, bi, particle)

    def add_force(self, bid, force, location):
        lib().oracle_ssb_add_force(self._h, bid, _f64(force), _f64(location))

    def step(self, dt):
        lib().oracle_ssb_step(self._h, float(dt))

    def samples(self, bi):
        """(positions, velocities, volumes, center of mass or None)."""
        n = lib().oracle_ssb_len(self._h, bi)
        pos, vel, vol, com = np.zeros((n, 3)), np.zeros((n, 3)), np.zeros(n), np.zeros(3)
        dyn = lib().oracle_ssb_samples(self._h, bi, pos.reshape(-1), vel.reshape(-1), vol, com)
        return pos, vel, vol, (com if dyn else None)


def integrate_probe(scheme, position, velocity, acceleration, dt, slot_position=None, slot_velocity=None):
    """IntegrationScheme::integrate ("EulerCromer" or "TakePredicted") on the
    given (n, 3) arrays; returns position, velocity, acceleration and, for
    TakePredicted, the two integrator slots afterwards."""
    code = {"EulerCromer": 0, "TakePredicted": 1}[scheme]
    arrs = [np.array(a, np.float64, order="C").reshape(-1, 3) for a in (position, velocity, acceleration)]
    slots = [None if a is None else np.array(a, np.float64, order="C").reshape(-1, 3)
             for a in (slot_position, slot_velocity)]
    n = arrs[0].shape[0]
    assert all(a.shape[0] == n for a in arrs + [s for s in slots if s is not None])
    rc = lib().oracle_integrate_probe(code, n, *arrs, *[None if s is None else s.ctypes.data for s in slots],
                                      float(dt))
    assert rc == 0, rc
    return tuple(arrs) + ((tuple(slots),) if code == 1 else ())


def rigid_probe(init32, op, point=(0.0, 0.0, 0.0), restore=None, forces=(), locations=(),
                reset=False, dt=0.0, n_steps=0):
    """A RigidBodyMotion built from `init32`, optionally restored from a
    19-value checkpoint (com, orientation w,i,j,k, linear velocity, angular
    momentum, force, torque), given forces at locations, reset, and stepped.
    op "velocity_at_point", "world_to_local", "local_to_world" or
    "local_to_world_vector" of `point`, or "state": the checkpoint's 19
    values and the angular velocity (22)."""
    code = {"velocity_at_point": 0, "world_to_local": 1, "local_to_world": 2, "local_to_world_vector": 3,
            "state": 4}[op]
    fr = _f64(np.reshape(forces, (-1, 3)))
    lc = _f64(np.reshape(locations, (-1, 3)))
    assert fr.shape == lc.shape
    keep = None if restore is None else _f64(restore)
    assert keep is None or keep.size == 19
    out = np.zeros(22)
    rc = lib().oracle_rigid_probe(_f64(init32), None if keep is None else keep.ctypes.data, fr.shape[0],
                                  fr.ravel(), lc.ravel(), int(bool(reset)), float(dt), int(n_steps), code,
                                  _f64(point), out)
    assert rc == 0
    return out if code == 4 else out[:3]


def set_num_threads(n):
    lib().oracle_set_num_threads(int(n))


def num_threads():
    return lib().oracle_num_threads()


# ---- system ---------------------------------------------------------------------
def make_config(cfg: dict) -> OracleConfig:
    c = OracleConfig()
    for name, _ in OracleConfig._fields_:
        if name == "gravity_center":
            c.gravity_center[:] = cfg.get("gravity_center", (0.0, 0.0, 0.0))
        elif name in cfg:
            setattr(c, name, cfg[name])
    return c


class OracleSystem:
    """An f64 CPU `System<K,I,P,N,B>` restatement driven through its C API."""

    def __init__(self, cfg: dict):
        self._cfg = make_config(cfg)
        self.h = lib().oracle_system_create(C.byref(self._cfg))

    def __del__(self):
        h = getattr(self, "h", None)
        if h and _lib is not None:
            _lib.oracle_destroy(h)
            self.h = None

    def clone(self):
        o = OracleSystem.__new__(OracleSystem)
        o._cfg = self._cfg
        o.h = lib().oracle_clone(self.h)
        return o

    def upload_fluid(self, pos, vel, mass, fluid_id=None):
        pos = _f64(pos).reshape(-1, 3)
        n = pos.shape[0]
        vel = _f64(vel if vel is not None else np.zeros((n, 3))).reshape(-1, 3)
        mass = _f64(np.broadcast_to(mass, (n,)))
        fid = np.ascontiguousarray(fluid_id if fluid_id is not None else np.zeros(n), np.uint32)
        assert lib().oracle_upload_fluid(self.h, n, pos.ravel(), vel.ravel(), mass, fid) == 0

    def add_sample_boundary(self, positions, rigid=None):
        p = _f64(positions).reshape(-1, 3)
        r = None if rigid is None else _f64(rigid).ctypes.data_as(C.c_void_p)
        keep = None if rigid is None else _f64(rigid)
        if keep is not None:
            r = keep.ctypes.data_as(C.c_void_p)
        assert lib().oracle_add_sample_boundary(self.h, p.shape[0], p.ravel(), r) == 0

    def add_volume_map_boundary(self, sdf: Field, vm: Field, rigid=None):
        keep = None if rigid is None else _f64(rigid)
        r = None if keep is None else keep.ctypes.data_as(C.c_void_p)
        assert lib().oracle_add_volume_map_boundary(self.h, sdf.desc, sdf.n, sdf.nodes, vm.desc,
                                                    vm.n, vm.nodes, r) == 0

    def set_vm_aabb(self, bi, center, half_extents):
        """Body-frame mesh bounding box of volume-map boundary `bi` (enables
        its rigid-rigid contact)."""
        assert lib().oracle_set_vm_aabb(self.h, int(bi), _f64(center), _f64(half_extents)) == 0

    def reconstruct_surfaces(self):
        """Fluid::reconstruct_surfaces on the current fluid."""
        return _meshes(lib().oracle_surfaces(self.h))

    def contact_probe(self, dt, nb):
        """One contact solve on the current state, not applied:
        (force[nb,3], torque[nb,3], cells, sweeps)."""
        f, t = np.zeros(3 * nb), np.zeros(3 * nb)
        cells, its = C.c_size_t(), C.c_uint()
        assert lib().oracle_contact_probe(self.h, float(dt), f, t, C.byref(cells), C.byref(its)) == 0
        return f.reshape(nb, 3), t.reshape(nb, 3), cells.value, its.value

    def initialize(self):
        assert lib().oracle_initialize(self.h) == 0

    def step(self, n=1):
        assert lib().oracle_step(self.h, int(n)) == 0

    @property
    def n(self):
        return lib().oracle_num_particles(self.h)

    def time(self):
        return lib().oracle_time(self.h)

    def time_steps_propagated(self):
        return lib().oracle_steps(self.h)

    def hash_duplicates(self):
        return lib().oracle_hash_duplicates(self.h)

    def measurement(self) -> dict:
        out = np.zeros(16)
        lib().oracle_measure(self.h, out)
        return dict(zip(MEASUREMENT_FIELDS, out.tolist()))

    def download(self, field):
        n = self.n
        shape = (n, 3) if field in _VEC_FIELDS else (n,)
        out = np.zeros(int(np.prod(shape)))
        rc = lib().oracle_download(self.h, int(field), out)
        if rc:
            raise RuntimeError(f"oracle field {field} unavailable")
        return out.reshape(shape)

    def quantity_at_positions(self, quantity, positions):
        """ScalarQuantity `quantity` at positions (n x 3, cast to f32 like the
        reference's `&[[f32; 3]]`), f32 values."""
        pos = np.ascontiguousarray(positions, np.float32).reshape(-1, 3)
        out = np.zeros(pos.shape[0], np.float32)
        if lib().oracle_quantity_at_positions(self.h, int(quantity), pos.shape[0], pos.reshape(-1), out):
            raise ValueError(f"unknown quantity {quantity}")
        return out

    def fluid_neighbors(self):
        tot = lib().oracle_fluid_neighbor_total(self.h)
        off = np.zeros(self.n + 1, np.uint64)
        idx = np.zeros(max(tot, 1), np.uint64)
        lib().oracle_fluid_neighbors(self.h, off, idx)
        return off, idx[:tot]

    def boundary_neighbors(self, bi):
        tot = lib().oracle_boundary_neighbor_total(self.h, bi)
        off = np.zeros(self.n + 1, np.uint64)
        idx = np.zeros(max(tot, 1), np.uint64)
        lib().oracle_boundary_neighbors(self.h, bi, off, idx)
        return off, idx[:tot]

    def boundary_volumes(self, bi, nb):
        out = np.zeros(nb)
        assert lib().oracle_boundary_volumes(self.h, bi, out) == 0
        return out

    def vm_samples(self, bi):
        n = self.n
        has = np.zeros(n, np.uint8)
        xb, vb, vol = np.zeros(3 * n), np.zeros(3 * n), np.zeros(n)
        assert lib().oracle_vm_samples(self.h, bi, has, xb, vb, vol) == 0
        return has.astype(bool), xb.reshape(n, 3), vb.reshape(n, 3), vol

    def rigid_state(self, bi):
        out = np.zeros(19)
        if lib().oracle_rigid_state(self.h, bi, out):
            return None
        return out
