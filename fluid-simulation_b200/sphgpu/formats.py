"""Checkpoint and recording formats (the readbacks either side of the step).

`Checkpoint` is SerSystemCheckpoint (simulation_lib/src/sph/mod.rs:883-915):
`encode_checkpoint` writes it as the RON text sci-phi-backend saves
(recording.rs:37-61) or as bincode bytes, `decode_checkpoint` reads either
back (the `--state` path, sph/setup/mod.rs:142-153). `encode_frame` writes a
TimeStepInfo (render_info.rs:71-106) as bincode, and `RecordingWriter` lays
frames out the way TSInfoAppender does (recording.rs:104-210). The encoders
and decoders are the library's (sph_formats.cpp); this module only moves
arrays across the C ABI.
"""
from __future__ import annotations

import ctypes as C
import os
import struct
from dataclasses import dataclass, field

import numpy as np

from . import _capi as A


@dataclass
class Checkpoint:
    """SystemCheckpoint: arrays in reference index order; `boundaries` holds
    one entry per boundary, None for a static one or the 19 doubles of
    sph_get_rigid_state (com, q as w,i,j,k, v, L, F, T) for a dynamic one."""
    time_steps_propagated: int
    current_time: float
    fluid_id: np.ndarray
    position: np.ndarray
    velocity: np.ndarray
    mass: np.ndarray
    integrator_position_slots: list = field(default_factory=list)
    integrator_velocity_slots: list = field(default_factory=list)
    boundaries: list = field(default_factory=list)


def _bytes(handle) -> bytes:
    L = A.load()
    data = C.POINTER(C.c_uint8)()
    n = C.c_size_t()
    try:
        A.check(L.sph_bytes_get(handle, C.byref(data), C.byref(n)))
        return C.string_at(data, n.value) if n.value else b""
    finally:
        L.sph_bytes_free(handle)


def _to_handle(ck: Checkpoint):
    """An owned sph_checkpoint_t built from `ck` (the caller frees it)."""
    L = A.load()
    n = int(np.asarray(ck.mass).shape[0])
    keep = []

    def arr(a, dtype, size):
        a = np.ascontiguousarray(np.asarray(a, dtype).reshape(-1))
        if a.size != size:
            raise ValueError(f"array of {a.size} values where {size} are needed")
        keep.append(a)
        return a.ctypes.data if a.size else None

    v = A.SphCheckpointView()
    v.time_steps_propagated = int(ck.time_steps_propagated)
    v.current_time = float(ck.current_time)
    v.n = n
    v.fluid_id = arr(ck.fluid_id, np.uint32, n)
    v.position = arr(ck.position, np.float64, 3 * n)
    v.velocity = arr(ck.velocity, np.float64, 3 * n)
    v.mass = arr(ck.mass, np.float64, n)
    for name, slots in (("integrator_position", ck.integrator_position_slots),
                        ("integrator_velocity", ck.integrator_velocity_slots)):
        setattr(v, name + "_slots", len(slots))
        flat = np.concatenate([np.asarray(s, np.float64).reshape(-1) for s in slots]) if slots else np.zeros(0)
        setattr(v, name, arr(flat, np.float64, 3 * n * len(slots)))
    nb = len(ck.boundaries)
    v.num_boundaries = nb
    dyn = np.array([b is not None for b in ck.boundaries], np.uint8)
    rigid = np.zeros((max(nb, 1), 19))
    for i, b in enumerate(ck.boundaries):
        if b is not None:
            rigid[i] = np.asarray(b, np.float64).reshape(19)
    v.dynamic = arr(dyn, np.uint8, nb)
    v.rigid_state = arr(rigid, np.float64, 19 * max(nb, 1))
    h = C.c_void_p()
    A.check(L.sph_checkpoint_from_view(C.byref(v), C.byref(h)))
    return h


def _from_handle(h) -> Checkpoint:
    L = A.load()
    v = A.SphCheckpointView()
    A.check(L.sph_checkpoint_view_of(h, C.byref(v)))
    n = v.n

    def get(ptr, dtype, size):
        if size == 0:
            return np.zeros(0, dtype)
        buf = (C.c_char * (size * np.dtype(dtype).itemsize)).from_address(ptr)
        return np.frombuffer(buf, dtype).copy()

    xi = get(v.integrator_position, np.float64, 3 * n * v.integrator_position_slots)
    vi = get(v.integrator_velocity, np.float64, 3 * n * v.integrator_velocity_slots)
    dyn = get(v.dynamic, np.uint8, v.num_boundaries)
    rigid = get(v.rigid_state, np.float64, 19 * v.num_boundaries).reshape(-1, 19)
    return Checkpoint(
        time_steps_propagated=v.time_steps_propagated, current_time=v.current_time,
        fluid_id=get(v.fluid_id, np.uint32, n), position=get(v.position, np.float64, 3 * n).reshape(n, 3),
        velocity=get(v.velocity, np.float64, 3 * n).reshape(n, 3), mass=get(v.mass, np.float64, n),
        integrator_position_slots=[s.reshape(n, 3) for s in np.split(xi, v.integrator_position_slots)]
        if v.integrator_position_slots else [],
        integrator_velocity_slots=[s.reshape(n, 3) for s in np.split(vi, v.integrator_velocity_slots)]
        if v.integrator_velocity_slots else [],
        boundaries=[rigid[i].copy() if dyn[i] else None for i in range(v.num_boundaries)])


def encode_checkpoint(ck: Checkpoint, fmt: int = A.FORMAT_RON) -> bytes:
    L = A.load()
    h = _to_handle(ck)
    try:
        out = C.c_void_p()
        A.check(L.sph_checkpoint_encode(h, int(fmt), C.byref(out)))
        return _bytes(out)
    finally:
        L.sph_checkpoint_free(h)


def decode_checkpoint(data: bytes, fmt: int = A.FORMAT_RON) -> Checkpoint:
    L = A.load()
    if isinstance(data, str):
        data = data.encode()
    h = C.c_void_p()
    A.check(L.sph_checkpoint_decode(data, len(data), int(fmt), C.byref(h)))
    try:
        return _from_handle(h)
    finally:
        L.sph_checkpoint_free(h)


def save_state(ck: Checkpoint, path: str):
    """recording.rs:37-61: the RON text into a new file (an existing file is
    an error, as in the reference)."""
    if os.path.exists(path):
        raise FileExistsError(path)
    parent = os.path.dirname(os.path.abspath(path))
    os.makedirs(parent, exist_ok=True)
    with open(path, "wb") as f:
        f.write(encode_checkpoint(ck, A.FORMAT_RON))


def load_state(path: str) -> Checkpoint:
    with open(path, "rb") as f:
        return decode_checkpoint(f.read(), A.FORMAT_RON)


# ---- recording frames -----------------------------------------------------------
def _measurement(m) -> A.SphMeasurement:
    if isinstance(m, A.SphMeasurement):
        return m
    out = A.SphMeasurement()
    for name, _ in A.SphMeasurement._fields_:
        setattr(out, name, m.get(name, 0))
    return out


def render_meshes(meshes, keep):
    """ctypes array of sph_render_mesh for [(vertices (n, 6), indices)]; the
    arrays are appended to `keep`."""
    arr = (A.SphRenderMesh * max(1, len(meshes)))()
    for k, (v, idx) in enumerate(meshes):
        v = np.ascontiguousarray(np.asarray(v, np.float64).reshape(-1, 6))
        idx = np.ascontiguousarray(idx, np.uint32).reshape(-1)
        keep += [v, idx]
        arr[k].vertices = v.ctypes.data if v.size else None
        arr[k].num_vertices = v.shape[0]
        arr[k].indices = idx.ctypes.data if idx.size else None
        arr[k].num_indices = idx.shape[0]
    keep.append(arr)
    return arr


def encode_frame(time_step_number: int, measurement, fluid: dict, boundary: dict) -> bytes:
    """TimeStepInfo from host arrays. `fluid` is {"kind": "samples",
    "positions", "coloring": "uniform" | ("id", ids) | ("quantity", q, data)}
    or {"kind": "sensor_plane", "quantity", "planes": [(positions, data,
    rows, cols)]}; `boundary` is {"positions", "coloring": "uniform" |
    ("id", ids)} or {"kind": "triangle_mesh", "meshes": [(vertices (n, 6),
    indices)], "poses": [translation + rotation (i, j, k, w)], "coloring":
    "original" | "uniform" | ("id", ids)}."""
    L = A.load()
    keep = []

    def ptr(a, dtype):
        a = np.ascontiguousarray(np.asarray(a, dtype).reshape(-1))
        keep.append(a)
        return a.ctypes.data if a.size else None

    f = A.SphFrameView()
    f.time_step_number = int(time_step_number)
    f.measurement = _measurement(measurement)
    if fluid["kind"] == "samples":
        f.fluid = A.FLUID_SAMPLES
        pos = np.asarray(fluid["positions"], np.float32).reshape(-1, 3)
        f.n = pos.shape[0]
        f.fluid_positions = ptr(pos, np.float32)
        col = fluid.get("coloring", "uniform")
        if col == "uniform":
            f.fluid_coloring = A.COLORING_UNIFORM
        elif col[0] == "id":
            f.fluid_coloring = A.COLORING_ID
            f.fluid_ids = ptr(col[1], np.uint32)
        else:
            f.fluid_coloring = A.COLORING_QUANTITY
            f.quantity = int(col[1])
            f.fluid_data = ptr(col[2], np.float32)
    else:
        f.fluid = A.FLUID_SENSOR_PLANE
        f.quantity = int(fluid["quantity"])
        planes = (A.SphSensorPlane * max(1, len(fluid["planes"])))()
        for k, (pos, data, rows, cols) in enumerate(fluid["planes"]):
            planes[k].positions = ptr(pos, np.float32)
            planes[k].data = ptr(data, np.float32)
            planes[k].rows, planes[k].cols = int(rows), int(cols)
        keep.append(planes)
        f.num_planes = len(fluid["planes"])
        f.planes = planes
    if boundary.get("kind", "samples") == "triangle_mesh":
        f.boundary_visualization = A.BOUNDARY_TRIANGLE_MESH
        meshes = boundary["meshes"]
        arr = render_meshes(meshes, keep)
        f.num_boundary_meshes = len(meshes)
        f.boundary_meshes = arr
        f.boundary_poses = ptr(np.asarray(boundary["poses"], np.float32).reshape(-1, 7), np.float32)
        col = boundary.get("coloring", "original")
        if col == "original":
            f.boundary_mesh_coloring = A.MESH_ORIGINAL
        elif col == "uniform":
            f.boundary_mesh_coloring = A.MESH_UNIFORM
        else:
            f.boundary_mesh_coloring = A.MESH_BOUNDARY_ID
            ids = np.asarray(col[1], np.uint32)
            f.num_mesh_ids = ids.shape[0]
            f.mesh_ids = ptr(ids, np.uint32)
    else:
        bpos = np.asarray(boundary.get("positions", np.zeros((0, 3))), np.float32).reshape(-1, 3)
        f.num_boundary_samples = bpos.shape[0]
        f.boundary_positions = ptr(bpos, np.float32)
        col = boundary.get("coloring", "uniform")
        if col == "uniform":
            f.boundary_coloring = A.COLORING_UNIFORM
        else:
            f.boundary_coloring = A.COLORING_ID
            f.boundary_ids = ptr(col[1], np.uint32)
    out = C.c_void_p()
    A.check(L.sph_frame_encode(C.byref(f), C.byref(out)))
    return _bytes(out)


class RecordingWriter:
    """TSInfoAppender (sci-phi-backend/src/recording.rs:104-210): records of a
    little-endian u64 length and the encoded bytes; a time step written again
    (after a rewind) truncates the file back to its first record."""

    def __init__(self, path: str, header: bytes | None = None):
        if os.path.exists(path):
            raise FileExistsError(path)
        os.makedirs(os.path.dirname(os.path.abspath(path)), exist_ok=True)
        self.path = path
        self.offsets: dict[int, int] = {}
        with open(path, "wb") as f:
            if header is not None:
                f.write(struct.pack("<Q", len(header)) + header)

    def append(self, time_step_number: int, frame: bytes):
        with open(self.path, "r+b") as f:
            if time_step_number in self.offsets:
                off = self.offsets[time_step_number]
                f.truncate(off)
                self.offsets = {t: o for t, o in self.offsets.items() if t < time_step_number}
            else:
                f.seek(0, os.SEEK_END)
                off = f.tell()
            f.seek(off)
            f.write(struct.pack("<Q", len(frame)) + frame)
        self.offsets[time_step_number] = off


def read_records(path: str) -> list[bytes]:
    """The length-prefixed records of a recording file, in order."""
    out = []
    with open(path, "rb") as f:
        data = f.read()
    i = 0
    while i < len(data):
        (n,) = struct.unpack_from("<Q", data, i)
        out.append(data[i + 8:i + 8 + n])
        i += 8 + n
    return out
