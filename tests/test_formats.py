"""Checkpoint (RON / bincode) and recording-frame (bincode) formats.

The reference's serializers are the ron 0.12 and bincode 2.0 crates, which
cannot run here (no Rust toolchain). The encoders are therefore pinned to
the published encodings, restated independently below: byte strings and
text derived by hand for the reference's own checkpoint test values
(simulation_lib/src/sph/mod.rs:1080-1125,
simulation_lib/tests/sph/boundary_handling/mod.rs:203-245), a separate
bincode reader in this file for larger frames, and Rust's float `Display`
rule (shortest round-trip digits, positional) checked against Python's
shortest repr. These run on the CPU: the format code is host-only.
"""
import math
import struct

import numpy as np
import pytest

from sphgpu import _capi as A
from sphgpu import formats as F


@pytest.fixture(scope="module", autouse=True)
def lib():
    A.load()


def _reference_test_checkpoint(boundaries=None):
    # make_test_checkpoint, sph/mod.rs:1080-1096
    return F.Checkpoint(
        time_steps_propagated=42, current_time=12.5, fluid_id=np.array([0, 0], np.uint32),
        position=np.array([[1.0, 2.0, 3.0], [4.0, 5.0, 6.0]]), velocity=np.array([[0.1, 0.0, 0.0], [0.0, 0.0, 0.0]]),
        mass=np.array([1.0, 1.5]), boundaries=[None] if boundaries is None else boundaries)


def _f64(*xs):
    return b"".join(struct.pack("<d", x) for x in xs)


def test_reference_checkpoint_bincode_bytes():
    want = (bytes([42]) + _f64(12.5)                      # time_steps_propagated, current_time
            + bytes([2, 0, 0])                            # fluid_id: len 2, two u32 varints
            + bytes([2]) + _f64(1, 2, 3, 4, 5, 6)         # position: [[f64; 3]]
            + bytes([2]) + _f64(0.1, 0, 0, 0, 0, 0)       # velocity
            + bytes([2]) + _f64(1.0, 1.5)                 # mass
            + bytes([0]) + bytes([0])                     # integrator slots: empty
            + bytes([1, 0]))                              # dynamic_states: [None]
    assert F.encode_checkpoint(_reference_test_checkpoint(), A.FORMAT_BINCODE) == want


def test_reference_checkpoint_ron_text():
    want = ("(time_steps_propagated:42,current_time:12.5,fluid:(fluid_id:[0,0],"
            "position:[(1.0,2.0,3.0),(4.0,5.0,6.0)],velocity:[(0.1,0.0,0.0),(0.0,0.0,0.0)],"
            "mass:[1.0,1.5],integrator_position_slots:[],integrator_velocity_slots:[]),"
            "boundary:(dynamic_states:[None]))")
    assert F.encode_checkpoint(_reference_test_checkpoint(), A.FORMAT_RON).decode() == want


def _rigid(com=(7.0, 8.0, 9.0), q=(1.0, 0.0, 0.0, 0.0), v=(0, 0, 0), L=(0, 0, 0), Fo=(0, 0, 0), T=(0, 0, 0)):
    return np.array([*com, *q, *v, *L, *Fo, *T], np.float64)


def test_boundary_states_round_trip_like_the_reference_tests():
    # boundary_handling/mod.rs:203-245: [None, Some(identity at (7, 8, 9))]
    ck = _reference_test_checkpoint([None, _rigid()])
    text = F.encode_checkpoint(ck, A.FORMAT_RON).decode()
    assert text.endswith("boundary:(dynamic_states:[None,Some((center_of_mass:(7.0,8.0,9.0),"
                         "orientation:(0.0,0.0,0.0,1.0),linear_velocity:(0.0,0.0,0.0),"
                         "angular_momentum:(0.0,0.0,0.0),force:(0.0,0.0,0.0),torque:(0.0,0.0,0.0)))]))")
    back = F.decode_checkpoint(text)
    assert back.boundaries[0] is None and np.array_equal(back.boundaries[1], _rigid())
    b = F.encode_checkpoint(ck, A.FORMAT_BINCODE)
    # orientation is stored (i, j, k, w)
    assert b.endswith(bytes([2, 0, 1]) + _f64(7, 8, 9, 0, 0, 0, 1) + _f64(*([0.0] * 12)))
    back = F.decode_checkpoint(b, A.FORMAT_BINCODE)
    assert back.boundaries[0] is None and np.array_equal(back.boundaries[1], _rigid())


def _rust_display(x):
    """Rust's `{}` for f64, from Python's shortest repr digits."""
    from decimal import Decimal
    x = float(x)
    if math.isnan(x):
        return "NaN"
    if math.isinf(x):
        return "inf" if x > 0 else "-inf"
    sign, digits, exp = Decimal(repr(x)).as_tuple()
    ds = "".join(map(str, digits)).lstrip("0")
    if not ds:
        return ("-" if sign else "") + "0"
    while ds.endswith("0"):
        ds, exp = ds[:-1], exp + 1
    point = len(ds) + exp  # digits before the decimal point
    if exp >= 0:
        out = ds + "0" * exp
    elif point > 0:
        out = ds[:point] + "." + ds[point:]
    else:
        out = "0." + "0" * (-point) + ds
    return ("-" if sign else "") + out


def _ron_float(x):
    s = _rust_display(x)
    if math.isfinite(x) and float(x).is_integer():
        s += ".0"
    return s


def test_float_syntax_follows_rust_display():
    rng = np.random.default_rng(0)
    vals = [0.0, -0.0, 1.0, -1.0, 0.1, 1e-7, 1.5e-300, 5e-324, 1e21, 1.7976931348623157e308, 123456789.125,
            0.30000000000000004, 2.0 ** 60, -2.5e-5, 1e16, 1e15 + 0.5]
    vals += list(rng.normal(0, 1, 200)) + list(10.0 ** rng.uniform(-30, 30, 200) * rng.choice([-1, 1], 200))
    vals += list(rng.integers(-2 ** 62, 2 ** 62, 50).astype(np.float64))
    n = len(vals)
    ck = F.Checkpoint(0, 0.0, np.zeros(n, np.uint32), np.zeros((n, 3)), np.zeros((n, 3)), np.array(vals))
    text = F.encode_checkpoint(ck, A.FORMAT_RON).decode()
    mass = text.split("mass:[")[1].split("]")[0].split(",")
    assert mass == [_ron_float(v) for v in vals]
    back = F.decode_checkpoint(text)
    assert np.array_equal(back.mass.view(np.uint64), np.array(vals).view(np.uint64))


def _random_checkpoint(seed, n=40, slots=1, nb=3):
    rng = np.random.default_rng(seed)
    bnd = [None if k % 2 == 0 else rng.normal(size=19) for k in range(nb)]
    return F.Checkpoint(
        time_steps_propagated=int(rng.integers(0, 2 ** 63)), current_time=float(rng.uniform(0, 100)),
        fluid_id=rng.integers(0, 2 ** 32, n, dtype=np.uint64).astype(np.uint32),
        position=rng.normal(size=(n, 3)), velocity=rng.normal(size=(n, 3)), mass=rng.uniform(0, 1, n),
        integrator_position_slots=[rng.normal(size=(n, 3)) for _ in range(slots)],
        integrator_velocity_slots=[rng.normal(size=(n, 3)) for _ in range(slots)], boundaries=bnd)


def _same(a, b):
    assert a.time_steps_propagated == b.time_steps_propagated
    assert a.current_time == b.current_time
    for k in ("fluid_id", "position", "velocity", "mass"):
        assert np.array_equal(getattr(a, k), getattr(b, k)), k
    for k in ("integrator_position_slots", "integrator_velocity_slots"):
        assert len(getattr(a, k)) == len(getattr(b, k))
        for x, y in zip(getattr(a, k), getattr(b, k)):
            assert np.array_equal(x, y)
    assert len(a.boundaries) == len(b.boundaries)
    for x, y in zip(a.boundaries, b.boundaries):
        assert (x is None) == (y is None)
        if x is not None:
            assert np.array_equal(x, y)


@pytest.mark.parametrize("fmt", [A.FORMAT_RON, A.FORMAT_BINCODE])
@pytest.mark.parametrize("seed,n,slots,nb", [(1, 40, 1, 3), (2, 0, 0, 0), (3, 300, 0, 1), (4, 1, 1, 5)])
def test_round_trip_is_exact(fmt, seed, n, slots, nb):
    ck = _random_checkpoint(seed, n, slots, nb)
    _same(F.decode_checkpoint(F.encode_checkpoint(ck, fmt), fmt), ck)


def test_ron_reader_accepts_what_ron_writes_and_readers_accept():
    text = """#![enable(implicit_some)]
    // a pretty-printed state with struct names, comments and trailing commas
    SerSystemCheckpoint(
        current_time: 12.5,              /* fields in another order */
        time_steps_propagated: 4_2,
        boundary: SerBoundaryCheckpoint(dynamic_states: [
            None,
            Some(SerRigidBodyMotionCheckpoint(
                center_of_mass: (7, 8.0, 9e0), orientation: [0.0, 0.0, 0.0, 1.0],
                linear_velocity: (0.0, 0.0, 0.0), angular_momentum: (0.0, 0.0, 0.0),
                force: (0.0, 0.0, 0.0), torque: (0.0, 0.0, 0.0,),
            )),
        ]),
        fluid: SerFluidCheckpoint(
            fluid_id: [0, 0,],
            position: [(1.0, 2.0, 3.0), (4.0, 5.0, 6.0)],
            velocity: [(1e-1, 0.0, 0.0), (0.0, 0.0, -0.0)],
            mass: [1, 1.5],
            integrator_position_slots: [],
            integrator_velocity_slots: [],
            unknown_field: (ignored: [1, 2]),
        ),
    )
    """
    ck = F.decode_checkpoint(text)
    _same(ck, _reference_test_checkpoint([None, _rigid()]))


@pytest.mark.parametrize("bad", [
    "", "(", "(time_steps_propagated:1)", "(time_steps_propagated:-1,current_time:0.0)",
    "(time_steps_propagated:1,current_time:0.0,fluid:(fluid_id:[0],position:[(1.0,2.0)],velocity:[(0.0,0.0,0.0)],"
    "mass:[1.0],integrator_position_slots:[],integrator_velocity_slots:[]),boundary:(dynamic_states:[]))",
    "(time_steps_propagated:1,current_time:0.0,fluid:(fluid_id:[0,1],position:[(1.0,2.0,3.0)],velocity:[(0.0,0.0,0.0)],"
    "mass:[1.0],integrator_position_slots:[],integrator_velocity_slots:[]),boundary:(dynamic_states:[]))",
    "(time_steps_propagated:1,current_time:x)", "(time_steps_propagated:1,current_time:0.0) trailing",
])
def test_ron_errors_are_invalid_status(bad):
    with pytest.raises(A.SPHError) as e:
        F.decode_checkpoint(bad)
    assert e.value.code == A.SPH_ERR_INVALID


def test_bincode_truncation_and_oversized_lengths_are_invalid():
    b = F.encode_checkpoint(_random_checkpoint(5, 7, 1, 2), A.FORMAT_BINCODE)
    for k in range(len(b)):
        with pytest.raises(A.SPHError) as e:
            F.decode_checkpoint(b[:k], A.FORMAT_BINCODE)
        assert e.value.code == A.SPH_ERR_INVALID
    huge = bytes([1]) + _f64(0.0) + bytes([253]) + struct.pack("<Q", 2 ** 60)
    with pytest.raises(A.SPHError):
        F.decode_checkpoint(huge, A.FORMAT_BINCODE)
    bad_tag = bytes([0]) + _f64(0.0) + bytes([0, 0, 0, 0, 0, 0, 1, 7])
    with pytest.raises(A.SPHError):
        F.decode_checkpoint(bad_tag, A.FORMAT_BINCODE)


def test_varint_boundaries():
    ids = np.array([0, 250, 251, 65535, 65536, 2 ** 32 - 1], np.uint32)
    ck = F.Checkpoint(2 ** 40, 0.0, ids, np.zeros((6, 3)), np.zeros((6, 3)), np.zeros(6))
    b = F.encode_checkpoint(ck, A.FORMAT_BINCODE)
    assert b[:9] == bytes([253]) + struct.pack("<Q", 2 ** 40)
    ids_bytes = bytes([6, 0, 250, 251]) + struct.pack("<H", 251) + bytes([251]) + struct.pack("<H", 65535) \
        + bytes([252]) + struct.pack("<I", 65536) + bytes([252]) + struct.pack("<I", 2 ** 32 - 1)
    assert b[17:17 + len(ids_bytes)] == ids_bytes
    _same(F.decode_checkpoint(b, A.FORMAT_BINCODE), ck)


# ---- recording frames -----------------------------------------------------------
class _Reader:
    """bincode standard-configuration reader (spec restated for the tests)."""

    def __init__(self, b):
        self.b, self.i = b, 0

    def u8(self):
        self.i += 1
        return self.b[self.i - 1]

    def varint(self):
        t = self.u8()
        for marker, fmt, size in ((251, "<H", 2), (252, "<I", 4), (253, "<Q", 8)):
            if t == marker:
                (v,) = struct.unpack_from(fmt, self.b, self.i)
                self.i += size
                return v
        assert t < 251
        return t

    def f(self, fmt, size):
        (v,) = struct.unpack_from(fmt, self.b, self.i)
        self.i += size
        return v

    def f64(self):
        return self.f("<d", 8)

    def f32(self):
        return self.f("<f", 4)

    def vec(self, item):
        return [item() for _ in range(self.varint())]


MEASUREMENT_F64 = ("time", "density", "density_error", "kinetic_energy", "stiffness", "fluid_viscosity",
                   "boundary_viscosity", "fluid_depth", "rest_density_grid_spacing", "kernel_support_radius",
                   "time_step_size", "target_density_error")


def _decode_frame(b):
    r = _Reader(b)
    out = {"time_step_number": r.varint(), "measurement": {k: r.f64() for k in MEASUREMENT_F64}}
    out["measurement"]["solver_iterations"] = r.varint()
    for k in ("relaxation_factor", "time_step_wall_clock_time", "predicted_density_error"):
        out["measurement"][k] = r.f64()
    v3 = lambda: (r.f32(), r.f32(), r.f32())  # noqa: E731
    kind = r.varint()
    if kind == 1:
        pos = r.vec(v3)
        c = r.varint()
        col = "uniform" if c == 0 else (("id", r.vec(r.varint), r.varint()) if c == 1 else
                                        ("quantity", r.varint(), r.vec(r.f32)))
        out["fluid"] = ("samples", pos, col)
    else:
        assert kind == 2
        q = r.varint()
        planes = r.vec(lambda: (r.vec(v3), r.vec(r.f32), r.varint(), r.varint()))
        out["fluid"] = ("sensor_plane", q, planes)
    assert r.varint() == 1
    bpos = r.vec(v3)
    c = r.varint()
    out["boundary"] = (bpos, "uniform" if c == 0 else ("id", r.vec(r.varint), r.varint()))
    assert r.i == len(b)
    return out


def _measurement(seed):
    rng = np.random.default_rng(seed)
    m = {k: float(rng.normal()) for k in MEASUREMENT_F64 + ("relaxation_factor", "time_step_wall_clock_time",
                                                            "predicted_density_error")}
    m["solver_iterations"] = 300
    return m


def test_small_frame_bytes():
    m = {k: 0.0 for k in MEASUREMENT_F64 + ("relaxation_factor", "time_step_wall_clock_time",
                                            "predicted_density_error")}
    m["solver_iterations"] = 3
    b = F.encode_frame(7, m, {"kind": "samples", "positions": [[1.0, 2.0, 3.0]], "coloring": ("id", [5])},
                       {"positions": np.zeros((0, 3)), "coloring": "uniform"})
    want = (bytes([7]) + _f64(*([0.0] * 12)) + bytes([3]) + _f64(0.0, 0.0, 0.0)
            + bytes([1, 1]) + struct.pack("<3f", 1, 2, 3)          # Samples, one position
            + bytes([1, 1, 5, 5])                                  # FluidId { id: [5], max_id: 5 }
            + bytes([1, 0, 0]))                                    # boundary Samples, empty, Uniform
    assert b == want


@pytest.mark.parametrize("coloring", ["uniform", "id", "quantity"])
def test_sample_frames_decode_to_their_inputs(coloring):
    rng = np.random.default_rng(6)
    n, nb = 500, 77
    pos = rng.normal(size=(n, 3)).astype(np.float32)
    ids = rng.integers(0, 70000, n).astype(np.uint32)
    data = rng.normal(size=n).astype(np.float32)
    col = {"uniform": "uniform", "id": ("id", ids), "quantity": ("quantity", 4, data)}[coloring]
    bpos = rng.normal(size=(nb, 3)).astype(np.float32)
    bids = rng.integers(0, 3, nb).astype(np.uint32)
    b = F.encode_frame(123456, _measurement(1), {"kind": "samples", "positions": pos, "coloring": col},
                       {"positions": bpos, "coloring": ("id", bids)})
    d = _decode_frame(b)
    assert d["time_step_number"] == 123456
    assert d["measurement"] == pytest.approx(_measurement(1), abs=0)
    kind, p, c = d["fluid"]
    assert np.array_equal(np.array(p, np.float32), pos)
    if coloring == "uniform":
        assert c == "uniform"
    elif coloring == "id":
        assert c[0] == "id" and np.array_equal(c[1], ids) and c[2] == ids.max()
    else:
        assert c[0] == "quantity" and c[1] == 4 and np.array_equal(np.array(c[2], np.float32), data)
    bp, bc = d["boundary"]
    assert np.array_equal(np.array(bp, np.float32), bpos)
    assert np.array_equal(bc[1], bids) and bc[2] == bids.max()


def test_sensor_plane_frame_decodes_to_its_inputs():
    rng = np.random.default_rng(7)
    planes = []
    for rows, cols in ((4, 5), (0, 0), (16, 300)):
        planes.append((rng.normal(size=(rows * cols, 3)).astype(np.float32),
                       rng.normal(size=rows * cols).astype(np.float32), rows, cols))
    b = F.encode_frame(9, _measurement(2), {"kind": "sensor_plane", "quantity": 1, "planes": planes}, {})
    d = _decode_frame(b)
    kind, q, got = d["fluid"]
    assert kind == "sensor_plane" and q == 1 and len(got) == 3
    for (p, v, rows, cols), (gp, gv, gr, gc) in zip(planes, got):
        assert (gr, gc) == (rows, cols)
        assert np.array_equal(np.array(gp, np.float32).reshape(-1, 3), p)
        assert np.array_equal(np.array(gv, np.float32), v)


def test_frame_errors():
    with pytest.raises(A.SPHError):
        F.encode_frame(0, {}, {"kind": "samples", "positions": [[0, 0, 0]], "coloring": ("quantity", 9, [0.0])}, {})


def test_recording_writer_truncates_a_rewound_time_step(tmp_path):
    path = str(tmp_path / "rec.bin")
    w = F.RecordingWriter(path, header=b"hdr")
    for t in (1, 2, 3):
        w.append(t, bytes([t]) * t)
    w.append(2, b"again")  # a rewind: step 2 again drops 2 and 3
    assert F.read_records(path) == [b"hdr", b"\x01", b"again"]
    w.append(3, b"x")
    assert F.read_records(path) == [b"hdr", b"\x01", b"again", b"x"]
    with pytest.raises(FileExistsError):
        F.RecordingWriter(path)


def test_save_state_refuses_an_existing_file(tmp_path):
    path = str(tmp_path / "state.ron")
    F.save_state(_reference_test_checkpoint(), path)
    _same(F.load_state(path), _reference_test_checkpoint())
    with pytest.raises(FileExistsError):
        F.save_state(_reference_test_checkpoint(), path)


def _decode_boundary_meshes(b, r):
    """BoundaryVisualization at reader position: ("triangle_mesh", meshes,
    poses, coloring) or ("samples", ...) is not expected here."""
    assert r.varint() == 0
    meshes, poses = [], []
    for _ in range(r.varint()):
        nv = r.varint()
        v = np.frombuffer(b[r.i:r.i + 48 * nv], "<f8").reshape(nv, 6)
        r.i += 48 * nv
        idx = r.vec(r.varint)
        pose = np.frombuffer(b[r.i:r.i + 28], "<f4")
        r.i += 28
        meshes.append((v, idx))
        poses.append(pose)
    c = r.varint()
    col = ["original", "uniform", None][c] if c < 2 else ("id", r.vec(r.varint), r.varint())
    assert r.i == len(b)
    return meshes, poses, col


@pytest.mark.parametrize("coloring", ["original", "uniform", "id"])
def test_boundary_mesh_frames_decode_to_their_inputs(coloring):
    rng = np.random.default_rng(8)
    meshes = [(rng.normal(size=(5, 6)), rng.integers(0, 5, 9).astype(np.uint32)),
              (rng.normal(size=(0, 6)), np.zeros(0, np.uint32))]
    poses = np.array([[0, 0, 0, 0, 0, 0, 1], [1.5, -2, 0.25, 0.1, 0.2, 0.3, 0.9]], np.float32)
    ids = np.array([4, 4, 4, 9], np.uint32)
    col = {"original": "original", "uniform": "uniform", "id": ("id", ids)}[coloring]
    b = F.encode_frame(3, _measurement(3), {"kind": "samples", "positions": np.zeros((0, 3))},
                       {"kind": "triangle_mesh", "meshes": meshes, "poses": poses, "coloring": col})
    r = _Reader(b)
    r.varint()
    r.i += 12 * 8  # the measurement: 12 f64, a u32 varint, 3 f64
    r.varint()
    r.i += 3 * 8
    assert r.varint() == 1 and r.varint() == 0 and r.varint() == 0  # fluid Samples, empty, Uniform
    got, gp, gc = _decode_boundary_meshes(b, r)
    for (v, idx), (gv, gi) in zip(meshes, got):
        assert np.array_equal(gv, v) and np.array_equal(gi, idx)
    assert np.array_equal(np.array(gp), poses)
    if coloring == "id":
        assert gc[0] == "id" and np.array_equal(gc[1], ids) and gc[2] == 9
    else:
        assert gc == coloring
