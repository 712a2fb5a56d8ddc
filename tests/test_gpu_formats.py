"""Checkpoints and recording frames taken from a system's device state.

The `--state` round trip (SystemCheckpoint::from_sph_system -> RON or
bincode -> SPHSystem::continue_from_checkpoint, sph/mod.rs:362-378, 849-915)
continues a run bit for bit, and a frame from sph_encode_time_step_info is
byte for byte the encoding of the system's own readbacks
(TimeStepInfo::from_system, render_info.rs:83-158).
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def A():
    from sphgpu import _capi
    _capi.load()
    return _capi


def _ost_vm_scene():
    from sphgpu import scenes
    from sphgpu.fields import build_volume_map_fields
    sc = scenes.dam_break_iisph_box(n_side=12, spacing=0.02, box=(0.6, 0.32, 0.32))
    sc.procedures = dict(sc.procedures, pressure_solver="IISPHwOST", integration_scheme="TakePredicted")
    sc.cfl_time_step = False
    sc.parameters = dict(sc.parameters, max_solver_iterations=30, time_increment=1e-3)
    verts, faces = sc.mesh
    return sc, build_volume_map_fields(verts, faces, 0.08, 0.04)


@pytest.mark.parametrize("case", ["sesph_samples_f32_ron", "ost_volume_map_f64_bincode"])
def test_state_round_trip_continues_the_run(A, tmp_path, case):
    from sphgpu import formats as F
    from sphgpu import scenes
    if case.startswith("sesph"):
        sc, fields, prec, fmt = scenes.dam_break_sesph_8k(n_side=12), None, "f32", A.FORMAT_RON
    else:
        (sc, fields), prec, fmt = _ost_vm_scene(), "f64", A.FORMAT_BINCODE
    a = scenes.build_system(sc, precision=prec, fields=fields)
    a.step_forward_in_time(12)
    ck = a.get_checkpoint()
    assert ck.time_steps_propagated == 12
    assert np.array_equal(ck.position, a.download(A.FIELD_POSITION))
    assert np.array_equal(ck.velocity, a.download(A.FIELD_VELOCITY))
    assert np.array_equal(ck.fluid_id, a.get_fluid_ids())
    assert len(ck.integrator_position_slots) == (1 if case.startswith("ost") else 0)
    path = tmp_path / "state.bin"
    path.write_bytes(F.encode_checkpoint(ck, fmt))
    b = scenes.build_system(sc, precision=prec, fields=fields)
    b.restore_checkpoint(F.decode_checkpoint(path.read_bytes(), fmt))
    assert b.time_steps_propagated() == 12
    a.step_forward_in_time(15)
    b.step_forward_in_time(15)
    for f in (A.FIELD_POSITION, A.FIELD_VELOCITY, A.FIELD_PRESSURE):
        assert np.array_equal(a.download(f), b.download(f)), f
    a.close()
    b.close()


def test_rigid_states_restore_like_the_reference(A):
    """Dynamic bodies get their saved state back. As in the reference, the
    saved force and torque stay and the update after the restore adds the
    fluid's reaction again (RigidBodyMotion::restore_from_checkpoint,
    rigid_body_motion.rs:214-222, then System::update): restored from the
    state they were saved in, they hold twice the saved values. A checkpoint
    whose boundary count differs leaves the bodies as they are
    (static_sample_boundary.rs:263-273)."""
    from sphgpu import scenes
    sc = scenes.floating_cube_scene()
    a = scenes.build_system(sc)
    a.step_forward_in_time(30)
    ck = a.get_checkpoint()
    assert ck.boundaries[0] is None and ck.boundaries[1] is not None
    saved = ck.boundaries[1]
    assert np.abs(saved[13:16]).max() > 0  # a reaction force is pending
    b = scenes.build_system(sc)
    b.restore_checkpoint(ck)
    got = b.get_checkpoint().boundaries[1]
    assert np.array_equal(got[:13], saved[:13])
    assert np.allclose(got[13:19], 2.0 * saved[13:19], rtol=1e-6, atol=1e-12)
    assert np.array_equal(b.download(A.FIELD_POSITION), a.download(A.FIELD_POSITION))
    c = scenes.build_system(sc)
    before = c.get_checkpoint().boundaries[1]
    ck.boundaries = [None]
    c.restore_checkpoint(ck)
    assert np.array_equal(c.get_checkpoint().boundaries[1][:13], before[:13])
    for s in (a, b, c):
        s.close()


def _frame_from_readbacks(g, fluid, boundary_ids=None):
    from sphgpu import formats as F
    bpos, bcol = np.zeros((0, 3)), "uniform"
    if g._cfg.boundary_handling == 0:
        parts = [g.boundary_positions(bi, nb) for bi, (_, nb) in enumerate(g._boundaries)]
        bpos = np.concatenate(parts).astype(np.float32)
        if boundary_ids is not None:
            bcol = ("id", np.concatenate([np.full(nb, boundary_ids[bi], np.uint32)
                                          for bi, (_, nb) in enumerate(g._boundaries)]))
    return F.encode_frame(g.time_steps_propagated(), g.take_measurement(), fluid,
                          {"positions": bpos, "coloring": bcol})


def test_sample_frames_equal_the_encoded_readbacks(A):
    from sphgpu import scenes
    sc = scenes.floating_cube_scene()
    g = scenes.build_system(sc)
    g.step_forward_in_time(20)
    pos = g.get_fluid_pos()
    ids = [3, 9]
    got = g.encode_time_step_info("samples", "uniform")
    assert got == _frame_from_readbacks(g, {"kind": "samples", "positions": pos})
    got = g.encode_time_step_info("samples", "id", boundary_coloring="id", render_mesh_ids=ids)
    assert got == _frame_from_readbacks(g, {"kind": "samples", "positions": pos,
                                            "coloring": ("id", g.get_fluid_ids())}, boundary_ids=ids)
    for q in (A.Q_SPEED, A.Q_PRESSURE):
        got = g.encode_time_step_info("samples", "quantity", quantity=q)
        data = g.get_quantity_of_fluid_samples(q)
        assert got == _frame_from_readbacks(g, {"kind": "samples", "positions": pos,
                                                "coloring": ("quantity", q, data)})
    g.close()


def test_sensor_plane_frames_equal_the_encoded_readbacks(A):
    from sphgpu import scenes
    sc, fields = _ost_vm_scene()
    g = scenes.build_system(sc, fields=fields)
    g.step_forward_in_time(10)
    u = np.linspace(-0.3, 0.3, 30, dtype=np.float32)
    w = np.linspace(-0.16, 0.16, 20, dtype=np.float32)
    U, W = np.meshgrid(u, w, indexing="ij")
    p1 = np.stack([U.ravel(), np.zeros(U.size, np.float32), W.ravel()], 1)
    p2 = np.stack([U.ravel(), W.ravel(), np.full(U.size, -0.1, np.float32)], 1)
    planes = [(p1, 30, 20), (p2, 30, 20), (np.zeros((0, 3), np.float32), 0, 0)]
    for q in (A.Q_VOLUME, A.Q_DENSITY):
        got = g.encode_time_step_info("sensor_plane", quantity=q, planes=planes, boundary_coloring="id")
        want_planes = [(p, g.get_quantity_at_positions(q, p), r, c) for p, r, c in planes]
        # a volume-map system has no boundary samples: an empty, uniform set
        assert got == _frame_from_readbacks(g, {"kind": "sensor_plane", "quantity": q, "planes": want_planes})
    g.close()


def test_boundary_mesh_frame_carries_the_device_poses(A):
    """BoundaryVisualization::TriangleMesh (static_sample_boundary.rs:194-219):
    the caller's render meshes, identity for the static container and the
    rigid state's pose (f32 translation, rotation as i, j, k, w) for the
    body; BoundaryId coloring lists each boundary's id once per sample."""
    from sphgpu import scenes
    from test_formats import _Reader, _decode_boundary_meshes
    sc = scenes.floating_cube_scene()
    g = scenes.build_system(sc)
    g.step_forward_in_time(7)
    rng = np.random.default_rng(2)
    meshes = [(rng.normal(size=(8, 6)), rng.integers(0, 8, 12).astype(np.uint32)) for _ in range(2)]
    frame = g.encode_time_step_info("samples", boundary="triangle_mesh", render_meshes=meshes,
                                    boundary_coloring="id", render_mesh_ids=[5, 11])
    r = _Reader(frame)
    r.varint()
    r.i += 12 * 8
    r.varint()
    r.i += 3 * 8
    assert r.varint() == 1  # fluid Samples
    n = r.varint()
    r.i += 12 * n
    assert r.varint() == 0  # uniform coloring
    got, poses, col = _decode_boundary_meshes(frame, r)
    for (v, idx), (gv, gi) in zip(meshes, got):
        assert np.array_equal(gv, v) and np.array_equal(gi, idx)
    assert np.array_equal(poses[0], np.array([0, 0, 0, 0, 0, 0, 1], np.float32))
    st = g.rigid_state(1)
    want = np.array([st[0], st[1], st[2], st[4], st[5], st[6], st[3]]).astype(np.float32)
    assert np.array_equal(poses[1], want)
    counts = [nb for _, nb in g._boundaries]
    assert col[0] == "id" and np.array_equal(col[1], np.repeat([5, 11], counts)) and col[2] == 11
    g.close()
