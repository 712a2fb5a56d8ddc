"""Graph-captured stepping (sph_set_step_graphs) against the per-step path.

Both paths run the same kernels in the same order on the same data, so the
states they reach are compared bit for bit: positions, velocities, volumes,
pressures, fluid ids and their order, simulated time and step count. The
cases cover each solver's graph (SESPH, IISPH with its Jacobi while-node,
uncapped and capped, IISPHwOST with TakePredicted), CFL time accumulation, a
dynamic sample boundary (sample buffers swapped inside the graph), the f64
engine, and a chunk that disables particles and is therefore replayed on the
per-step path.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def A():
    from sphgpu import _capi
    _capi.load()
    return _capi


def _run(A, sc, steps, chunk, precision="f32", fields=None, extra=None):
    from sphgpu import scenes
    g = scenes.build_system(sc, precision=precision, fields=fields, extra_parameters=extra)
    if chunk:
        g.set_step_graphs(chunk)
    status = g.step_forward_in_time(steps)
    out = {
        "status": status,
        "x": g.download(A.FIELD_POSITION), "v": g.download(A.FIELD_VELOCITY),
        "V": g.download(A.FIELD_VOLUME), "p": g.download(A.FIELD_PRESSURE),
        "ids": g.get_fluid_ids(), "n": g.n, "time": g.time(), "steps": g.time_steps_propagated(),
        "stats": g.step_stats(), "replays": g.graph_replays(),
    }
    g.close()
    return out


def _assert_same(a, b):
    assert a["n"] == b["n"]
    assert a["steps"] == b["steps"]
    assert a["time"] == b["time"]
    assert a["status"] == b["status"]
    for k in ("x", "v", "V", "p", "ids"):
        assert np.array_equal(a[k], b[k]), k
    for k in ("solver_iterations", "max_neighbors", "time_increment", "average_density"):
        assert a["stats"][k] == b["stats"][k], k


@pytest.mark.parametrize("precision", ["f32", "f64"])
def test_graph_steps_equal_per_step_sesph(A, precision):
    from sphgpu import scenes
    sc = scenes.dam_break_sesph_8k()
    plain = _run(A, sc, 60, 0, precision)
    graph = _run(A, sc, 60, 25, precision)
    _assert_same(plain, graph)
    assert graph["replays"] == 0


def test_graph_steps_equal_per_step_iisph_uncapped(A):
    from sphgpu import scenes
    sc = scenes.serving_dam_break(6000, "IISPH", viscosity=0.02, rest_density=900.0, seed=3)
    sc.parameters = dict(sc.parameters, max_solver_iterations=0)
    plain = _run(A, sc, 50, 0)
    graph = _run(A, sc, 50, 16)
    _assert_same(plain, graph)
    assert graph["stats"]["solver_iterations"] >= 3


def test_graph_steps_equal_per_step_iisph_volume_map_cfl(A):
    from sphgpu import scenes
    from sphgpu.fields import build_volume_map_fields
    sc = scenes.dam_break_iisph_box(n_side=14, spacing=0.02, box=(0.6, 0.32, 0.32))
    sc.parameters = dict(sc.parameters, max_solver_iterations=40)
    verts, faces = sc.mesh
    fields = build_volume_map_fields(verts, faces, 0.08, 0.04)
    plain = _run(A, sc, 30, 0, fields=fields)
    graph = _run(A, sc, 30, 12, fields=fields)
    _assert_same(plain, graph)
    assert graph["time"] > 0


def test_graph_steps_equal_per_step_iisph_w_ost_take_predicted(A):
    from sphgpu import scenes
    from sphgpu.fields import build_volume_map_fields
    sc = scenes.dam_break_iisph_box(n_side=12, spacing=0.02, box=(0.6, 0.32, 0.32))
    sc.procedures = dict(sc.procedures, pressure_solver="IISPHwOST", integration_scheme="TakePredicted")
    sc.cfl_time_step = False
    sc.parameters = dict(sc.parameters, max_solver_iterations=30, time_increment=1e-3)
    pos = sc.position
    side = pos[:, 0] > np.median(pos[:, 0])
    sc.fluid_id = side.astype(np.uint32)
    sc.mass = np.where(side, 500.0, 1000.0) * 0.02 ** 3
    verts, faces = sc.mesh
    fields = build_volume_map_fields(verts, faces, 0.08, 0.04)
    plain = _run(A, sc, 20, 0, fields=fields)
    graph = _run(A, sc, 20, 8, fields=fields)
    _assert_same(plain, graph)


def test_graph_steps_equal_per_step_dynamic_body(A):
    from sphgpu import scenes
    sc = scenes.floating_cube_scene()
    plain = _run(A, sc, 40, 0)
    graph = _run(A, sc, 40, 15)
    _assert_same(plain, graph)


def test_graph_chunk_with_disabled_particles_is_replayed(A):
    """A free-falling block crosses `disable_particles_below` inside a chunk:
    the chunk is redone per step, which renumbers the survivors exactly as
    the reference's swap-remove does."""
    from sphgpu import scenes
    pos = scenes.lattice_block((8, 8, 8), 0.02, origin=(0.0, 0.0, 0.0), jitter=0.01, seed=4)
    sc = scenes.Scene(
        procedures={"kernel_function": "CubicBSpline3D", "integration_scheme": "EulerCromer",
                    "pressure_solver": "SESPH", "neighbor_search": "SpatialHashing",
                    "boundary_handling": "StaticSampleBoundary"},
        parameters={"rest_density_grid_spacing": 0.02, "kernel_support_radius": 0.04,
                    "disable_particles_below": -0.012, "fluid_viscosity": 0.01, "boundary_viscosity": 0.01,
                    "boundary_pressure_acceleration_weighting": 0.7, "boundary_rest_volume_weighting": 1.0,
                    "stiffness": 1000.0, "time_increment": 1e-3},
        cfl_time_step=False, position=pos, mass=np.full(pos.shape[0], 1000.0 * 0.02 ** 3))
    plain = _run(A, sc, 100, 0)
    graph = _run(A, sc, 100, 25)
    assert plain["n"] < pos.shape[0]
    _assert_same(plain, graph)
    assert graph["replays"] >= 1


def test_graph_chunk_that_outgrows_the_neighbor_capacity_is_rerun(A):
    """A soft SESPH dam break compresses, so its neighbor counts outgrow the
    capacity sized at the first update: the chunk is rerun as graphs after
    the capacity grows, and the results stay those of the per-step path."""
    from sphgpu import scenes
    sc = scenes.serving_dam_break(8000, "SESPH", stiffness=500.0, viscosity=0.01, rest_density=1000.0, seed=9)
    # start from a small capacity so that it is outgrown during the run
    plain = _run(A, sc, 150, 0, extra={"neighbor_capacity": 8})
    graph = _run(A, sc, 150, 25, extra={"neighbor_capacity": 8})
    _assert_same(plain, graph)
    assert graph["replays"] >= 1


def test_runs_are_bit_identical_run_to_run():
    """Two systems built from the same scene step to the same state bit for
    bit: the block halos' layout does not depend on thread timing (ordered
    hash insertion), so neither does the bank-aware order of the lists."""
    from sphgpu import _capi as A, scenes
    sc = scenes.serving_dam_break(30000, "IISPH", viscosity=0.03, rest_density=700.0, seed=4)
    xs = []
    for _ in range(2):
        g = scenes.build_system(sc)
        g.step_forward_in_time(60)
        xs.append((g.download(A.FIELD_POSITION), g.download(A.FIELD_PRESSURE)))
        g.close()
    assert np.array_equal(xs[0][0], xs[1][0]) and np.array_equal(xs[0][1], xs[1][1])
