"""Shared test setup: import paths, the `gpu` marker, and helpers."""
import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, os.path.join(ROOT, "fluid-simulation_b200"))
sys.path.insert(0, os.path.join(ROOT, "oracle"))


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200) and libsphgpu.so")


def has_gpu():
    try:
        import torch
        return torch.cuda.is_available()
    except Exception:
        return False


@pytest.fixture(scope="session")
def oracle():
    import oracle as O
    O.lib()
    return O


def oracle_config(scene):
    """Oracle config dict for a sphgpu Scene (same field meaning as sph_config)."""
    from sphgpu.system import PROCEDURES
    cfg = dict(scene.parameters)
    cfg.pop("device", None)
    cfg.pop("neighbor_capacity", None)
    cfg.setdefault("max_solver_iterations", 0)
    cfg["integration_scheme"] = PROCEDURES["integration_scheme"][scene.procedures["integration_scheme"]]
    cfg["pressure_solver"] = PROCEDURES["pressure_solver"][scene.procedures["pressure_solver"]]
    cfg["boundary_handling"] = PROCEDURES["boundary_handling"][scene.procedures["boundary_handling"]]
    cfg["cfl_time_step"] = 1 if scene.cfl_time_step else 0
    if "time_increment" not in cfg:
        cfg["time_increment"] = 0.0
    return cfg


def build_oracle(scene, fields=None, extra=None):
    """The oracle set up like `scene` (plus optional volume-map `fields`);
    `extra` adds oracle-only config fields (e.g. contact_fixed_sweeps)."""
    import oracle as O
    cfg = oracle_config(scene)
    if extra:
        cfg.update(extra)
    s = O.OracleSystem(cfg)
    s.upload_fluid(scene.position, scene.velocity, scene.mass, scene.fluid_id)
    boxes = []
    for pts, rigid in scene.sample_boundaries:
        s.add_sample_boundary(pts, None if rigid is None else rigid.to_array32())
    for sdf, vm, rigid, *aabb in scene.volume_maps:
        s.add_volume_map_boundary(_oracle_field(sdf), _oracle_field(vm),
                                  None if rigid is None else rigid.to_array32())
        if aabb:
            s.set_vm_aabb(len(boxes), *aabb[0])
        boxes.append(bool(aabb))
    if fields is not None:
        s.add_volume_map_boundary(*(_oracle_field(f) for f in fields))
    s.initialize()
    return s


def _oracle_field(f):
    """The oracle's Field for a field built by either side."""
    import oracle as O
    if hasattr(f, "desc"):
        return f
    return O.Field(f.x_min, f.x_max, f.dx, f.n, f.nodes)


def rel_err(a, b, floor):
    a = np.asarray(a, np.float64)
    b = np.asarray(b, np.float64)
    return np.max(np.abs(a - b) / np.maximum(np.abs(b), floor)) if a.size else 0.0


def csr_multisets_equal(off_a, idx_a, off_b, idx_b):
    """True when two CSR neighbor tables hold the same multiset in every row
    (rows compared after a per-row sort), vectorized for millions of rows."""
    off_a = np.asarray(off_a, np.int64)
    off_b = np.asarray(off_b, np.int64)
    if off_a.shape != off_b.shape or not np.array_equal(off_a, off_b):
        return False
    n = off_a.size - 1
    row = np.repeat(np.arange(n, dtype=np.int64), np.diff(off_a))
    ka = (row << 32) | np.asarray(idx_a, np.int64)
    kb = (row << 32) | np.asarray(idx_b, np.int64)
    ka.sort()
    kb.sort()
    return np.array_equal(ka, kb)
