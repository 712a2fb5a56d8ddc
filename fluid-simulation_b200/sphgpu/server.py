"""Scene server: continuous batching of independent scene solves on one GPU.

The reference's backend worker steps one `Box<dyn SPHSystem>` at a time
(sci-phi-backend/src/lib.rs:190-210). `SceneServer` is the request-loop form:
scenes are submitted whenever they arrive, admitted while the device has a
free slot and memory for them, advanced concurrently in chunks of
graph-captured steps, and retired at their step count with their completion
time. Each scene's result is the one the single-scene path gives for it.
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import _capi as A
from .scenes import Scene
from .system import grid_desc, make_config


def _result_dict(r: A.SphSceneResult) -> dict:
    m = r.measurement
    return {
        "status": r.status, "steps": r.steps, "time": r.time, "particles": r.particles,
        "submit_s": r.submit_s, "start_s": r.start_s, "finish_s": r.finish_s,
        "latency_s": r.finish_s - r.submit_s, "device_bytes_reserved": r.device_bytes_reserved,
        "graph_replays": r.graph_replays, "kernel_launches": r.kernel_launches,
        "measurement": {name: getattr(m, name) for name, _ in A.SphMeasurement._fields_},
    }


class SceneServer:
    """Owns an `sph_server_t` on one device."""

    def __init__(self, device=0, memory_budget_bytes=0, max_active=0, chunk_steps=0):
        self._L = A.load()
        cfg = A.SphServerConfig(device=device, memory_budget_bytes=memory_budget_bytes,
                                max_active=max_active, chunk_steps=chunk_steps)
        h = C.c_void_p()
        A.check(self._L.sph_server_create(C.byref(cfg), C.byref(h)))
        self._h = h
        self.device = device

    def close(self):
        if getattr(self, "_h", None):
            self._L.sph_server_destroy(self._h)
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

    def submit(self, scene: Scene, steps: int, keep_state=False, precision="f32",
               extra_parameters=None) -> int:
        """Queue `steps` time steps of `scene`; returns the ticket."""
        params = dict(scene.parameters)
        params["device"] = self.device
        if extra_parameters:
            params.update(extra_parameters)
        cfg = make_config(scene.procedures, params, precision=precision, cfl_time_step=scene.cfl_time_step)
        keep = []  # arrays and structs referenced by the request until submit returns

        def arr(a, dtype):
            if a is None:
                return None
            a = np.ascontiguousarray(a, dtype)
            keep.append(a)
            return a.ctypes.data

        req = A.SphSceneRequest()
        req.config = cfg
        req.n = scene.position.shape[0]
        req.position = arr(scene.position, np.float64)
        req.velocity = arr(scene.velocity, np.float64)
        req.mass = arr(scene.mass, np.float64)
        req.fluid_id = arr(scene.fluid_id, np.uint32)
        sets = (A.SphSampleSet * max(1, len(scene.sample_boundaries)))()
        for k, (pts, rigid) in enumerate(scene.sample_boundaries):
            sets[k].count = pts.shape[0]
            sets[k].positions = arr(pts, np.float64)
            if rigid is not None:
                rc = rigid.to_c()
                keep.append(rc)
                sets[k].rigid = C.pointer(rc)
        req.num_sample_sets = len(scene.sample_boundaries)
        req.sample_sets = sets
        vsets = (A.SphVolumeMapSet * max(1, len(scene.volume_maps)))()
        # a request carries no bounding boxes: served volume-map scenes run without
        # rigid-rigid contact
        for k, (sdf, vm, rigid, *_) in enumerate(scene.volume_maps):
            d1 = grid_desc(sdf.x_min, sdf.x_max, sdf.dx, sdf.n)
            d2 = grid_desc(vm.x_min, vm.x_max, vm.dx, vm.n)
            keep += [d1, d2]
            vsets[k].sdf = C.pointer(d1)
            vsets[k].sdf_nodes = arr(sdf.nodes, np.float64)
            vsets[k].vm = C.pointer(d2)
            vsets[k].vm_nodes = arr(vm.nodes, np.float64)
            if rigid is not None:
                rc = rigid.to_c()
                keep.append(rc)
                vsets[k].rigid = C.pointer(rc)
        req.num_volume_maps = len(scene.volume_maps)
        req.volume_maps = vsets
        req.steps = int(steps)
        req.keep_state = 1 if keep_state else 0
        t = C.c_uint64()
        A.check(self._L.sph_server_submit(self._h, C.byref(req), C.byref(t)))
        return t.value

    def poll(self, ticket: int):
        """The result dict once the scene finished, else None."""
        r = A.SphSceneResult()
        rc = self._L.sph_server_poll(self._h, ticket, C.byref(r))
        if rc == A.SPH_PENDING:
            return None
        A.check(rc)
        return _result_dict(r)

    def wait(self, ticket: int, timeout_s: float = -1.0):
        """Blocks until the scene finished (None after `timeout_s` seconds)."""
        r = A.SphSceneResult()
        rc = self._L.sph_server_wait(self._h, ticket, float(timeout_s), C.byref(r))
        if rc == A.SPH_PENDING:
            return None
        A.check(rc)
        return _result_dict(r)

    def fetch_state(self, ticket: int, particles: int):
        x = np.empty(3 * particles, np.float64)
        v = np.empty(3 * particles, np.float64)
        A.check(self._L.sph_server_fetch_state(self._h, ticket, x, v))
        return x.reshape(-1, 3), v.reshape(-1, 3)

    def release(self, ticket: int):
        A.check(self._L.sph_server_release(self._h, ticket))

    def stats(self) -> dict:
        s = A.SphServerStats()
        A.check(self._L.sph_server_get_stats(self._h, C.byref(s)))
        return {name: getattr(s, name) for name, _ in A.SphServerStats._fields_}
