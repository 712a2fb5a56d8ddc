"""Volume-map boundary fields built on the GPU.

`build_volume_map_fields` is DiscretizedBoundaryFields::new
(sim_lib sph/boundary_handling/volume_map_boundary.rs:1547-1636): the mesh
signed-distance field pruned to |sd| <= 3.1 r, then the volume map integrated
over balls of radius r on that field. Both are dense cubic-serendipity node
lattices (NaN = absent node) ready for GpuSystem.add_volume_map_boundary.
"""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass

import numpy as np

from . import _capi as A


@dataclass
class Field:
    x_min: np.ndarray
    x_max: np.ndarray
    dx: float
    n: np.ndarray
    nodes: np.ndarray

    @property
    def shape(self):
        return tuple(int(v) for v in (3 * self.n[::-1] + 1))


def _to_field(g: A.SphGridDesc, nodes: np.ndarray) -> Field:
    return Field(np.array(g.x_min[:]), np.array(g.x_max[:]), float(g.dx), np.array(g.n[:], np.int64),
                 nodes)


def grids(verts, dx, kernel_support_radius):
    L = A.load()
    v = np.ascontiguousarray(verts, np.float64).reshape(-1, 3)
    sg, vg = A.SphGridDesc(), A.SphGridDesc()
    A.check(L.sph_volume_map_grids(v.ravel(), v.shape[0], float(dx), float(kernel_support_radius),
                                   C.byref(sg), C.byref(vg)))
    return sg, vg


def build_volume_map_fields(verts, faces, dx, kernel_support_radius, quadrature_degree=30, device=0):
    """(sdf, vm) fields of a closed triangle mesh; dx is the reference's
    4 * rest_density_grid_spacing."""
    L = A.load()
    v = np.ascontiguousarray(verts, np.float64).reshape(-1, 3)
    f = np.ascontiguousarray(faces, np.uint32).reshape(-1, 3)
    sg, vg = grids(v, dx, kernel_support_radius)
    ns = int(np.prod([3 * sg.n[d] + 1 for d in range(3)]))
    nv = int(np.prod([3 * vg.n[d] + 1 for d in range(3)]))
    sdf_nodes = np.zeros(ns, np.float64)
    A.check(L.sph_build_sdf_field(v.ravel(), v.shape[0], f.ravel(), f.shape[0], C.byref(sg),
                                  float(kernel_support_radius), sdf_nodes, device))
    vm_nodes = np.zeros(nv, np.float64)
    A.check(L.sph_build_volume_map_field(C.byref(sg), sdf_nodes, C.byref(vg),
                                         float(kernel_support_radius), int(quadrature_degree),
                                         vm_nodes, device))
    return _to_field(sg, sdf_nodes), _to_field(vg, vm_nodes)
