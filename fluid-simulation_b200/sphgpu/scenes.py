"""Seeded synthetic scenes for the SPH engine.

Fluid blocks are cubic lattices with uniform jitter, stored as f32-representable
values so that an f64 restatement sees exactly the positions the f32 engine holds
(the reference injects such a state through its `--state` checkpoint path,
sim_lib sph/setup/mod.rs:142-153). Containers are the reference's cube mesh
(cube_face_normals_inwards.obj: 8 vertices, 12 inward-facing triangles) under
the reference's mesh transform (utilities/triangle_mesh.rs:314-334: scale,
then rotate, then translate).

Every fluid block keeps its first particle centers WALL_GAP = 1.5 spacings
from the container walls. Both boundary handlings add the wall's density
where a fluid neighbor layer would be: sample boundaries at the wall plane,
volume maps at max(sd + 1/4 dx, dx) from the particle. A fluid layer closer
than that is over-dense at rest: at half a spacing, corner particles start
at up to three times the rest density, and the IISPH solve of such a state
does not converge and blows the scene apart within a few steps.
"""
from __future__ import annotations

from dataclasses import dataclass, field

import numpy as np

WALL_GAP = 1.5  # spacings between a container wall and the first fluid particle centers

# Unit cube [-1, 1]^3 with inward-facing triangles, vertex order of the
# reference's OBJ file.
CUBE_VERTICES = np.array([
    [1, 1, 1], [1, 1, -1], [1, -1, 1], [1, -1, -1],
    [-1, 1, 1], [-1, 1, -1], [-1, -1, 1], [-1, -1, -1]], dtype=np.float64)
CUBE_FACES_INWARD = np.array([
    [3, 5, 1], [8, 3, 4], [6, 7, 8], [8, 2, 6], [4, 1, 2], [2, 5, 6],
    [3, 7, 5], [8, 7, 3], [6, 5, 7], [8, 4, 2], [4, 3, 1], [2, 1, 5]], dtype=np.uint32) - 1
CUBE_FACES_OUTWARD = CUBE_FACES_INWARD[:, ::-1].copy()


def euler_to_matrix(rx, ry, rz):
    """nalgebra Rotation3::from_euler_angles(roll, pitch, yaw) = Rz * Ry * Rx."""
    cx, sx, cy, sy, cz, sz = np.cos(rx), np.sin(rx), np.cos(ry), np.sin(ry), np.cos(rz), np.sin(rz)
    Rx = np.array([[1, 0, 0], [0, cx, -sx], [0, sx, cx]])
    Ry = np.array([[cy, 0, sy], [0, 1, 0], [-sy, 0, cy]])
    Rz = np.array([[cz, -sz, 0], [sz, cz, 0], [0, 0, 1]])
    return Rz @ Ry @ Rx


def transform_mesh(verts, translation=(0, 0, 0), rotation_euler_deg=(0, 0, 0), scale=(1, 1, 1)):
    v = np.asarray(verts, np.float64) * np.broadcast_to(np.asarray(scale, np.float64), (3,))
    R = euler_to_matrix(*np.radians(rotation_euler_deg))
    return v @ R.T + np.asarray(translation, np.float64)


def sample_triangle_surface(v0, v1, v2, spacing):
    """Isotropic raster of one triangle (utilities/sampling.rs:59-106): grid
    points (min + i*spacing, min + j*spacing) of the triangle's 2D frame, row
    j outer, kept when inside or on the triangle (no two edge functions of
    opposite sign), mapped back as v0 + e_u x + e_v y."""
    e1, e2 = v1 - v0, v2 - v0
    l1 = np.sqrt((e1[0] * e1[0] + e1[1] * e1[1]) + e1[2] * e1[2])
    if l1 < 1e-12:
        return np.zeros((0, 3))
    eu = e1 / l1
    proj = (e2[0] * eu[0] + e2[1] * eu[1]) + e2[2] * eu[2]
    perp = e2 - eu * proj
    pl = np.sqrt((perp[0] * perp[0] + perp[1] * perp[1]) + perp[2] * perp[2])
    if pl < 1e-12:
        return np.zeros((0, 3))
    ev = perp / pl
    p = np.array([[0.0, 0.0], [l1, 0.0], [proj, pl]])
    min_x, max_x = p[:, 0].min(), p[:, 0].max()
    min_y, max_y = p[:, 1].min(), p[:, 1].max()
    nx = int(np.ceil((max_x - min_x) / spacing))
    ny = int(np.ceil((max_y - min_y) / spacing))
    a, b, c = p
    y = min_y + np.arange(ny + 1, dtype=np.float64) * spacing
    x = min_x + np.arange(nx + 1, dtype=np.float64) * spacing
    Y, X = np.meshgrid(y, x, indexing="ij")
    X, Y = X.ravel(), Y.ravel()

    def edge(p0, p1):
        return (p1[0] - p0[0]) * (Y - p0[1]) - (p1[1] - p0[1]) * (X - p0[0])
    d1, d2, d3 = edge(a, b), edge(b, c), edge(c, a)
    has_neg = (d1 < 0.0) | (d2 < 0.0) | (d3 < 0.0)
    has_pos = (d1 > 0.0) | (d2 > 0.0) | (d3 > 0.0)
    keep = ~(has_neg & has_pos)
    X, Y = X[keep], Y[keep]
    return (v0[None, :] + eu[None, :] * X[:, None]) + ev[None, :] * Y[:, None]


def _cross2(a, b):
    return a[0] * b[1] - a[1] * b[0]


def sample_triangle_mesh_surface(verts, faces, spacing):
    """All triangles in order (utilities/sampling.rs:169-178)."""
    parts = [sample_triangle_surface(verts[f[0]], verts[f[1]], verts[f[2]], spacing) for f in faces]
    return np.concatenate(parts, axis=0) if parts else np.zeros((0, 3))


def lattice_block(counts, spacing, origin, jitter=0.01, seed=0):
    """Cubic lattice of counts[0]*counts[1]*counts[2] particles starting half a
    spacing inside `origin`, with uniform jitter of +-jitter*spacing per axis;
    returned as f32-representable f64 values (x fastest)."""
    nx, ny, nz = counts
    rng = np.random.default_rng(seed)
    k, j, i = np.meshgrid(np.arange(nz), np.arange(ny), np.arange(nx), indexing="ij")
    base = np.stack([i.ravel(), j.ravel(), k.ravel()], axis=1).astype(np.float64)
    pos = np.asarray(origin, np.float64) + (base + 0.5) * spacing
    pos += rng.uniform(-jitter * spacing, jitter * spacing, size=pos.shape)
    return pos.astype(np.float32).astype(np.float64)


@dataclass
class Scene:
    """Inputs of one system: configuration, fluid state and boundaries."""
    procedures: dict
    parameters: dict
    cfl_time_step: bool
    position: np.ndarray
    mass: np.ndarray
    velocity: np.ndarray | None = None
    fluid_id: np.ndarray | None = None
    sample_boundaries: list = field(default_factory=list)   # [(positions, RigidInit|None)]
    volume_maps: list = field(default_factory=list)         # [(sdf, vm, RigidInit|None[, (center, half)])]
    mesh: tuple | None = None                               # (verts, faces) of the container
    description: str = ""
    container: tuple | None = None                          # box extents of a box container


def dam_break_sesph_8k(jitter_seed=0, n_side=20):
    """SESPH dam break: a 20^3 lattice (spacing 0.02, +-1 % jitter) in the
    corner (1.5 spacings from the walls) of a 0.6 m cube container of StaticSampleBoundary samples taken at
    0.7 * spacing from the reference's inward cube mesh scaled 0.3; support 2h,
    rest density 1000, stiffness 1000, viscosity 0.01, dt 1e-3, EulerCromer."""
    h = 0.02
    verts = transform_mesh(CUBE_VERTICES, scale=(0.3, 0.3, 0.3))
    samples = sample_triangle_mesh_surface(verts, CUBE_FACES_INWARD, 0.7 * h)
    o = -0.3 + (WALL_GAP - 0.5) * h
    pos = lattice_block((n_side, n_side, n_side), h, origin=(o, o, o), jitter=0.01, seed=jitter_seed)
    return Scene(
        procedures={"kernel_function": "CubicBSpline3D", "integration_scheme": "EulerCromer",
                    "pressure_solver": "SESPH", "neighbor_search": "SpatialHashing",
                    "boundary_handling": "StaticSampleBoundary"},
        parameters={"rest_density_grid_spacing": h, "kernel_support_radius": 2 * h,
                    "disable_particles_below": -50.0, "fluid_viscosity": 0.01,
                    "boundary_viscosity": 0.01, "boundary_pressure_acceleration_weighting": 0.7,
                    "boundary_rest_volume_weighting": 1.0, "stiffness": 1000.0,
                    "time_increment": 1e-3},
        cfl_time_step=False, position=pos, mass=np.full(pos.shape[0], 1000.0 * h ** 3),
        sample_boundaries=[(samples, None)], mesh=(verts, CUBE_FACES_INWARD),
        description=f"SESPH dam break {pos.shape[0]} particles, sample boundary {samples.shape[0]}")


def dam_break_iisph_box(n_side=100, spacing=0.01, jitter_seed=0, box=(2.0, 1.0, 1.0)):
    """IISPH dam break: an n_side^3 lattice (+-1 % jitter) at the -x end of a
    box container (the reference's inward cube mesh scaled to `box`, each axis
    widened where needed so the block keeps 1.5 spacings from every wall:
    100^3 at 0.01 m makes the 2 x 1 x 1 m box 2 x 1.02 x 1.02 m) handled as a
    VolumeMapBoundary with the reference's field spacing dx = 4 * spacing;
    omega 0.5, target density error 0.1 %, CFL 0.4 with dt <= 2e-3."""
    h = spacing
    need = n_side * h + 2.0 * (WALL_GAP - 0.5) * h
    box = tuple(max(float(b), need) for b in box)
    verts = transform_mesh(CUBE_VERTICES, scale=(box[0] / 2, box[1] / 2, box[2] / 2))
    lo = -0.5 * np.asarray(box) + (WALL_GAP - 0.5) * h
    pos = lattice_block((n_side, n_side, n_side), h, origin=lo, jitter=0.01, seed=jitter_seed)
    return Scene(
        procedures={"kernel_function": "CubicBSpline3D", "integration_scheme": "EulerCromer",
                    "pressure_solver": "IISPH", "neighbor_search": "SpatialHashing",
                    "boundary_handling": "VolumeMapBoundary"},
        parameters={"rest_density_grid_spacing": h, "kernel_support_radius": 2 * h,
                    "disable_particles_below": -50.0, "fluid_viscosity": 0.01,
                    "boundary_viscosity": 0.01, "boundary_pressure_acceleration_weighting": 0.7,
                    "boundary_rest_volume_weighting": 1.0, "target_density_error": 0.1,
                    "relaxation_factor": 0.5, "min_diagonal_element": 1e-10,
                    "max_time_increment": 2e-3, "cfl_number": 0.4},
        cfl_time_step=True, position=pos, mass=np.full(pos.shape[0], 1000.0 * h ** 3),
        mesh=(verts, CUBE_FACES_INWARD), container=box,
        description=f"IISPH dam break {pos.shape[0]} particles in a {box} box volume map")


def build_system(scene: Scene, precision="f32", device=0, fields=None, extra_parameters=None):
    """Create, fill and initialize a GpuSystem for `scene`. `fields` supplies the
    (sdf, vm) volume-map fields of the container when the scene uses one."""
    from .system import GpuSystem, make_config
    params = dict(scene.parameters)
    params["device"] = device
    if extra_parameters:
        params.update(extra_parameters)
    cfg = make_config(scene.procedures, params, precision=precision,
                      cfl_time_step=scene.cfl_time_step)
    s = GpuSystem(cfg)
    s.upload_fluid(scene.position, scene.velocity, scene.mass, scene.fluid_id)
    for pts, rigid in scene.sample_boundaries:
        s.add_sample_boundary(pts, rigid)
    for sdf, vm, rigid, *aabb in scene.volume_maps:
        s.add_volume_map_boundary(sdf, vm, rigid, aabb[0] if aabb else None)
    if fields is not None:
        s.add_volume_map_boundary(fields[0], fields[1])
    s.initialize()
    return s


def icosphere(subdivisions=4, radius=1.0, inward=False):
    """Subdivided icosahedron (10*4^s+2 vertices, 20*4^s triangles); outward
    winding unless `inward` (a container)."""
    t = (1.0 + 5 ** 0.5) / 2.0
    v = [(-1, t, 0), (1, t, 0), (-1, -t, 0), (1, -t, 0), (0, -1, t), (0, 1, t), (0, -1, -t), (0, 1, -t),
         (t, 0, -1), (t, 0, 1), (-t, 0, -1), (-t, 0, 1)]
    verts = [np.array(p, np.float64) / np.linalg.norm(p) for p in v]
    faces = [(0, 11, 5), (0, 5, 1), (0, 1, 7), (0, 7, 10), (0, 10, 11), (1, 5, 9), (5, 11, 4), (11, 10, 2),
             (10, 7, 6), (7, 1, 8), (3, 9, 4), (3, 4, 2), (3, 2, 6), (3, 6, 8), (3, 8, 9), (4, 9, 5),
             (2, 4, 11), (6, 2, 10), (8, 6, 7), (9, 8, 1)]
    for _ in range(subdivisions):
        cache = {}

        def mid(a, b):
            key = (min(a, b), max(a, b))
            if key not in cache:
                m = verts[a] + verts[b]
                verts.append(m / np.linalg.norm(m))
                cache[key] = len(verts) - 1
            return cache[key]
        nf = []
        for a, b, c in faces:
            ab, bc, ca = mid(a, b), mid(b, c), mid(c, a)
            nf += [(a, ab, ca), (b, bc, ab), (c, ca, bc), (ab, bc, ca)]
        faces = nf
    V = np.array(verts) * radius
    F = np.array(faces, np.uint32)
    if inward:
        F = F[:, ::-1].copy()
    return V, F


def box_inertia(mass, side):
    """Inertia tensor of a solid cube of the given side about its center."""
    i = mass * side * side / 6.0
    return np.diag([i, i, i])


def floating_cube_scene(n_side=12, spacing=0.02, body_side=0.12, body_density=500.0, seed=0):
    """SESPH pool in the 0.6 m sample-boundary cube with a dynamic sample-boundary
    cube body (two-way coupled RigidBodyMotion) just above the water."""
    sc = dam_break_sesph_8k(jitter_seed=seed, n_side=n_side)
    verts = transform_mesh(CUBE_VERTICES, scale=(body_side / 2,) * 3)
    samples = sample_triangle_mesh_surface(verts, CUBE_FACES_OUTWARD, 0.7 * spacing)
    top = sc.position[:, 2].max()
    mass = body_density * body_side ** 3
    from .system import RigidInit
    rigid = RigidInit(mass=mass, inertia_body=box_inertia(mass, body_side),
                      center_of_mass=(-0.15, -0.15, top + 0.5 * body_side + 0.25 * spacing),
                      orientation=(np.cos(0.1), np.sin(0.1), 0.0, 0.0),
                      angular_velocity=(0.0, 0.5, 0.0))
    sc.sample_boundaries.append((samples, rigid))
    sc.description += f", dynamic cube body with {samples.shape[0]} samples"
    return sc


def serving_dam_break(n_target, solver="SESPH", stiffness=1000.0, viscosity=0.01, rest_density=1000.0,
                      spacing=0.02, time_increment=1e-3, seed=0):
    """Dam break of the scene sweep: an n_side^3 lattice block (n_side =
    round(n_target^(1/3)), +-1 % jitter) at the -x end of a box container
    of 2 x 1 x 1.5 block lengths plus the wall gaps, sampled as a StaticSampleBoundary
    at 0.7 * spacing from the reference's inward cube mesh; support 2h, fixed
    dt, EulerCromer. IISPH uses omega 0.5, target density error 0.1 % and at
    most 100 sweeps."""
    n_side = max(4, int(round(n_target ** (1.0 / 3.0))))
    h = spacing
    L = n_side * h
    g = (WALL_GAP - 0.5) * h
    half = np.array([L, 0.5 * L, 0.75 * L]) + g
    verts = transform_mesh(CUBE_VERTICES, scale=tuple(half))
    samples = sample_triangle_mesh_surface(verts, CUBE_FACES_INWARD, 0.7 * h)
    pos = lattice_block((n_side, n_side, n_side), h, origin=-half + g, jitter=0.01, seed=seed)
    params = {"rest_density_grid_spacing": h, "kernel_support_radius": 2 * h,
              "disable_particles_below": -50.0, "fluid_viscosity": viscosity,
              "boundary_viscosity": viscosity, "boundary_pressure_acceleration_weighting": 0.7,
              "boundary_rest_volume_weighting": 1.0, "time_increment": time_increment}
    if solver == "SESPH":
        params["stiffness"] = stiffness
    else:
        params.update({"target_density_error": 0.1, "relaxation_factor": 0.5, "min_diagonal_element": 1e-10,
                       "max_solver_iterations": 100})
    return Scene(
        procedures={"kernel_function": "CubicBSpline3D", "integration_scheme": "EulerCromer",
                    "pressure_solver": solver, "neighbor_search": "SpatialHashing",
                    "boundary_handling": "StaticSampleBoundary"},
        parameters=params, cfl_time_step=False, position=pos,
        mass=np.full(pos.shape[0], rest_density * h ** 3), sample_boundaries=[(samples, None)],
        mesh=(verts, CUBE_FACES_INWARD),
        description=f"{solver} dam break {pos.shape[0]} particles, {samples.shape[0]} boundary samples")


@dataclass
class SceneRequest:
    """One request of the scene sweep."""
    arrival_s: float
    n_target: int
    solver: str
    stiffness: float
    viscosity: float
    rest_density: float
    steps: int
    seed: int

    def scene(self) -> Scene:
        return serving_dam_break(self.n_target, self.solver, self.stiffness, self.viscosity, self.rest_density,
                                 seed=self.seed)


def scene_sweep(count=256, rate_per_s=20.0, n_min=5000, n_max=500000, steps=500, seed=5):
    """Seeded parameter sweep of dam-break scenes: Poisson arrivals at
    `rate_per_s`, particle counts log-uniform in [n_min, n_max], SESPH or
    IISPH with equal probability, stiffness U[500, 5000], viscosity
    U[0.001, 0.05], rest density U[500, 1500], `steps` time steps each."""
    rng = np.random.default_rng(seed)
    arrivals = np.cumsum(rng.exponential(1.0 / rate_per_s, count))
    n = np.exp(rng.uniform(np.log(n_min), np.log(n_max), count))
    solver = rng.integers(0, 2, count)
    k = rng.uniform(500.0, 5000.0, count)
    nu = rng.uniform(0.001, 0.05, count)
    rho = rng.uniform(500.0, 1500.0, count)
    return [SceneRequest(float(arrivals[i]), int(n[i]), "SESPH" if solver[i] == 0 else "IISPH", float(k[i]),
                         float(nu[i]), float(rho[i]), int(steps), int(seed * 100003 + i)) for i in range(count)]


def two_fluid_ball(radius=1.0, spacing=0.008, seed=0, subdivisions=4):
    """IISPHwOST two-fluid ball (precision study): a jittered lattice filling
    the lower half of a sphere container of `radius` (inward icosphere of
    20*4^subdivisions triangles, handled as a VolumeMapBoundary at the
    reference's field spacing 4 * spacing), split by a seeded random plane
    through the center into fluid ids 0 / 1 with rest densities 1000 / 500;
    viscosity 0.005, TakePredicted, fixed dt 5e-4."""
    h = spacing
    rng = np.random.default_rng(seed)
    n = int(np.ceil(radius / h))
    g = (np.arange(-n, n) + 0.5) * h
    Z, Y, X = np.meshgrid(g, g, g, indexing="ij")
    pos = np.stack([X.ravel(), Y.ravel(), Z.ravel()], axis=1)
    inside = (np.linalg.norm(pos, axis=1) < radius - WALL_GAP * h) & (pos[:, 2] < 0.0)
    pos = pos[inside]
    pos = pos + rng.uniform(-0.01 * h, 0.01 * h, size=pos.shape)
    pos = pos.astype(np.float32).astype(np.float64)
    normal = rng.normal(size=3)
    normal /= np.linalg.norm(normal)
    side = (pos @ normal) > 0.0
    verts, faces = icosphere(subdivisions, radius, inward=True)
    return Scene(
        procedures={"kernel_function": "CubicBSpline3D", "integration_scheme": "TakePredicted",
                    "pressure_solver": "IISPHwOST", "neighbor_search": "SpatialHashing",
                    "boundary_handling": "VolumeMapBoundary"},
        parameters={"rest_density_grid_spacing": h, "kernel_support_radius": 2 * h,
                    "disable_particles_below": -50.0, "fluid_viscosity": 0.005, "boundary_viscosity": 0.005,
                    "boundary_pressure_acceleration_weighting": 0.7, "boundary_rest_volume_weighting": 1.0,
                    "target_density_error": 0.1, "relaxation_factor": 0.5, "min_diagonal_element": 1e-10,
                    "time_increment": 5e-4},
        cfl_time_step=False, position=pos, mass=np.where(side, 500.0, 1000.0) * h ** 3,
        fluid_id=side.astype(np.uint32), mesh=(verts, faces),
        description=f"IISPHwOST two-fluid ball, {pos.shape[0]} particles, radius {radius}")


def rigid_body_tank(spacing=0.02, tank=(0.8, 0.4, 0.5), fill=0.2, n_cubes=4, n_spheres=4, cube_side=0.15,
                    sphere_radius=0.08, seed=0):
    """IISPH rigid-body coupling, all StaticSampleBoundary: a box tank sampled
    at 0.7 * spacing, a fluid layer of height `fill`, and n_cubes cubes plus
    n_spheres spheres (two-way coupled RigidBodyMotion bodies sampled at
    0.7 * spacing) placed above the surface with seeded densities U[300, 1500];
    CFL time step (0.4, dt <= 2e-3)."""
    from .system import RigidInit
    h = spacing
    rng = np.random.default_rng(seed)
    half = 0.5 * np.asarray(tank, np.float64)
    verts = transform_mesh(CUBE_VERTICES, scale=tuple(half))
    walls = sample_triangle_mesh_surface(verts, CUBE_FACES_INWARD, 0.7 * h)
    g = (WALL_GAP - 0.5) * h
    counts = (int(round((tank[0] - 2 * g) / h)), int(round((tank[1] - 2 * g) / h)), int(fill / h))
    pos = lattice_block(counts, h, origin=-half + g, jitter=0.01, seed=seed)
    bodies = []
    nb = n_cubes + n_spheres
    cols = int(np.ceil(nb / 2))
    for b in range(nb):
        cube = b < n_cubes
        size = cube_side if cube else 2 * sphere_radius
        cx = -half[0] + (b % cols + 0.5) * (tank[0] / cols)
        cy = -half[1] + (b // cols + 0.5) * (tank[1] / 2)
        cz = -half[2] + fill + 0.6 * size + 0.02 * (b % 3)
        com = (cx + rng.uniform(-0.01, 0.01), cy + rng.uniform(-0.01, 0.01), cz)
        rho = rng.uniform(300.0, 1500.0)
        if cube:
            bv = transform_mesh(CUBE_VERTICES, scale=(cube_side / 2,) * 3)
            samples = sample_triangle_mesh_surface(bv, CUBE_FACES_OUTWARD, 0.7 * h)
            mass = rho * cube_side ** 3
            inertia = box_inertia(mass, cube_side)
        else:
            bv, bf = icosphere(2, sphere_radius)
            samples = sample_triangle_mesh_surface(bv, bf, 0.7 * h)
            mass = rho * 4.0 / 3.0 * np.pi * sphere_radius ** 3
            inertia = np.eye(3) * 0.4 * mass * sphere_radius ** 2
        rigid = RigidInit(mass=mass, inertia_body=inertia, center_of_mass=com,
                          orientation=tuple(np.r_[np.cos(0.05 * b), np.sin(0.05 * b) * np.array([0.6, 0.0, 0.8])]),
                          angular_velocity=(0.0, 0.2 * (b % 2), 0.0))
        bodies.append((samples, rigid))
    return Scene(
        procedures={"kernel_function": "CubicBSpline3D", "integration_scheme": "EulerCromer",
                    "pressure_solver": "IISPH", "neighbor_search": "SpatialHashing",
                    "boundary_handling": "StaticSampleBoundary"},
        parameters={"rest_density_grid_spacing": h, "kernel_support_radius": 2 * h,
                    "disable_particles_below": -50.0, "fluid_viscosity": 0.01, "boundary_viscosity": 0.01,
                    "boundary_pressure_acceleration_weighting": 0.7, "boundary_rest_volume_weighting": 1.0,
                    "target_density_error": 0.1, "relaxation_factor": 0.5, "min_diagonal_element": 1e-10,
                    "max_time_increment": 2e-3, "cfl_number": 0.4, "max_solver_iterations": 100},
        cfl_time_step=True, position=pos, mass=np.full(pos.shape[0], 1000.0 * h ** 3),
        sample_boundaries=[(walls, None)] + bodies, mesh=(verts, CUBE_FACES_INWARD),
        description=f"IISPH tank, {pos.shape[0]} particles, {n_cubes} cubes + {n_spheres} spheres")
