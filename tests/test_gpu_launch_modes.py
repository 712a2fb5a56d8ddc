"""The sweep passes' launch options change scheduling only, never a result.

The Jacobi sweep passes are launched as programmatic dependents of the pass
before them (SPHGPU_DEPENDENT_LAUNCH, on by default) and prefetch the next
wave's streams into L2 (SPHGPU_SWEEP_PREFETCH, on by default). Both settings
are read when a system is created, so each mode runs in a child process: the
same 216k-particle IISPH dam break (large enough that the prefetch reaches
blocks of every pass), the same steps, and the states compared bit for bit
with the default's (positions, velocities, volumes, pressures, sweep counts).
"""
import os
import subprocess
import sys

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))

CHILD = r"""
import sys, numpy as np
sys.path.insert(0, sys.argv[2])
from sphgpu import _capi as A, scenes
from sphgpu.fields import build_volume_map_fields
sc = scenes.dam_break_iisph_box(n_side=60, box=(1.2, 0.6, 0.6))
verts, faces = sc.mesh
sp = sc.parameters["rest_density_grid_spacing"]
fields = build_volume_map_fields(verts, faces, 4 * sp, sc.parameters["kernel_support_radius"], 30)
g = scenes.build_system(sc, precision="f32", fields=fields)
sweeps = []
for _ in range(6):
    g.step_forward_in_time(1)
    sweeps.append(g.step_stats()["solver_iterations"])
np.savez(sys.argv[1], x=g.download(A.FIELD_POSITION), v=g.download(A.FIELD_VELOCITY),
         V=g.download(A.FIELD_VOLUME), p=g.download(A.FIELD_PRESSURE), sweeps=np.array(sweeps))
g.close()
"""


def _run_mode(tmp_path, name, env_extra):
    out = tmp_path / f"{name}.npz"
    env = dict(os.environ, **env_extra)
    subprocess.run([sys.executable, "-c", CHILD, str(out), os.path.join(ROOT, "fluid-simulation_b200")],
                   env=env, check=True, timeout=300)
    return dict(np.load(out))


def test_dependent_launch_and_prefetch_leave_results_unchanged(tmp_path):
    base = _run_mode(tmp_path, "default", {})
    assert base["x"].shape[0] == 60 ** 3 and base["sweeps"].min() > 0
    for name, env in (("no_dependent_launch", {"SPHGPU_DEPENDENT_LAUNCH": "0"}),
                      ("no_prefetch", {"SPHGPU_SWEEP_PREFETCH": "0"})):
        other = _run_mode(tmp_path, name, env)
        for key in ("x", "v", "V", "p", "sweeps"):
            assert np.array_equal(base[key], other[key]), (name, key)
