#!/usr/bin/env python
"""Throughput benchmark: IISPH dam break at 1M particles, particle-updates/s.

Workload (one "step" = one SPH time step, sim_lib sph/mod.rs:125-144, of the
whole scene): a 100^3 lattice (spacing 0.01 m, +-1 % seeded jitter, rest
density 1000) at the -x end of a 2 x 1 x 1 m box, widened to 1.02 m so the
block keeps 1.5 spacings from every wall, handled as a VolumeMapBoundary
(fields at the reference's dx = 4 * spacing, built on the GPU before timing),
IISPH with omega 0.5, target density error 0.1 %, at most 100 sweeps per
solve, CFL time step (0.4, dt <= 2e-3), viscosity 0.01, f32 state. Inputs
are synthetic and seeded.

Arms:
  default          the CUDA engine through the C ABI; `value` is device time
                   (CUDA events on the engine's stream), `e2e` runs the same
                   steps through sph_step_host with host buffers in and out.
                   `cpu_baseline` is the reference's CPU algorithm (the f64
                   C++ restatement in oracle/, all host threads) on the same
                   1M scene from the same seeded state and warm-up, timed on
                   its first steps after the warm-up (about 10-30 s of CPU
                   work). The line's `serving` object is the scene sweep
                   (Poisson-arrival dam breaks of 5k-500k particles, 500 steps
                   each) served batched by the scene server and one at a time
                   on the plain path, the same requests in both arms.
  --impl reference the reference's CPU algorithm (the oracle restatement, all
                   host threads) on the same 1M scene: same seeded state, same
                   warm-up steps, then the timed steps (all of --steps unless
                   --ref-seconds runs out first; the line says how many).
Multi-GPU: scenes are independent, so N GPUs run N replicas (weak scaling,
no collective on the data path); rank 0 prints the JSON line.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
# The scene server runs every resident scene on its own stream; more hardware
# work queues than the default 8 keep their kernels from serializing.
os.environ.setdefault("CUDA_DEVICE_MAX_CONNECTIONS", "32")
sys.path.insert(0, os.path.join(ROOT, "fluid-simulation_b200"))

METRIC = "particle-updates/s at 1M IISPH (VolumeMapBoundary dam break)"
UNIT = "particle-updates/s"
# Algorithmic bytes per particle for each kernel class (f32 words; neighbor
# gathers cache-served and counted 0), after the per-pass stream model of the
# IISPH step: reads/writes of the per-particle SoA state each pass touches.
BYTES_PER_PARTICLE = {
    "iisph_jacobi": 60,          # R x,V, acc_p, s, a_ii, p, boundary agg.  W p
    "iisph_pressure_accel": 52,  # R x,V, m, p, boundary agg.               W acc_p
    "iisph_source_diag": 72,     # R x,v,a,V,m, boundary agg.              W s,a_ii,p
    "accel_nonpressure": 60,     # R x,v,V,m, boundary samples             W a, v*
    "pressure_accel": 64,        # R x,V,m,p,a, boundary agg.              W a
    "neighbors_density": 32,     # R x, boundary agg.                      W V
    "vm_near": 20,               # R x                                     W near list (wall particles)
    "boundary_samples": 28,      # R x                                     W samples
    "integrate_key": 60,         # R x,v,a                                 W x,v
    "sort": 84,                  # R x,key,idx; permute x,v,ids
    "order_lists": 128,          # R lists (about 64 B) W lists
}


def parse():
    p = argparse.ArgumentParser()
    p.add_argument("--gpus", type=int, default=1)
    p.add_argument("--steps", type=int, default=200)
    p.add_argument("--warmup", type=int, default=3)
    p.add_argument("--impl", default="engine", choices=["engine", "reference"])
    p.add_argument("--n-side", type=int, default=100)
    p.add_argument("--max-iters", type=int, default=100)
    p.add_argument("--cpu-steps", type=int, default=2,
                   help="timed CPU-baseline steps at least (more while under --cpu-seconds)")
    p.add_argument("--cpu-seconds", type=float, default=15.0)
    p.add_argument("--ref-seconds", type=float, default=150.0,
                   help="reference arm: stop timing after this much CPU time (at least one step)")
    p.add_argument("--no-f64", action="store_true", help="skip the f64-twin engine timing")
    p.add_argument("--no-cpu-baseline", action="store_true")
    p.add_argument("--no-e2e", action="store_true")
    p.add_argument("--serving-requests", type=int, default=256,
                   help="scene-sweep requests served batched and one at a time (0: skip)")
    p.add_argument("--serving-plain-requests", type=int, default=-1,
                   help="requests of both serving arms, the first ones of the sweep (-1: all)")
    p.add_argument("--serving-steps", type=int, default=500)
    p.add_argument("--study", choices=["sesph8k", "ball", "tank"],
                   help="run one configuration study instead of the benchmark: 'sesph8k' (8k SESPH "
                        "dam break, 1,000 steps against the oracle, and the CPU path timed), 'ball' "
                        "(4M IISPHwOST two-fluid ball, f32 against the f64 engine, per-field errors), "
                        "'tank' (2M IISPH tank with 8 coupled bodies, 1,500 CFL steps, f32 against f64)")
    p.add_argument("--study-steps", type=int, default=0, help="steps of the study (0: its configuration's)")
    return p.parse_args()


def scene(n_side, max_iters, box=(2.0, 1.0, 1.0)):
    from sphgpu import scenes
    sc = scenes.dam_break_iisph_box(n_side=n_side, box=box)
    sc.parameters = dict(sc.parameters, max_solver_iterations=max_iters)
    return sc


class ClockSampler:
    """nvidia-smi clock / throttle sampling during the timed region."""

    QUERY = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device):
        self.device = device
        self.proc = None
        self.lines = []

    def start(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.device), f"--query-gpu={self.QUERY}",
                 "--format=csv,noheader,nounits", "-lms", "50"],
                stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.thread = threading.Thread(target=self._read, daemon=True)
            self.thread.start()
        except OSError:
            self.proc = None

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def stop(self):
        if not self.proc:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        sm, smax, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            parts = [p.strip() for p in ln.split(",")]
            if len(parts) < 9:
                continue
            try:
                sm.append(float(parts[1]))
                smax = float(parts[2])
            except ValueError:
                continue
            for nm, val in zip(names, parts[5:9]):
                if val.lower() == "active":
                    reasons.add(nm)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": smax,
                "reasons": sorted(reasons), "samples": len(sm)}


def dist_env():
    ws = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return ws, rank, local


def peaks():
    path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(path):
        with open(path) as f:
            d = json.load(f)
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


def oracle_module():
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle
    return oracle


def oracle_system(sc, fields=None):
    """The oracle (f64 restatement of the reference CPU path) set up with
    `sc`'s fluid, sample boundaries and, when given, the (sdf, vm) fields of
    its container, initialized (first update done)."""
    O = oracle_module()
    from sphgpu.system import PROCEDURES
    cfg = dict(sc.parameters)
    cfg.pop("device", None)
    cfg.pop("neighbor_capacity", None)
    cfg.setdefault("max_solver_iterations", 0)
    cfg.setdefault("time_increment", 0.0)
    cfg.update(integration_scheme=PROCEDURES["integration_scheme"][sc.procedures["integration_scheme"]],
               pressure_solver=PROCEDURES["pressure_solver"][sc.procedures["pressure_solver"]],
               boundary_handling=PROCEDURES["boundary_handling"][sc.procedures["boundary_handling"]],
               cfl_time_step=1 if sc.cfl_time_step else 0)
    s = O.OracleSystem(cfg)
    s.upload_fluid(sc.position, sc.velocity, sc.mass, sc.fluid_id)
    for pts, rigid in sc.sample_boundaries:
        s.add_sample_boundary(pts, None if rigid is None else rigid.to_array32())
    if fields is not None:
        s.add_volume_map_boundary(*(O.Field(f.x_min, f.x_max, f.dx, f.n, f.nodes) for f in fields))
    s.initialize()
    return s


def run_cpu(args, fields, min_steps, stop_seconds):
    """The reference's CPU algorithm (oracle restatement, f64, all host
    threads) on the benchmark scene: the same seeded state and fields, the
    same `args.warmup` untimed steps, then the timed steps: `args.steps` of
    them, or fewer once at least `min_steps` have run and `stop_seconds` of
    CPU time have been timed. Returns (updates/s, seconds, cores, particles,
    steps timed, sweeps per timed step)."""
    O = oracle_module()
    sc = scene(args.n_side, args.max_iters)
    s = oracle_system(sc, fields)
    if args.warmup:
        s.step(args.warmup)
    t0 = time.perf_counter()
    updates, done, sweeps = 0, 0, []
    while done < args.steps:
        if done >= min_steps and time.perf_counter() - t0 >= stop_seconds:
            break
        s.step(1)
        updates += s.n
        done += 1
        sweeps.append(int(s.measurement()["solver_iterations"]))
    dt = time.perf_counter() - t0
    return updates / dt, dt, O.num_threads(), sc.position.shape[0], done, sweeps


def _pct(values, q):
    return float(np.percentile(np.asarray(values, np.float64), q)) if len(values) else None


def serving_sweep(args, device, rank, ws):
    """The scene sweep (Poisson arrivals at 20/s, 5k-500k particles, SESPH or
    IISPH, 500 steps each) served two ways on this GPU, the same requests in
    both: batched by the scene server (continuous admission, concurrent
    graph-captured scenes) and one scene at a time through the plain
    single-scene C ABI path, in arrival order. Scenes/s = completed scenes / (last completion - first arrival);
    latency = completion - arrival. The first requests of both arms keep their
    final state, which must agree bit for bit."""
    import torch
    from sphgpu import scenes
    from sphgpu.replicas import aggregate, share
    from sphgpu.server import SceneServer
    reqs = share(scenes.scene_sweep(count=args.serving_requests, steps=args.serving_steps), rank, ws)
    if args.serving_plain_requests >= 0:
        reqs = reqs[:args.serving_plain_requests]
    built = [r.scene() for r in reqs]
    n_check = min(4, len(reqs))

    srv = SceneServer(device=device)
    t0 = time.perf_counter()
    tickets = []
    for k, (r, sc) in enumerate(zip(reqs, built)):
        wait = t0 + r.arrival_s - time.perf_counter()
        if wait > 0:
            time.sleep(wait)
        tickets.append(srv.submit(sc, r.steps, keep_state=k < n_check))
    res = [srv.wait(t, -1) for t in tickets]
    kept = [srv.fetch_state(t, x["particles"]) for t, x in zip(tickets[:n_check], res[:n_check])]
    st = srv.stats()
    srv.close()
    span = max(x["finish_s"] for x in res) - min(x["submit_s"] for x in res)
    lat = [x["latency_s"] for x in res]
    pu = sum(x["particles"] * x["steps"] for x in res)
    span_ms, done = aggregate(span * 1000.0, len(res), device="cuda")
    batched = {"scenes_per_s": done / (span_ms / 1000.0), "span_s": span_ms / 1000.0,
               "p50_s": _pct(lat, 50), "p95_s": _pct(lat, 95), "p99_s": _pct(lat, 99),
               "particle_updates_per_s": pu / span, "peak_active": st["peak_active"],
               "graph_replays": st["graph_replays"], "kernel_launches": st["kernel_launches"],
               "statuses": sorted({x["status"] for x in res})}

    m = len(reqs)
    from sphgpu import capi
    t0 = time.perf_counter()
    lat, same, service, step_s = [], 0, [], []
    for k, (r, sc) in enumerate(zip(reqs[:m], built[:m])):
        ta = t0 + r.arrival_s
        wait = ta - time.perf_counter()
        if wait > 0:
            time.sleep(wait)
        ts = time.perf_counter()
        g = scenes.build_system(sc, device=device)
        gs = torch.cuda.ExternalStream(g.stream(), device=device)
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(gs)
        g.step_forward_in_time(r.steps)
        e1.record(gs)
        g.take_measurement()
        e1.synchronize()
        step_s.append(e0.elapsed_time(e1) / 1000.0)
        if k < n_check:
            same += int(np.array_equal(g.download(capi.FIELD_POSITION), kept[k][0]) and
                        np.array_equal(g.download(capi.FIELD_VELOCITY), kept[k][1]))
        g.close()
        te = time.perf_counter()
        service.append(te - ts)
        lat.append(te - ta)
    span = time.perf_counter() - (t0 + reqs[0].arrival_s) if m else 0.0
    span_ms, done = aggregate(span * 1000.0, m, device="cuda")
    plain = {"scenes_per_s": done / (span_ms / 1000.0) if span_ms else None, "span_s": span_ms / 1000.0,
             "requests": m, "p50_s": _pct(lat, 50), "p95_s": _pct(lat, 95), "p99_s": _pct(lat, 99),
             "service_s": sum(service)}
    # Where the batched time goes: the device time of the step loops of the
    # scenes of 50k particles and more, each run alone (CUDA events on its
    # stream in the plain arm), and plain span / that time, the ratio batching
    # would reach if every smaller scene and all setup cost nothing and the
    # large scenes did not overlap one another. Scenes below about 190k
    # particles (fewer blocks than the GPU holds at once) do overlap, so the
    # batched arm can exceed it.
    big = [k for k in range(m) if built[k].position.shape[0] >= 50000]
    big_s = sum(step_s[k] for k in big)
    split = {"scenes_50k_up": len(big), "step_device_s_50k_up": big_s,
             "step_device_s_under_50k": sum(step_s) - big_s,
             "service_s_50k_up": sum(service[k] for k in big),
             "ratio_if_small_scenes_free_and_large_serial": (span_ms / 1000.0) / big_s if big_s else None}
    return {"metric": "scenes/s (Poisson scene sweep, batched server vs one-at-a-time plain GPU solves)",
            "requests": args.serving_requests, "arrival_rate_per_s": 20.0, "steps_per_scene": args.serving_steps,
            "particles_per_scene": "log-uniform 5k-500k (cubic blocks)", "solvers": "SESPH / IISPH 50:50",
            "batched": batched, "plain": plain, "device_split": split,
            "batched_over_plain": (batched["scenes_per_s"] / plain["scenes_per_s"]) if plain["scenes_per_s"] else None,
            "identical_final_state": f"{same}/{n_check if m >= n_check else min(m, n_check)}"}


WORKLOAD = ("IISPH dam break, {n}^3 particles at 0.01 m in a 2 x 1.02 x 1.02 m VolumeMapBoundary box "
            "(1.5-spacing wall gap), CFL dt <= 2e-3, omega 0.5, 0.1 % target density error")


def workload_config(args):
    return {"workload": WORKLOAD.format(n=args.n_side), "particles_per_gpu": args.n_side ** 3,
            "solver": "IISPH", "omega": 0.5, "target_density_error_pct": 0.1,
            "max_solver_iterations": args.max_iters, "cfl": 0.4, "max_dt": 2e-3,
            "initial_state": "seeded lattice + 1 % jitter (seed 0), then the warm-up steps"}


def gpu_fields(sc, device):
    from sphgpu.fields import build_volume_map_fields
    verts, faces = sc.mesh
    sp = sc.parameters["rest_density_grid_spacing"]
    return build_volume_map_fields(verts, faces, 4 * sp, sc.parameters["kernel_support_radius"], 30,
                                   device=device)


def time_steps(torch, sysm, steps, stream, clocks=None):
    """CUDA-event time of `steps` per-step calls on the engine's stream.
    Returns (ms, particle updates, sweeps per step)."""
    torch.cuda.synchronize()
    if clocks:
        clocks.start()
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    ev0.record(stream)
    updates, iters = 0, []
    for _ in range(steps):
        sysm.step_forward_in_time(1)
        st = sysm.step_stats()
        updates += st["particles"]
        iters.append(st["solver_iterations"])
    ev1.record(stream)
    torch.cuda.synchronize()
    return ev0.elapsed_time(ev1), updates, iters


def main():
    args = parse()
    ws, rank, local = dist_env()
    if args.study:
        return STUDIES[args.study](args, local)
    if args.impl == "reference":
        return reference_arm(args, ws, rank)
    import torch
    import torch.distributed as dist
    if ws > 1:
        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=__import__("datetime").timedelta(seconds=600))
    torch.cuda.set_device(local)
    from sphgpu import capi, scenes

    sc = scene(args.n_side, args.max_iters)
    fields = gpu_fields(sc, local)
    sysm = scenes.build_system(sc, precision="f32", device=local, fields=fields)
    stream = torch.cuda.ExternalStream(sysm.stream(), device=local)
    for _ in range(args.warmup):
        sysm.step_forward_in_time(1)
    # Copies of the warmed-up state: the kernel times and the end-to-end
    # number run exactly the steps the device-timed region runs.
    sys_prof = sysm.clone()
    sys_e2e = None if args.no_e2e else sysm.clone()
    launches0 = sysm.launch_count()
    if ws > 1:
        torch.cuda.synchronize()
        dist.barrier()
    clocks = ClockSampler(local)
    ms, updates, iters = time_steps(torch, sysm, args.steps, stream, clocks)
    clk = clocks.stop()
    launches = sysm.launch_count() - launches0
    # Per-kernel CUDA-event times of the same steps on the first copy. Timed
    # solves run one sweep per host check, so every timed sweep launch is a
    # sweep the solve needed (no launch that finds the loop converged).
    sys_prof.set_profiling(True)
    prof_iters = []
    for _ in range(args.steps):
        sys_prof.step_forward_in_time(1)
        prof_iters.append(sys_prof.step_stats()["solver_iterations"])
    kernel_times = {}
    for name in BYTES_PER_PARTICLE:
        kt = sys_prof.kernel_time(name)
        if kt:
            kernel_times[name] = kt
    sys_prof.close()
    # whole-job aggregate: sum of updates over ranks / max time over ranks
    from sphgpu.replicas import aggregate
    ms_max, total_updates = aggregate(ms, updates, device="cuda")
    value = total_updates / (ms_max / 1000.0)

    # e2e: the plugin call with host buffers (reference order), copies inside
    e2e = None
    if sys_e2e is not None:
        n = sys_e2e.n
        e_stream = torch.cuda.ExternalStream(sys_e2e.stream(), device=local)
        xin = torch.empty((n, 3), dtype=torch.float64).pin_memory()
        vin = torch.empty((n, 3), dtype=torch.float64).pin_memory()
        xout = torch.empty((n, 3), dtype=torch.float64).pin_memory()
        vout = torch.empty((n, 3), dtype=torch.float64).pin_memory()
        xin.numpy()[:] = sys_e2e.download(capi.FIELD_POSITION)
        vin.numpy()[:] = sys_e2e.download(capi.FIELD_VELOCITY)
        torch.cuda.synchronize()
        if ws > 1:
            dist.barrier()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(e_stream)
        e_updates = 0
        for _ in range(args.steps):
            sys_e2e.step_host(1, xin, vin, xout, vout)
            e_updates += sys_e2e.n
            xin, xout = xout, xin
            vin, vout = vout, vin
        e1.record(e_stream)
        torch.cuda.synchronize()
        ems = e0.elapsed_time(e1)
        sys_e2e.close()
        ems, e_updates = aggregate(ems, e_updates, device="cuda")
        e2e = {"value": e_updates / (ems / 1000.0), "unit": UNIT,
               "h2d_bytes_per_step": 2 * 3 * 8 * n, "d2h_bytes_per_step": 2 * 3 * 8 * n}

    # the f64 twin of every kernel on the same scene and steps (the reference's
    # own precision), device time
    f64 = None
    if not args.no_f64:
        s64 = scenes.build_system(sc, precision="f64", device=local, fields=fields)
        for _ in range(args.warmup):
            s64.step_forward_in_time(1)
        st64 = torch.cuda.ExternalStream(s64.stream(), device=local)
        ms64, upd64, it64 = time_steps(torch, s64, args.steps, st64)
        s64.close()
        ms64, upd64 = aggregate(ms64, upd64, device="cuda")
        f64 = {"value": upd64 / (ms64 / 1000.0), "unit": UNIT, "ms_per_step": ms64 / args.steps,
               "mean_solver_iterations": statistics.mean(it64) if it64 else None}

    peak, peak_kind = peaks()
    roofline = None
    if kernel_times:
        n_particles = updates / max(args.steps, 1)
        shares = {k: round(v[0] / sum(x[0] for x in kernel_times.values()), 4)
                  for k, v in sorted(kernel_times.items(), key=lambda kv: -kv[1][0])}
        dom = max(kernel_times, key=lambda k: kernel_times[k][0])
        tot_ms, cnt = kernel_times[dom]
        avg_s = tot_ms / cnt / 1000.0
        bytes_per_launch = BYTES_PER_PARTICLE[dom] * n_particles
        achieved = bytes_per_launch / avg_s / 1e9
        roofline = {"bound": "hbm", "kernel": dom, "achieved": round(achieved, 1), "peak": peak,
                    "peak_kind": peak_kind, "unit": "GB/s", "frac": round(achieved / peak, 4),
                    "traffic": None,
                    "traffic_note": "DRAM bytes per launch come from ncu captures (profiles/), not from this run",
                    "bytes_per_launch": bytes_per_launch, "avg_launch_us": round(avg_s * 1e6, 2),
                    "launches": cnt, "kernel_share": shares}
        if "iisph_jacobi" in kernel_times and "iisph_pressure_accel" in kernel_times:
            # one Jacobi sweep = pass A (pressure accelerations) + pass B
            # (pressure update and residual): 52 + 60 B per particle
            ta, ca = kernel_times["iisph_pressure_accel"]
            tb, cb = kernel_times["iisph_jacobi"]
            sweeps = sum(prof_iters)
            pair_s = (ta / ca + tb / cb) / 1000.0
            pair_bytes = (BYTES_PER_PARTICLE["iisph_pressure_accel"] + BYTES_PER_PARTICLE["iisph_jacobi"]) * n_particles
            roofline["sweep"] = {"sweeps_run": sweeps, "pass_a_launches": ca, "pass_b_launches": cb,
                                 "pass_a_us": round(ta / ca * 1000.0, 2), "pass_b_us": round(tb / cb * 1000.0, 2),
                                 "bytes_per_sweep": pair_bytes,
                                 "achieved": round(pair_bytes / pair_s / 1e9, 1),
                                 "frac": round(pair_bytes / pair_s / 1e9 / peak, 4)}

    cpu = None
    if rank == 0 and not args.no_cpu_baseline:
        v, secs, cores, n_cpu, done, sweeps = run_cpu(args, fields, args.cpu_steps, args.cpu_seconds)
        cpu = {"value": v, "unit": UNIT, "cores": cores, "kind": "port",
               "sample": f"steps {args.warmup + 1}-{args.warmup + done} of the same {n_cpu}-particle scene "
                         f"(same seeded state and fields, {args.warmup} untimed warm-up steps), "
                         f"{statistics.mean(sweeps):.1f} IISPH sweeps per step {sweeps}, f64 C++ restatement "
                         f"of the reference CPU path on all host threads, {secs:.1f} s"}

    sysm.close()
    serving = serving_sweep(args, local, rank, ws) if args.serving_requests > 0 else None
    if ws > 1:
        dist.barrier()
    if rank == 0:
        cfg = workload_config(args)
        cfg.update({"precision": "f32 state, f64 reductions", "parallelism": f"replicas x{ws}",
                    "l2": "no flush: a step touches about 260 MB of distinct data (> 126 MB L2)",
                    "mean_solver_iterations": statistics.mean(iters) if iters else None,
                    "solver_iterations": iters})
        line = {
            "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": ws, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": ms_max / args.steps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic (seeded lattice + jitter)",
            "config": cfg, "gpu_launches": launches, "clocks": clk, "roofline": roofline, "cpu_baseline": cpu,
            "e2e": e2e, "f64_engine": f64, "serving": serving,
        }
        print(json.dumps(line))
    if ws > 1:
        dist.destroy_process_group()


def reference_arm(args, ws, rank):
    """The reference's CPU algorithm on the benchmark scene itself (f64 C++
    restatement; the Rust reference cannot be built here). Fields are built
    by the oracle's CPU restatement of the reference's field construction."""
    if rank != 0:
        return
    O = oracle_module()
    sc = scene(args.n_side, args.max_iters)
    verts, faces = sc.mesh
    sp = sc.parameters["rest_density_grid_spacing"]
    t0 = time.perf_counter()
    fields = O.build_fields(verts, faces, 4 * sp, sc.parameters["kernel_support_radius"], 30)
    t_fields = time.perf_counter() - t0
    v, secs, cores, n_cpu, done, sweeps = run_cpu(args, fields, 1, args.ref_seconds)
    cfg = workload_config(args)
    cfg.update({"precision": "f64", "steps_timed": done,
                "mean_solver_iterations": statistics.mean(sweeps) if sweeps else None,
                "solver_iterations": sweeps})
    line = {
        "metric": METRIC, "value": v, "unit": UNIT, "n_gpus": ws, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": secs * 1000.0 / max(done, 1), "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic (seeded lattice + jitter)",
        "impl": "reference", "config": cfg,
        "cpu_baseline": {"value": v, "unit": UNIT, "cores": cores, "kind": "port",
                         "sample": f"steps {args.warmup + 1}-{args.warmup + done} of the {n_cpu}-particle scene "
                                   f"after {args.warmup} untimed warm-up steps"
                                   f"{'' if done == args.steps else f' (the first {done} of the {args.steps} steps: --ref-seconds ran out)'}, "
                                   f"{statistics.mean(sweeps):.1f} IISPH sweeps per step; f64 C++ restatement of "
                                   f"the reference CPU path (the Rust reference cannot be built here); fields built "
                                   f"on the CPU in {t_fields:.0f} s, untimed"},
        "e2e": {"value": v, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line))


# ---------------------------------------------------------------------------
# Configuration studies (one JSON line each)
# ---------------------------------------------------------------------------
def _field_errors(A, got, ref, spacing):
    """Per-field errors of a run (`got`) against a reference run (`ref`)."""
    def mx(a):
        return float(np.abs(a).max()) if a.size else 0.0
    out = {}
    out["position_max_over_spacing"] = mx(got[A.FIELD_POSITION] - ref[A.FIELD_POSITION]) / spacing
    out["position_rms_over_spacing"] = float(np.sqrt(np.mean(np.sum(
        (got[A.FIELD_POSITION] - ref[A.FIELD_POSITION]) ** 2, axis=1)))) / spacing
    out["velocity_max_rel_to_max"] = mx(got[A.FIELD_VELOCITY] - ref[A.FIELD_VELOCITY]) / max(mx(ref[A.FIELD_VELOCITY]), 1e-30)
    if A.FIELD_VOLUME in ref:
        out["volume_max_rel"] = float(np.max(np.abs(got[A.FIELD_VOLUME] - ref[A.FIELD_VOLUME]) /
                                             np.abs(ref[A.FIELD_VOLUME])))
    if A.FIELD_PRESSURE in ref:
        out["pressure_max"] = mx(ref[A.FIELD_PRESSURE])
        out["pressure_max_rel_to_max"] = mx(got[A.FIELD_PRESSURE] - ref[A.FIELD_PRESSURE]) / max(mx(ref[A.FIELD_PRESSURE]), 1e-30)
        out["pressure_rms_rel_to_max"] = float(np.sqrt(np.mean((got[A.FIELD_PRESSURE] - ref[A.FIELD_PRESSURE]) ** 2))) / max(mx(ref[A.FIELD_PRESSURE]), 1e-30)
    if A.FIELD_ACCELERATION in ref:
        out["acceleration_max_rel_to_max"] = mx(got[A.FIELD_ACCELERATION] - ref[A.FIELD_ACCELERATION]) / max(mx(ref[A.FIELD_ACCELERATION]), 1e-30)
    return {k: float(f"{v:.3e}") for k, v in out.items()}


def _grab(sysm, A, fields):
    return {f: sysm.download(f) for f in fields}


def study_sesph8k(args, device):
    """Configuration 1: the 8,000-particle SESPH dam break (sample-boundary
    container, fixed dt 1e-3) for 1,000 steps on the f32 engine and on the
    oracle (the reference's CPU path, timed: the CPU-1 baseline), with the
    drift between them every 100 steps."""
    import torch
    O = oracle_module()
    from sphgpu import _capi as A, scenes
    steps = args.study_steps or 1000
    sc = scenes.dam_break_sesph_8k()
    g = scenes.build_system(sc, precision="f32", device=device)
    o = oracle_system(sc)
    h = sc.parameters["rest_density_grid_spacing"]
    stream = torch.cuda.ExternalStream(g.stream(), device=device)
    rows, gpu_ms, cpu_s = [], 0.0, 0.0
    for k in range(0, steps, 100):
        n = min(100, steps - k)
        ms, _, _ = time_steps(torch, g, n, stream)
        gpu_ms += ms
        t0 = time.perf_counter()
        o.step(n)
        cpu_s += time.perf_counter() - t0
        mg, mo = g.take_measurement(), o.measurement()
        got = _grab(g, A, (A.FIELD_POSITION, A.FIELD_VELOCITY, A.FIELD_VOLUME))
        ref = {A.FIELD_POSITION: o.download(O.F_POSITION), A.FIELD_VELOCITY: o.download(O.F_VELOCITY),
               A.FIELD_VOLUME: o.download(O.F_VOLUME)}
        row = {"step": k + n, **_field_errors(A, got, ref, h),
               "density_rel": float(f"{abs(mg['density'] - mo['density']) / mo['density']:.3e}"),
               "kinetic_energy_rel": float(f"{abs(mg['kinetic_energy'] - mo['kinetic_energy']) / max(mo['kinetic_energy'], 1e-30):.3e}")}
        rows.append(row)
    n = g.n
    print(json.dumps({"study": "sesph8k", "particles": n, "steps": steps,
                      "engine_f32_updates_per_s": n * steps / (gpu_ms / 1000.0),
                      "cpu_updates_per_s": n * steps / cpu_s, "cpu_cores": O.num_threads(),
                      "cpu_kind": "f64 C++ restatement of the reference CPU path (CPU-1)",
                      "drift": rows}))


def study_ball(args, device):
    """Configuration 3: the IISPHwOST two-fluid ball, 4M particles in the
    lower half of a radius-1 m sphere (inward icosphere of 5,120 triangles,
    fields at dx 0.032), rest densities 1000 / 500 split by a seeded plane,
    TakePredicted at dt 5e-4 for 500 steps. The f32 engine runs against its
    f64 twin from the same state; per-field errors every 100 steps."""
    from sphgpu import _capi as A, scenes
    steps = args.study_steps or 500
    sc = scenes.two_fluid_ball(radius=1.0, spacing=0.008, seed=0, subdivisions=4)
    sc.parameters = dict(sc.parameters, max_solver_iterations=args.max_iters)
    t0 = time.perf_counter()
    fields = gpu_fields(sc, device)
    t_fields = time.perf_counter() - t0
    g32 = scenes.build_system(sc, precision="f32", device=device, fields=fields)
    g64 = scenes.build_system(sc, precision="f64", device=device, fields=fields)
    keep = (A.FIELD_POSITION, A.FIELD_VELOCITY, A.FIELD_VOLUME, A.FIELD_PRESSURE, A.FIELD_ACCELERATION)
    rows = []
    t32 = t64 = 0.0
    for k in range(0, steps, 100):
        n = min(100, steps - k)
        t0 = time.perf_counter(); g32.step_forward_in_time(n); t32 += time.perf_counter() - t0
        t0 = time.perf_counter(); g64.step_forward_in_time(n); t64 += time.perf_counter() - t0
        m32, m64 = g32.take_measurement(), g64.take_measurement()
        rows.append({"step": k + n, **_field_errors(A, _grab(g32, A, keep), _grab(g64, A, keep),
                                                    sc.parameters["rest_density_grid_spacing"]),
                     "sweeps_f32": m32["solver_iterations"], "sweeps_f64": m64["solver_iterations"],
                     "density_error_f32": m32["density_error"], "density_error_f64": m64["density_error"]})
        print(json.dumps(rows[-1]), file=sys.stderr, flush=True)
    print(json.dumps({"study": "ball", "particles": g32.n, "steps": steps, "fields_s": round(t_fields, 1),
                      "f32_ms_per_step": 1000.0 * t32 / steps, "f64_ms_per_step": 1000.0 * t64 / steps,
                      "errors_f32_vs_f64": rows}))


def study_tank(args, device):
    """Configuration 4: IISPH tank with eight two-way coupled bodies (4 cubes
    of side 0.15 m, 4 spheres of radius 0.08 m, densities U[300, 1500]), all
    StaticSampleBoundary, 2M fluid particles at 0.01 m (a 2 x 1 x 1.5 m tank
    filled to 1.03 m, the bodies above the surface), CFL steps; f32 engine
    against its f64 twin, body states and fluid fields every 100 steps."""
    from sphgpu import _capi as A, scenes
    steps = args.study_steps or 1500
    sc = scenes.rigid_body_tank(spacing=0.01, tank=(2.0, 1.0, 1.5), fill=1.03, seed=0)
    sc.parameters = dict(sc.parameters, max_solver_iterations=args.max_iters)
    g32 = scenes.build_system(sc, precision="f32", device=device)
    g64 = scenes.build_system(sc, precision="f64", device=device)
    keep = (A.FIELD_POSITION, A.FIELD_VELOCITY, A.FIELD_VOLUME, A.FIELD_PRESSURE)
    nb = len(sc.sample_boundaries)
    rows = []
    t32 = t64 = 0.0
    for k in range(0, steps, 100):
        n = min(100, steps - k)
        t0 = time.perf_counter(); g32.step_forward_in_time(n); t32 += time.perf_counter() - t0
        t0 = time.perf_counter(); g64.step_forward_in_time(n); t64 += time.perf_counter() - t0
        b32 = np.stack([g32.rigid_state(b) for b in range(1, nb)])
        b64 = np.stack([g64.rigid_state(b) for b in range(1, nb)])
        rows.append({"step": k + n, "time_f32": g32.time(), "time_f64": g64.time(),
                     "body_com_max_abs_m": float(f"{np.abs(b32[:, 0:3] - b64[:, 0:3]).max():.3e}"),
                     "body_q_max_abs": float(f"{np.abs(b32[:, 3:7] - b64[:, 3:7]).max():.3e}"),
                     "body_v_max_abs": float(f"{np.abs(b32[:, 7:10] - b64[:, 7:10]).max():.3e}"),
                     "body_com_travel_m": float(f"{np.abs(b64[:, 0:3] - np.array([r.center_of_mass for _, r in sc.sample_boundaries[1:]])).max():.3e}"),
                     **_field_errors(A, _grab(g32, A, keep), _grab(g64, A, keep),
                                     sc.parameters["rest_density_grid_spacing"]),
                     "sweeps_f32": g32.take_measurement()["solver_iterations"],
                     "sweeps_f64": g64.take_measurement()["solver_iterations"]})
        print(json.dumps(rows[-1]), file=sys.stderr, flush=True)
    print(json.dumps({"study": "tank", "particles": g32.n, "bodies": nb - 1, "steps": steps,
                      "f32_ms_per_step": 1000.0 * t32 / steps, "f64_ms_per_step": 1000.0 * t64 / steps,
                      "f32_vs_f64": rows}))


STUDIES = {"sesph8k": study_sesph8k, "ball": study_ball, "tank": study_tank}


if __name__ == "__main__":
    main()
