#!/usr/bin/env python
"""Throughput of solunar's particle-fluid substep on B200: one JSON line.

Workload: the one-million-particle DFSPH dam break (100^3 particles at 0.01 m, support 2, in a
2 x 1 x 1 m tank of boundary particles, jitter +-1e-5 m), advanced by FluidWorld::step(1e-3 s),
which takes as many DFSPH substeps as the flow needs.  A timed step is one such call; `value`
is substeps per second over all ranks, device-timed with CUDA events on the world's stream,
with the particle state resident in HBM and L2 flushed (a 256 MiB write) before each step.
Each DFSPH substep runs as one CUDA graph launch (sort, density, both solves with loops the
device ends, viscosity, advance), recorded when its launches first occur; the per-kernel
times of the roofline come from a second pass of the same steps with every launch timed by CUDA
events (the profiler runs the substep launch by launch).
`e2e` is the same metric through the C ABI with host-owned state: each step uploads positions
and velocities from pinned host memory, steps, and reads them back.
`forward_adjoint` tapes `--adjoint-steps` steps (every substep recorded, or a checkpoint every
`--adjoint-every` substeps) and runs step_backward; `warm_start` repeats the plain steps and,
with `--warm-adjoint-steps` (default: the same count), the forward+adjoint with warm-started
solves on a world of its own.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

N > 1 runs one independent replica per GPU under torchrun ("replicas only": the fluid step has
no exchange between GPUs), value = all ranks' substeps / the slowest rank's time.
`--impl reference` times the CPU restatement of the reference (the Rust reference cannot be
built here) on the host cores, on the same workload and metric.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import tempfile
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "1M-particle DFSPH substeps/s: plain vs fwd+adjoint, 0.1% density err, 1 B200"
UNIT = "substeps/s"
GRAPH_MODES = {0: "launch by launch, host-checked batches",
               1: "one CUDA graph per solve, loop ended on the device",
               2: "one CUDA graph per substep (sort, density, solves with device-ended loops, viscosity, advance)"}
FLUSH_BYTES = 256 << 20


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--scene", default="dfsph_dam_1m")
    ap.add_argument("--arithmetic", choices=["exact", "fast"], default="exact",
                    help="exact: the reference's rounding, bit-identical to the CPU restatement; "
                         "fast: fused arithmetic, within FP32 tolerance")
    ap.add_argument("--positions", choices=["absolute", "cell_relative"], default="absolute",
                    help="cell_relative: offsets from each particle's cell (FAST arithmetic, no adjoint)")
    ap.add_argument("--e2e-steps", type=int, default=10)
    ap.add_argument("--profile-steps", type=int, default=8,
                    help="steps of the per-kernel CUDA-event pass behind the roofline")
    ap.add_argument("--warm-steps", type=int, default=None,
                    help="timed steps of the opt-in warm-started leg on its own world, after the same "
                         "warm-up (default: --steps, the cold run's window; 0 skips it)")
    ap.add_argument("--no-graphs", action="store_true", help="queue the solves in host-checked batches")
    ap.add_argument("--graph-mode", type=int, default=2, choices=(0, 1, 2),
                    help="2 each substep one CUDA graph, 1 each solve one graph, 0 as --no-graphs")
    ap.add_argument("--adjoint-every", type=int, default=0,
                    help="tape checkpoint spacing of the forward+adjoint leg, in substeps; 0 records every "
                         "substep")
    ap.add_argument("--adjoint-steps", type=int, default=32,
                    help="steps of the forward+adjoint measurement (0 skips it)")
    ap.add_argument("--warm-adjoint-steps", type=int, default=None,
                    help="steps of the warm-started world's forward+adjoint (default: --adjoint-steps; 0 skips it)")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--cpu-budget", type=float, default=25.0, help="seconds of timed CPU work in the baseline")
    ap.add_argument("--no-density-error", action="store_true",
                    help="skip the FP64 restatement run behind the density error of the timed steps")
    return ap.parse_args()


def scene_of(name, arithmetic="exact", positions="absolute"):
    from solunar_b200 import scenes
    from solunar_b200.abi import Arithmetic, Positions

    sc = getattr(scenes, name)()
    sc.settings.arithmetic = Arithmetic.FAST if arithmetic == "fast" else Arithmetic.EXACT
    if positions == "cell_relative":
        sc.settings.positions = Positions.CELL_RELATIVE
        sc.settings.arithmetic = Arithmetic.FAST
    return sc


def workload(sc) -> dict:
    return {
        "workload": f"{sc.name}: {sc.particles} particles ({'x'.join(map(str, sc.block_counts))} at "
                    f"{sc.settings.spacing} m, support {sc.settings.support}) in a "
                    f"{'x'.join(map(str, sc.tank))} m tank, {sc.settings.solver.name}, step({sc.dt}) per timed step",
        "particles": sc.particles,
        "solver": sc.settings.solver.name,
        "arithmetic": sc.settings.arithmetic.name,
        "positions": sc.settings.positions.name,
        "solver_tolerances": {"divergence": sc.settings.divergence_tolerance, "density": sc.settings.density_tolerance},
        "warm_start": bool(sc.settings.warm_start),
        "l2": "flushed (256 MiB write) before every timed step",
    }


def peaks() -> dict:
    path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(path):
        with open(path) as f:
            d = json.load(f)
        return {"hbm_gbs": float(d["hbm_gbs"]), "source": "measured"}
    return {"hbm_gbs": 6650.0, "source": "fallback"}


def traffic_for(kernel: str, scene: str):
    """DRAM bytes per launch of `kernel` at this workload, from a committed ncu summary."""
    path = os.path.join(ROOT, "profiles", "traffic.json")
    if not os.path.exists(path):
        return None
    with open(path) as f:
        d = json.load(f)
    entry = d.get(scene, {}).get(kernel)
    return None if entry is None else float(entry["dram_bytes_per_launch"])


class Clocks:
    """SM clocks and clock-event reasons sampled while the timed region runs: through NVML every
    10 ms in a thread (reads only), or from `nvidia-smi -lms 200` where NVML is missing."""

    NAMES = ("hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap")

    def __init__(self, index: int):
        self.index = index
        self.rows = []
        self.thread = None
        self.proc = None
        self.done = None

    def start(self):
        try:
            import threading

            import pynvml

            pynvml.nvmlInit()
            h = pynvml.nvmlDeviceGetHandleByIndex(self.index)
            bits = (pynvml.nvmlClocksEventReasonHwSlowdown, pynvml.nvmlClocksEventReasonHwThermalSlowdown,
                    pynvml.nvmlClocksEventReasonSwThermalSlowdown, pynvml.nvmlClocksEventReasonSwPowerCap)
            self.done = threading.Event()
            self.max_mhz = float(pynvml.nvmlDeviceGetMaxClockInfo(h, pynvml.NVML_CLOCK_SM))

            def sample():
                while not self.done.is_set():
                    sm = float(pynvml.nvmlDeviceGetClockInfo(h, pynvml.NVML_CLOCK_SM))
                    active = pynvml.nvmlDeviceGetCurrentClocksEventReasons(h)
                    self.rows.append((sm, tuple(bool(active & b) for b in bits)))
                    self.done.wait(0.01)

            self.thread = threading.Thread(target=sample, daemon=True)
            self.thread.start()
        except Exception:  # no NVML: nvidia-smi's own polling
            self.thread = None
            self.file = tempfile.NamedTemporaryFile("w+", suffix=".csv", delete=False)
            fields = ("index,clocks.sm,clocks.max.sm,clocks_event_reasons.hw_slowdown,"
                      "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
                      "clocks_event_reasons.sw_power_cap")
            try:
                self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.index), f"--query-gpu={fields}",
                                              "--format=csv,noheader,nounits", "-lms", "200"],
                                             stdout=self.file, stderr=subprocess.DEVNULL)
            except OSError:
                self.proc = None

    def stop(self) -> dict:
        if self.thread is not None:
            self.done.set()
            self.thread.join(timeout=5)
            rows, mx = self.rows, self.max_mhz
        elif self.proc is not None:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()
            self.file.flush()
            rows, mx = [], None
            with open(self.file.name) as f:
                for line in f:
                    q = [x.strip() for x in line.split(",")]
                    if len(q) >= 7 and q[1].replace(".", "").isdigit():
                        rows.append((float(q[1]), tuple(v.lower() == "active" for v in q[3:7])))
                        mx = float(q[2]) if q[2].replace(".", "").isdigit() else mx
            os.unlink(self.file.name)
        else:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["no clock source"], "samples": 0}
        if not rows:
            return {"sm_mhz": None, "sm_max_mhz": mx, "reasons": ["no samples"], "samples": 0}
        reasons = sorted({self.NAMES[k] for _, act in rows for k in range(4) if act[k]})
        return {"sm_mhz": statistics.median(r[0] for r in rows), "sm_max_mhz": mx, "reasons": reasons,
                "samples": len(rows)}


def cpu_baseline(sc, budget_s: float, state=None, threads: int = 0) -> dict:
    """The CPU restatement (OpenMP over all host cores) on a bounded sample of the workload,
    continuing from `state` = (positions, velocities) in their sorted order when given: added in
    that order, the particles keep the same (cell, id) order and the same physics."""
    from oracle import py_oracle

    py_oracle.build()
    cores = threads or os.cpu_count()
    w = py_oracle.OracleWorld(sc.settings, residual_sum=0, threads=cores)
    if state is None:
        sc.build(w)
        where = "from rest"
    else:
        w.add_box_container((0.0, 0.0, 0.0), sc.tank)
        w.add_particles(state[0], state[1])
        where = "from the state the GPU's timed steps ended on"
    w.update_neighbors()
    substeps = iterations = 0
    t0 = time.perf_counter()
    steps = 0
    while True:
        r = w.step(sc.dt)
        substeps += r.substeps
        iterations += r.iterations
        steps += 1
        if time.perf_counter() - t0 >= budget_s:
            break
    dt = time.perf_counter() - t0
    return {"value": substeps / dt, "unit": UNIT, "cores": cores, "kind": "port",
            "solver_iterations_per_substep": iterations / max(substeps, 1),
            "sample": f"{steps} steps ({substeps} substeps) of the {sc.particles}-particle scene {where}, "
                      f"{dt:.1f} s on {cores} threads (C++ float restatement, OpenMP, the reference's f32 "
                      f"residual sum)"}


def density_error(sc, steps: int, gpu_ids, gpu_rho, threads: int = 0) -> dict:
    """Density error of the GPU run against the FP64 restatement of the same method: the double
    oracle from the same initial state over the same steps (warm-up and timed), then
    |rho - rho_64| / rho_0 particle by particle (matched by id)."""
    import numpy as np

    from oracle import py_oracle

    py_oracle.build()
    cores = threads or os.cpu_count()
    w = py_oracle.OracleWorld(sc.settings, precision=64, residual_sum=1, threads=cores)
    sc.build(w)
    t0 = time.perf_counter()
    its = subs = 0
    for _ in range(steps):
        r = w.step(sc.dt)
        its += r.iterations
        subs += r.substeps
    ids = w.ids()
    rho64 = np.empty(len(ids))
    rho64[ids] = w.densities()
    err = np.abs(np.asarray(gpu_rho, np.float64) - rho64[np.asarray(gpu_ids)]) / float(sc.settings.rest_density)
    return {"max": float(err.max()), "mean": float(err.mean()),
            "p99": float(np.quantile(err, 0.99)),
            "within_0p1_percent": bool(err.max() <= 1e-3),
            "fp64_solver_iterations_per_substep": its / max(subs, 1),
            "against": f"FP64 restatement (double, compensated residual) from the same initial state over the "
                       f"same {steps} steps (warm-up and timed), {time.perf_counter() - t0:.1f} s on {cores} "
                       f"threads; |rho - rho_64| / rho_0 by particle id after the last timed step"}


def run_reference(args, rank: int, world_size: int):
    if rank != 0:
        return
    sc = scene_of(args.scene)
    from oracle import py_oracle

    py_oracle.build()
    cores = os.cpu_count()

    def leg(residual_sum: int, budget: float):
        """Warm-up then timed steps of the restatement: (steps, substeps, iterations, seconds)."""
        w = py_oracle.OracleWorld(sc.settings, residual_sum=residual_sum, threads=cores)
        sc.build(w)
        w.update_neighbors()
        t_start = time.perf_counter()
        for _ in range(args.warmup):
            w.step(sc.dt)
            if time.perf_counter() - t_start > budget / 3:
                break
        substeps = iterations = steps = 0
        t0 = time.perf_counter()
        for _ in range(args.steps):
            r = w.step(sc.dt)
            substeps += r.substeps
            iterations += r.iterations
            steps += 1
            if time.perf_counter() - t0 > budget:
                break
        return steps, substeps, iterations, time.perf_counter() - t0

    # the reference's own stop test: the solver error summed in f32, sequentially (dfsph.rs:263-267)
    steps, substeps, iterations, dt = leg(0, 150.0)
    value = substeps / dt
    # beside it, the same steps with the compensated FP64 sum the CUDA library takes, so both
    # arms' solver iterations can be compared step for step
    c_steps, c_sub, c_its, c_dt = leg(1, 60.0)
    sample = (f"{steps} of {args.steps} timed steps ({substeps} substeps) of the {sc.particles}-particle scene, "
              f"{dt:.1f} s on {cores} threads (C++ float restatement of the reference, OpenMP; the Rust "
              f"reference has no toolchain here)")
    out = {"metric": METRIC, "value": value, "unit": UNIT, "impl": "reference", "n_gpus": world_size,
           "steps": steps, "warmup": args.warmup, "ms_per_step": dt * 1e3 / max(steps, 1),
           "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
           "data": "synthetic",
           "config": dict(workload(sc), substeps=substeps,
                          solver_iterations_per_substep=iterations / max(substeps, 1),
                          solver_iterations_per_s=iterations / dt,
                          residual_sum="f32 sequential (the reference's, dfsph.rs:263-267)"),
           "compensated_residual_leg": {"value": c_sub / c_dt, "unit": UNIT, "steps": c_steps, "substeps": c_sub,
                                        "solver_iterations_per_substep": c_its / max(c_sub, 1),
                                        "solver_iterations_per_s": c_its / c_dt,
                                        "residual_sum": "compensated FP64 (the CUDA library's)"},
           "cpu_baseline": {"value": value, "unit": UNIT, "cores": cores, "kind": "port", "sample": sample},
           "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(out), flush=True)


def main():
    args = parse()
    rank = int(os.environ.get("RANK", "0"))
    world_size = int(os.environ.get("WORLD_SIZE", "1"))
    local_rank = int(os.environ.get("LOCAL_RANK", "0"))
    if args.impl == "reference":
        run_reference(args, rank, world_size)
        return
    graph_mode = 0 if args.no_graphs else args.graph_mode

    import torch
    import torch.distributed as dist

    torch.cuda.set_device(local_rank)
    dev = torch.device("cuda", local_rank)
    if world_size > 1:
        import datetime

        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300))

    def barrier():
        if world_size > 1:
            dist.barrier(device_ids=[local_rank])
        torch.cuda.synchronize()

    from solunar_b200 import fluid
    from solunar_b200.replicas import reduce_timing

    sc = scene_of(args.scene, args.arithmetic, args.positions)
    sc.settings.device = local_rank
    world = fluid.FluidWorld(sc.settings)
    world.solver_graphs(graph_mode)
    sc.build(world)
    world.update_neighbors()
    stream = torch.cuda.ExternalStream(world.stream(), device=dev)
    flush = torch.empty(FLUSH_BYTES // 4, dtype=torch.float32, device=dev)

    for _ in range(max(args.warmup, 3)):
        world.step(sc.dt)

    clocks = Clocks(local_rank)
    clocks.start()
    launches0 = fluid.kernel_launches()
    graphed0 = world.graph_substeps()
    barrier()
    times_ms = []
    substeps = iterations = 0
    for _ in range(args.steps):
        flush.zero_()
        torch.cuda.synchronize()
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        r = world.step(sc.dt)
        e1.record(stream)
        e1.synchronize()
        times_ms.append(e0.elapsed_time(e1))
        substeps += r.substeps
        iterations += r.iterations
    barrier()
    launches = fluid.kernel_launches() - launches0
    graphed = world.graph_substeps() - graphed0
    clock_info = clocks.stop()
    # the state the timed steps ended on, for the density error against the FP64 restatement
    timed_end = (world.ids(), world.densities()) if rank == 0 and world_size == 1 else None

    all_substeps, total_ms = reduce_timing(substeps, sum(times_ms), world_size, dev)
    value = all_substeps / (total_ms / 1e3)

    # the per-kernel pass: the next steps of the same run, each launch timed with CUDA events
    world.profile(True)
    world.profile_reset()
    prof_substeps = prof_iterations = 0
    prof_ms = 0.0
    for _ in range(max(args.profile_steps, 1)):
        flush.zero_()
        torch.cuda.synchronize()
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        r = world.step(sc.dt)
        e1.record(stream)
        e1.synchronize()
        prof_ms += e0.elapsed_time(e1)
        prof_substeps += r.substeps
        prof_iterations += r.iterations
    prof = world.profile_read()
    world.profile(False)

    # roofline of the kernel with the largest share of device time
    pk = peaks()
    dominant = max(prof.items(), key=lambda kv: kv[1][1])
    name, (count, ms, abytes) = dominant
    avg_ms = ms / max(count, 1)
    per_launch = abytes / max(count, 1)
    achieved = per_launch / (avg_ms / 1e3) / 1e9
    traffic = traffic_for(name, sc.name)
    kernel_ms = sum(v[1] for v in prof.values())
    all_bytes = sum(v[2] for v in prof.values())
    roofline = {"bound": "hbm", "kernel": name, "achieved": achieved, "peak": pk["hbm_gbs"], "unit": "GB/s",
                "frac": achieved / pk["hbm_gbs"], "peak_source": pk["source"], "traffic": traffic,
                # the DRAM bytes the kernel moves (ncu, per launch; mostly neighbour lists) over its
                # event-timed launch: how busy HBM is, beside the algorithmic fraction above
                "traffic_gbs": traffic / (avg_ms / 1e3) / 1e9 if traffic else None,
                "traffic_frac": traffic / (avg_ms / 1e3) / 1e9 / pk["hbm_gbs"] if traffic else None,
                "algorithmic_bytes_per_launch": per_launch, "avg_launch_ms": avg_ms,
                "share_of_kernel_time": ms / kernel_ms if kernel_ms else None,
                "substep_algorithmic_gbs": (all_bytes / max(prof_substeps, 1)) * substeps / (sum(times_ms) / 1e3) / 1e9,
                "profiled": {"steps": max(args.profile_steps, 1), "substeps": prof_substeps,
                             "solver_iterations_per_substep": prof_iterations / max(prof_substeps, 1),
                             "ms_per_substep_launch_by_launch": prof_ms / max(prof_substeps, 1),
                             "kernel_ms_per_substep": kernel_ms / max(prof_substeps, 1)},
                "kernels": {k: {"launches": v[0], "ms": v[1], "gbs": (v[2] / v[0]) / (v[1] / v[0] / 1e3) / 1e9
                                if v[0] and v[1] else None} for k, v in prof.items()}}

    # end to end through the C ABI with host-owned state in pinned memory
    n = world.len()
    host_pos = torch.empty((n, 3), dtype=torch.float32).pin_memory()
    host_vel = torch.empty((n, 3), dtype=torch.float32).pin_memory()
    world.read_positions_ptr(host_pos.data_ptr(), n)
    world.read_velocities_ptr(host_vel.data_ptr(), n)
    # untimed round trips first: a state written from the host lands in another position slot, so
    # the substep graphs of that slot rotation are recorded here, not inside the timed steps
    for _ in range(3):
        world.write_state_ptr(host_pos.data_ptr(), host_vel.data_ptr(), n)
        world.step(sc.dt)
        world.read_state_ptr(host_pos.data_ptr(), host_vel.data_ptr(), n)
    barrier()
    e2e_ms = 0.0
    e2e_substeps = 0
    for _ in range(args.e2e_steps):
        flush.zero_()
        torch.cuda.synchronize()
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        world.write_state_ptr(host_pos.data_ptr(), host_vel.data_ptr(), n)
        r = world.step(sc.dt)
        world.read_state_ptr(host_pos.data_ptr(), host_vel.data_ptr(), n)
        e1.record(stream)
        e1.synchronize()
        e2e_ms += e0.elapsed_time(e1)
        e2e_substeps += r.substeps
    barrier()
    e2e_all, e2e_ms = reduce_timing(e2e_substeps, e2e_ms, world_size, dev)
    e2e = {"value": e2e_all / (e2e_ms / 1e3), "unit": UNIT, "h2d_bytes_per_step": 24 * n,
           "d2h_bytes_per_step": 24 * n}

    # forward + adjoint (step_backward) on the same world: a taped forward of K steps (each
    # substep's solver record kept, or checkpoints every --adjoint-every substeps), then the reverse
    # pass, for a loss of the kinetic energy of the water beyond x = 1 m (gradients with respect
    # to every initial velocity and the settings)
    import numpy as np

    def loss_grad(w):
        pos_now, vel_now = w.positions(), w.velocities()
        m = w.particle_mass()
        return np.where((pos_now[:, 0] > 1.0)[:, None], m * vel_now, 0.0).astype(np.float32)

    def taped_round(w, wstream, k, every):
        """A taped forward of k steps on world w and its reverse pass, each timed with CUDA events on
        the world's stream, after one untimed round (one segment long), as the rounds of an
        optimisation loop follow one another: the tape's memory is then in the allocator's pool."""
        torch.cuda.synchronize()
        free_b, total_b = torch.cuda.mem_get_info(dev)
        before_gb = (total_b - free_b) / 1e9
        w.tape_begin(every)
        for _ in range(k if every == 0 else min(k, every)):
            w.step(sc.dt)
        dv = loss_grad(w)
        w.step_backward(np.zeros_like(dv), dv)
        w.tape_end()
        barrier()
        w.tape_begin(every)
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record(wstream)
        substeps = 0
        for _ in range(k):
            substeps += w.step(sc.dt).substeps
        e1.record(wstream)
        e1.synchronize()
        fwd_ms = e0.elapsed_time(e1)
        # device memory in use with the tape held (the whole device: this process is its only user)
        free_b, total_b = torch.cuda.mem_get_info(dev)
        taped_gb = (total_b - free_b) / 1e9
        dv = loss_grad(w)
        torch.cuda.synchronize()
        e2 = torch.cuda.Event(enable_timing=True)
        e3 = torch.cuda.Event(enable_timing=True)
        e2.record(wstream)
        dp0, dv0, grads = w.step_backward(np.zeros_like(dv), dv)
        e3.record(wstream)
        e3.synchronize()
        bwd_ms = e2.elapsed_time(e3)
        free_b, total_b = torch.cuda.mem_get_info(dev)
        w.tape_end()
        return {"substeps": substeps, "fwd_ms": fwd_ms, "bwd_ms": bwd_ms, "taped_gb": taped_gb, "before_gb": before_gb,
                "backward_gb": (total_b - free_b) / 1e9, "total_gb": total_b / 1e9,
                "dp0": dp0, "dv0": dv0, "grads": grads}

    adjoint = None
    if args.adjoint_steps > 0 and args.positions == "absolute":
        k = args.adjoint_steps
        every = max(0, args.adjoint_every)
        tr = taped_round(world, stream, k, every)
        adj_substeps, dp0, dv0, grads = tr["substeps"], tr["dp0"], tr["dv0"], tr["grads"]
        taped_gb, backward_gb, total_b = tr["taped_gb"], tr["backward_gb"], tr["total_gb"] * 1e9
        adj_all, both_ms = reduce_timing(adj_substeps, tr["fwd_ms"] + tr["bwd_ms"], world_size, dev)
        _, fwd_ms = reduce_timing(adj_substeps, tr["fwd_ms"], world_size, dev)
        bwd_ms = both_ms - fwd_ms
        finite = bool(np.isfinite(dv0).all() and np.isfinite(dp0).all())

        # the backward's kernels: another round of up to 8 steps, its reverse pass profiled
        # launch by launch (CUDA events)
        pk_steps = min(k, 8)
        world.tape_begin(every)
        p_sub = 0
        for _ in range(pk_steps):
            p_sub += world.step(sc.dt).substeps
        dv = loss_grad(world)
        world.profile(True)
        world.profile_reset()
        world.step_backward(np.zeros_like(dv), dv)
        bprof = world.profile_read()
        world.profile(False)
        world.tape_end()
        backward_kernels = {name: {"launches": c, "us_per_launch": 1e3 * ms / max(c, 1),
                                   "ms_per_substep": ms / max(p_sub, 1)}
                            for name, (c, ms, _) in sorted(bprof.items(), key=lambda kv: -kv[1][1])}
        adjoint = {"value": adj_all / (both_ms / 1e3), "unit": UNIT,
                   "gradients_finite": finite,
                   "steps": k, "substeps": adj_substeps, "checkpoint_every": every,
                   "forward_ms": fwd_ms, "backward_ms": bwd_ms,
                   "ratio_to_forward": (fwd_ms + bwd_ms) / fwd_ms,
                   "ratio_to_plain_substeps": value / (adj_all / (both_ms / 1e3)),
                   "loss": "kinetic energy of the water beyond x = 1 m after the steps",
                   "backward_kernels": {"steps": pk_steps, "substeps": p_sub, "kernels": backward_kernels},
                   "device_memory_gb": {"taped_forward": taped_gb, "after_backward": backward_gb,
                                        "device_total": total_b / 1e9},
                   "grad_viscosity": grads["viscosity"], "grad_gravity": list(grads["gravity"]),
                   "grad_uniform_inflow": [float(x) for x in dv0.astype(np.float64).sum(axis=0)]}

    # the opt-in warm start (each solve starts with one push at half the last solve's stiffness
    # impulse) on its own world from the same initial state: the reference cold-starts, so this is
    # a variant beside the headline, not the headline
    warm = None
    warm_steps = args.steps if args.warm_steps is None else args.warm_steps
    if warm_steps > 0 and sc.settings.solver.name == "DFSPH":
        import dataclasses

        wsc = dataclasses.replace(sc, settings=dataclasses.replace(sc.settings, warm_start=True))
        ww = fluid.FluidWorld(wsc.settings)
        ww.solver_graphs(graph_mode)
        wsc.build(ww)
        wstream = torch.cuda.ExternalStream(ww.stream(), device=dev)
        for _ in range(max(args.warmup, 3)):
            ww.step(sc.dt)
        barrier()
        w_ms = 0.0
        w_sub = w_its = 0
        for _ in range(warm_steps):
            flush.zero_()
            torch.cuda.synchronize()
            e0 = torch.cuda.Event(enable_timing=True)
            e1 = torch.cuda.Event(enable_timing=True)
            e0.record(wstream)
            r = ww.step(sc.dt)
            e1.record(wstream)
            e1.synchronize()
            w_ms += e0.elapsed_time(e1)
            w_sub += r.substeps
            w_its += r.iterations
        # forward + adjoint of the warm-started world, as the cold leg's, from where its timed
        # steps ended (the impulses are taped with the state)
        wtr = None
        w_adj_steps = args.adjoint_steps if args.warm_adjoint_steps is None else args.warm_adjoint_steps
        if w_adj_steps > 0 and args.positions == "absolute":
            wtr = taped_round(ww, wstream, w_adj_steps, max(0, args.adjoint_every))
        ww.close()
        w_all, w_ms = reduce_timing(w_sub, w_ms, world_size, dev)
        warm = {"value": w_all / (w_ms / 1e3), "unit": UNIT, "steps": warm_steps,
                "after_steps": max(args.warmup, 3), "substeps": w_sub,
                "solver_iterations_per_substep": w_its / max(w_sub, 1),
                "setting": "warm_start=1: one push at half the stiffness impulse of the particle's last solve"}
        if wtr is not None:
            a_all, a_ms = reduce_timing(wtr["substeps"], wtr["fwd_ms"] + wtr["bwd_ms"], world_size, dev)
            _, a_fwd = reduce_timing(wtr["substeps"], wtr["fwd_ms"], world_size, dev)
            a_value = a_all / (a_ms / 1e3)
            warm["forward_adjoint"] = {
                "value": a_value, "unit": UNIT,
                "gradients_finite": bool(np.isfinite(wtr["dv0"]).all() and np.isfinite(wtr["dp0"]).all()),
                "steps": w_adj_steps, "substeps": wtr["substeps"],
                "checkpoint_every": max(0, args.adjoint_every),
                "forward_ms": a_fwd, "backward_ms": a_ms - a_fwd, "ratio_to_forward": a_ms / a_fwd,
                "ratio_to_plain_substeps": warm["value"] / a_value,
                "device_memory_gb": {"taped_forward": wtr["taped_gb"], "after_backward": wtr["backward_gb"],
                                     "before_tape": wtr["before_gb"],
                                     "note": "the whole device, the cold world and its tape's records included"},
                "grad_gravity": list(wtr["grads"]["gravity"]),
                "grad_uniform_inflow": [float(x) for x in wtr["dv0"].astype(np.float64).sum(axis=0)]}

    base = None
    if rank == 0 and world_size == 1 and not args.no_cpu_baseline:
        state = (world.positions(), world.velocities())
        world.close()
        base = cpu_baseline(sc, args.cpu_budget, state)
    dens_err = None
    if timed_end is not None and not args.no_density_error:
        dens_err = density_error(sc, max(args.warmup, 3) + args.steps, timed_end[0], timed_end[1])

    if rank == 0:
        out = {"metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world_size, "steps": args.steps,
               "warmup": max(args.warmup, 3), "ms_per_step": total_ms / args.steps, "higher_is_better": True,
               "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
               "config": dict(workload(sc), parallelism=f"replicas x{world_size}",
                              substeps=substeps, solver_iterations_per_substep=iterations / max(substeps, 1),
                              solver_iterations_per_s=iterations / (total_ms / 1e3),
                              particle_substeps_per_s=value * sc.particles,
                              solves=GRAPH_MODES[graph_mode], substeps_as_one_graph=graphed),
               "density_error": dens_err,
               "roofline": roofline, "cpu_baseline": base, "e2e": e2e, "forward_adjoint": adjoint,
               "warm_start": warm,
               "clocks": clock_info, "gpu_launches": launches}
        print(json.dumps(out), flush=True)
    if world_size > 1:
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
