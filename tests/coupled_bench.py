"""Cost of coupled bodies: ticks of a pool with a floating box against the same pool without it.

Pools: the reference's coupling pool (1 x 1.2 x 1 m tank, water 0.6 m deep at 0.05 m: 4,800
particles, couple.rs:519-530) and the same tank at 0.01 m (600,000 particles), a 0.3 m box of
850 kg/m^3 dropped from 0.9 m (couple.rs:532-540), driven by the stand-in rigid integrator of
tests/rigid.py.  After 30 untimed ticks, 30 ticks are timed on the host clock (a coupled tick
holds host work: the lift reads the state, the body points are placed and sorted on the host)
and with CUDA events on the world's stream; the CPU restatement runs the small pool for the
baseline.

    python tests/coupled_bench.py [--out FILE]
"""
import argparse
import os
import sys
import time

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.join(ROOT, "tests"))

import rigid  # noqa: E402
from solunar_b200 import fluid  # noqa: E402
from solunar_b200.abi import Arithmetic, FluidSettings, Shape  # noqa: E402

TICK = np.float32(1.0 / 60.0)


def pool(make, spacing):
    w = make(FluidSettings(spacing=spacing, arithmetic=Arithmetic.EXACT, max_particles=1 << 22))
    w.add_box_container((0.0, 0.0, 0.0), (1.0, 1.2, 1.0))
    w.fill_box((0.0, 0.0, 0.0), (1.0, 0.6, 1.0))
    return w


def measure(make, spacing, coupled, ticks=30, warm=30, stream=None):
    import torch

    w = pool(make, spacing)
    bodies = []
    if coupled:
        body = rigid.Body(1, Shape.CUBOID, (0.15, 0.15, 0.15), 850.0, (0.5, 0.9, 0.5))
        w.couple(body.handle, Shape.CUBOID, body.dims)
        bodies = [body]
    rigid.run(w, bodies, warm)
    sub = 0
    ev = None
    if stream is not None:
        s = torch.cuda.ExternalStream(w.stream())
        ev = [torch.cuda.Event(enable_timing=True) for _ in range(2)]
        torch.cuda.synchronize()
        ev[0].record(s)
    t = time.perf_counter()
    for r in rigid.run(w, bodies, ticks):
        sub += r.substeps
    if ev is not None:
        ev[1].record(s)
        ev[1].synchronize()
    host_ms = (time.perf_counter() - t) * 1e3 / ticks
    dev_ms = ev[0].elapsed_time(ev[1]) / ticks if ev is not None else None
    points = w.coupled()[0][1] if coupled else 0
    return {"particles": w.len(), "points": points, "host_ms_per_tick": host_ms, "device_ms_per_tick": dev_ms,
            "substeps_per_tick": sub / ticks, "height": float(bodies[0].x[1]) if bodies else None}


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--out", default=None)
    args = ap.parse_args()
    lines = ["| pool | body | particles | body points | substeps/tick | host ms/tick | device ms/tick | box height m |",
             "|---|---|---|---|---|---|---|---|"]
    gpu = lambda s: fluid.FluidWorld(s)
    for spacing in (0.05, 0.01):
        for coupled in (False, True):
            m = measure(gpu, spacing, coupled, stream=True)
            lines.append(f"| {spacing} m, CUDA | {'box' if coupled else 'none'} | {m['particles']} | {m['points']} | "
                         f"{m['substeps_per_tick']:.1f} | {m['host_ms_per_tick']:.2f} | {m['device_ms_per_tick']:.2f} | "
                         f"{m['height'] if m['height'] is None else round(m['height'], 3)} |")
            print(lines[-1], flush=True)
    from oracle import py_oracle

    py_oracle.build()
    cores = os.cpu_count() or 1
    for coupled in (False, True):
        m = measure(lambda s: py_oracle.OracleWorld(s, threads=cores), 0.05, coupled, ticks=10, warm=30)
        lines.append(f"| 0.05 m, CPU restatement ({cores} threads) | {'box' if coupled else 'none'} | {m['particles']} | "
                     f"{m['points']} | {m['substeps_per_tick']:.1f} | {m['host_ms_per_tick']:.2f} | — | "
                     f"{m['height'] if m['height'] is None else round(m['height'], 3)} |")
        print(lines[-1], flush=True)
    text = "\n".join(lines) + "\n"
    print(text)
    if args.out:
        with open(args.out, "w") as f:
            f.write(text)


if __name__ == "__main__":
    main()
