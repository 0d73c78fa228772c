"""The DFSPH adjoint on the one-million-particle dam, against central differences.

The bench's forward+adjoint workload (100^3 particles at 0.01 m in the 2 x 1 x 1 m tank, 32 steps of
1e-3 s, every substep's solver record kept), from a flowing state: 20 steps into the dam break.
Loss: the water's kinetic energy after the steps, sum of m |v|^2 / 2 (smooth, so differences do
not jump where particles cross a boundary).  The adjoint's derivatives along a uniform change of
the initial velocities (the inflow vector) and of gravity are compared with central differences of
the same FP32 forward at two step sizes.  Every evaluation starts from the same state handed to a
new world, so the differences and the adjoint see the same particle order.

    python tests/adjoint_c5.py [--steps 32] [--out FILE]
"""
import argparse
import dataclasses
import os
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)

from solunar_b200 import fluid, scenes  # noqa: E402


def world_from(sc, settings, pos, vel):
    w = fluid.FluidWorld(settings)
    w.add_box_container((0.0, 0.0, 0.0), sc.tank)
    w.add_particles(pos, vel)
    return w


def loss_of(w):
    v = np.asarray(w.velocities(), dtype=np.float64)
    return 0.5 * w.particle_mass() * float(np.sum(v * v))


def forward(sc, settings, pos, vel, steps):
    w = world_from(sc, settings, pos, vel)
    for _ in range(steps):
        w.step(sc.dt)
    loss = loss_of(w)
    w.close()
    return loss


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--steps", type=int, default=32)
    ap.add_argument("--warm", type=int, default=20)
    ap.add_argument("--out", default=None)
    args = ap.parse_args()

    sc = scenes.dfsph_dam_1m()
    w = fluid.FluidWorld(sc.settings)
    sc.build(w)
    for _ in range(args.warm):
        w.step(sc.dt)
    pos, vel = np.array(w.positions(), dtype=np.float32), np.array(w.velocities(), dtype=np.float32)
    w.close()

    # the adjoint over the steps
    w = world_from(sc, sc.settings, pos, vel)
    w.tape_begin(0)
    for _ in range(args.steps):
        w.step(sc.dt)
    L = loss_of(w)
    dv = (w.particle_mass() * np.asarray(w.velocities(), dtype=np.float64)).astype(np.float32)
    _, dv0, params = w.step_backward(np.zeros_like(dv), dv)
    w.tape_end()
    w.close()
    inflow = dv0.astype(np.float64).sum(axis=0)
    gravity = np.array(params["gravity"])

    lines = [f"1M DFSPH dam, {args.steps} steps of {sc.dt} s from {args.warm} steps in; loss (kinetic energy) "
             f"{L:.6e} J", "", "| derivative | adjoint | FD eps 1e-3 | rel | FD eps 1e-2 | rel |", "|---|---|---|---|---|---|"]
    worst = []
    for k, axis in enumerate("xyz"):
        row = [f"d/d inflow {axis}", f"{inflow[k]:.6e}"]
        rels = []
        for eps in (1e-3, 1e-2):
            e = np.zeros(3, dtype=np.float32)
            e[k] = eps
            num = (forward(sc, sc.settings, pos, vel + e, args.steps) -
                   forward(sc, sc.settings, pos, vel - e, args.steps)) / (2 * eps)
            rel = abs(inflow[k] - num) / max(abs(num), 1e-300)
            rels.append(rel)
            row += [f"{num:.6e}", f"{rel:.2e}"]
        worst.append(min(rels))
        lines.append("| " + " | ".join(row) + " |")
        print(lines[-1], flush=True)
    for k, axis in enumerate("xyz"):
        row = [f"d/d gravity {axis}", f"{gravity[k]:.6e}"]
        rels = []
        for eps in (1e-3, 1e-2):
            def with_g(delta):
                g = list(sc.settings.gravity)
                g[k] = g[k] + delta
                return dataclasses.replace(sc.settings, gravity=tuple(g))
            num = (forward(sc, with_g(eps), pos, vel, args.steps) -
                   forward(sc, with_g(-eps), pos, vel, args.steps)) / (2 * eps)
            rel = abs(gravity[k] - num) / max(abs(num), 1e-300)
            rels.append(rel)
            row += [f"{num:.6e}", f"{rel:.2e}"]
        worst.append(min(rels))
        lines.append("| " + " | ".join(row) + " |")
        print(lines[-1], flush=True)
    lines += ["", f"best-of-steps relative error: median {np.median(worst):.2e}, max {np.max(worst):.2e}"]
    text = "\n".join(lines) + "\n"
    print(text)
    if args.out:
        with open(args.out, "w") as f:
            f.write(text)


if __name__ == "__main__":
    main()
