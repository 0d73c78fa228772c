"""The DFSPH adjoint on the one-million-particle dam, against central differences.

The bench's forward+adjoint workload (100^3 particles at 0.01 m in the 2 x 1 x 1 m tank, 32 steps of
1e-3 s, every substep's solver record kept), from a flowing state: 20 steps into the dam break.
Loss: the water's kinetic energy after the steps, sum of m |v|^2 / 2 (smooth, so differences do
not jump where particles cross a boundary).  The adjoint's derivatives along a uniform change of
the initial velocities (the inflow vector) and of gravity are compared with central differences of
the same FP32 forward at two step sizes, and (--tangent 32) with the exact derivative of the FP32
program itself along the same directions: the restatement in forward-mode derivative numbers
whose values are the float restatement's, hence the library's, bit for bit, with derivatives in
double (oracle/dual.hpp; about a minute a direction on the host cores at this size).  It takes
every branch the library's run takes.  `--tangent 64` takes the FP64 method's derivative instead,
which over this flowing, strongly non-linear horizon is a different number: the FP32 and FP64
trajectories part.  The tangent is also held to the library's solver iteration counts (each
substep's divergence and density solves).  Differences at eps 1e-2 cross the loss's kinks (solver
stops, the < 20 neighbour rule, clamps), which is why they scatter.  Every evaluation starts from the same state handed to a
new world, so the differences and the adjoint see the same particle order.

    python tests/adjoint_c5.py [--steps 32] [--tangent 32|64] [--warm-start] [--out FILE]
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
    ap.add_argument("--tangent", type=int, choices=(32, 64), default=None,
                    help="add the column of the exact derivative of the FP32 program (32) or the FP64 method (64)")
    ap.add_argument("--warm-start", action="store_true",
                    help="warm-started solves (each run starts with no impulses: a world made from a state)")
    ap.add_argument("--out", default=None)
    args = ap.parse_args()

    sc = scenes.dfsph_dam_1m()
    if args.warm_start:
        sc = dataclasses.replace(sc, settings=dataclasses.replace(sc.settings, warm_start=True))
    w = fluid.FluidWorld(sc.settings)
    sc.build(w)
    for _ in range(args.warm):
        w.step(sc.dt)
    pos, vel = np.array(w.positions(), dtype=np.float32), np.array(w.velocities(), dtype=np.float32)
    w.close()

    # the adjoint over the steps
    w = world_from(sc, sc.settings, pos, vel)
    w.tape_begin(0)
    counts = []
    for _ in range(args.steps):
        r = w.step(sc.dt)
        if r.substeps != 1:
            raise SystemExit("a step took more than one substep: the solver counts would be incomplete")
        counts += list(w.last_iterations())
    L = loss_of(w)
    dv = (w.particle_mass() * np.asarray(w.velocities(), dtype=np.float64)).astype(np.float32)
    _, dv0, params = w.step_backward(np.zeros_like(dv), dv)
    w.tape_end()
    w_mass = w.particle_mass()
    w.close()
    inflow = dv0.astype(np.float64).sum(axis=0)
    gravity = np.array(params["gravity"])

    def tangent(dvel, dparams):
        """dL along the direction, from the FP64 restatement's exact derivative."""
        from oracle import py_oracle

        tank = ((0.0, 0.0, 0.0), sc.tank)
        _, V, _, dV, _ = py_oracle.tangent_run(sc.settings, tank, pos, vel, np.zeros(pos.shape), dvel,
                                               dparams=dparams, steps=args.steps, dt=sc.dt, forced_iterations=counts,
                                               precision=args.tangent)
        return w_mass * float(np.sum(V * dV))

    head = "| derivative | adjoint | FD eps 1e-3 | rel | FD eps 1e-2 | rel |"
    rule = "|---|---|---|---|---|---|"
    if args.tangent:
        head += f" FP{args.tangent} tangent | rel |"
        rule += "---|---|"
    # the inflow derivative sums a million per-particle terms: how much of their size cancels (an
    # FP32 error in each term grows by this factor in the sum)
    spread = np.abs(dv0.astype(np.float64)).sum(axis=0) / np.maximum(np.abs(inflow), 1e-300)
    lines = [f"1M DFSPH dam{' (warm-started solves)' if args.warm_start else ''}, {args.steps} steps of "
             f"{sc.dt} s from {args.warm} steps in; loss (kinetic energy) "
             f"{L:.6e} J", f"sum |dL/dv0| / |sum dL/dv0| per axis: {spread[0]:.3g}, {spread[1]:.3g}, {spread[2]:.3g}",
             "", head, rule]
    worst = []
    exact = []

    def tangent_cells(adj, dvel, dparams):
        t = tangent(dvel, dparams)
        rel = abs(adj - t) / max(abs(t), 1e-300)
        exact.append(rel)
        return [f"{t:.6e}", f"{rel:.2e}"]

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
        if args.tangent:
            e = np.zeros(3)
            e[k] = 1.0
            row += tangent_cells(inflow[k], np.tile(e, (len(pos), 1)), np.zeros(5))
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
        if args.tangent:
            q = np.zeros(5)
            q[2 + k] = 1.0
            row += tangent_cells(gravity[k], np.zeros(pos.shape), q)
        lines.append("| " + " | ".join(row) + " |")
        print(lines[-1], flush=True)
    lines += ["", f"best-of-steps relative error: median {np.median(worst):.2e}, max {np.max(worst):.2e}"]
    if exact:
        lines += [f"against the FP{args.tangent} tangent: median {np.median(exact):.2e}, max {np.max(exact):.2e}"]
    text = "\n".join(lines) + "\n"
    print(text)
    if args.out:
        with open(args.out, "w") as f:
            f.write(text)


if __name__ == "__main__":
    main()
