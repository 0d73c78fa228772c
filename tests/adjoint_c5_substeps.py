"""The DFSPH adjoint of single substeps of the 1M dam against the FP32 program's exact derivative.

Over 8 steps of the C5 window (20 steps into the dam break) the adjoint agrees with the exact
derivative of the FP32 program to 1e-6; over 16 steps inflow x parts by 1e-3 (the table of
profiles/dfsph_adjoint_c5_1m_fd_check.md), though an FP32 derivative code drifts by only 5e-9
there (tests/tangent_conditioning.py).  This driver finds the substep where the two part: from
each state of the window, a new world runs one substep under a tape and takes step_backward for
a cotangent g of the final state, and the restatement in forward-mode derivative numbers
(oracle/dual.hpp, values of the float restatement bit for bit, held to the library's solver
iteration counts) runs the same substep along a direction d of the initial state.  Per substep
it prints <g, J d> (tangent), <J^T g, d> (adjoint) and their relative difference, for d the
uniform inflow x with g the kinetic energy's gradient (the C5 loss), and for random g and d.
It also checks that the tangent's values are the library's, bit for bit.

    python tests/adjoint_c5_substeps.py [--from 20] [--count 16]
"""
import argparse
import os
import sys
import time

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)

from oracle import py_oracle  # noqa: E402
from solunar_b200 import fluid, scenes  # noqa: E402


def one_substep(sc, pos, vel, cases):
    """The adjoint of one substep from (pos, vel) for each (g_pos, g_vel) cotangent (id order), a
    new world and tape for each, with the substep's solver counts and its final state in id
    order."""
    counts, final, grads = None, None, []
    for gp, gv in cases:
        w = fluid.FluidWorld(sc.settings)
        w.add_box_container((0.0, 0.0, 0.0), sc.tank)
        w.add_particles(pos, vel)
        w.tape_begin(0)
        r = w.step(sc.dt)
        if r.substeps != 1:
            raise SystemExit("a step took more than one substep")
        counts = list(w.last_iterations())
        ids = np.asarray(w.ids())
        order = np.argsort(ids)
        final = (np.asarray(w.positions(), dtype=np.float32)[order],
                 np.asarray(w.velocities(), dtype=np.float32)[order])
        # cotangents in the world's current order (row k holds id ids[k])
        dp0, dv0, _ = w.step_backward(gp[ids].astype(np.float32), gv[ids].astype(np.float32))
        grads.append((dp0.astype(np.float64), dv0.astype(np.float64)))
        w.tape_end()
        w.close()
    return counts, final, grads


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--from", dest="start", type=int, default=20, help="steps into the dam break of the first substep")
    ap.add_argument("--count", type=int, default=16)
    args = ap.parse_args()
    py_oracle.build()

    sc = scenes.dfsph_dam_1m()
    main_world = fluid.FluidWorld(sc.settings)
    sc.build(main_world)
    for _ in range(args.start):
        main_world.step(sc.dt)
    tank = ((0.0, 0.0, 0.0), sc.tank)
    rng = np.random.default_rng(2024)
    print("| step | direction | tangent <g, J d> | adjoint <J^T g, d> | rel | values bit-identical |")
    print("|---|---|---|---|---|---|")
    for k in range(args.count):
        pos = np.asarray(main_world.positions(), dtype=np.float32)
        vel = np.asarray(main_world.velocities(), dtype=np.float32)
        n = len(pos)
        # the C5 loss's gradient on the final velocities needs the final state: take it from a
        # forward of the same substep first (the adjoint's world runs it again, bit for bit)
        probe = fluid.FluidWorld(sc.settings)
        probe.add_box_container((0.0, 0.0, 0.0), sc.tank)
        probe.add_particles(pos, vel)
        probe.step(sc.dt)
        order = np.argsort(np.asarray(probe.ids()))
        v_final = np.asarray(probe.velocities(), dtype=np.float64)[order]
        mass = probe.particle_mass()
        probe.close()
        inflow = np.zeros((n, 3))
        inflow[:, 0] = 1.0
        rand_d = (rng.normal(size=(n, 3)) * 1e-3, rng.normal(size=(n, 3)))
        rand_g = (rng.normal(size=(n, 3)), rng.normal(size=(n, 3)))
        cases = [((np.zeros((n, 3)), mass * v_final), (np.zeros((n, 3)), inflow), "inflow x, C5 loss"),
                 (rand_g, rand_d, "random g, d")]
        t0 = time.perf_counter()
        counts, final, grads = one_substep(sc, pos, vel, [c[0] for c in cases])
        t_adj = time.perf_counter() - t0
        for (g, d, name), (gp0, gv0) in zip(cases, grads):
            t0 = time.perf_counter()
            P, V, dP, dV, _ = py_oracle.tangent_run(sc.settings, tank, pos, vel, d[0], d[1], steps=1, dt=sc.dt,
                                                    forced_iterations=counts, precision=32)
            same = bool(np.array_equal(P.astype(np.float32), final[0]) and
                        np.array_equal(V.astype(np.float32), final[1]))
            tangent = float(np.sum(g[0] * dP) + np.sum(g[1] * dV))
            adjoint = float(np.sum(gp0 * d[0]) + np.sum(gv0 * d[1]))
            rel = abs(adjoint - tangent) / max(abs(tangent), abs(adjoint), 1e-300)
            print(f"| {args.start + k} | {name} | {tangent:.9e} | {adjoint:.9e} | {rel:.2e} | {same} |", flush=True)
            print(f"  (adjoint {t_adj:.1f} s, tangent {time.perf_counter() - t0:.1f} s, counts {counts})",
                  file=sys.stderr, flush=True)
        main_world.step(sc.dt)
    main_world.close()


if __name__ == "__main__":
    main()
