"""How far an FP32 derivative code drifts from the exact derivative of the FP32 program (CPU only).

The C5 workload's gradient check (tests/adjoint_c5.py) finds the CUDA adjoint within 1.2e-6 of the
exact derivative of the FP32 program over 8 steps of the 1M dam and 1.7e-3 (inflow x) over 16. This
driver asks whether FP32 derivative arithmetic alone drifts that far on the same scene: it runs
the float restatement (oracle/fluid_oracle.hpp, EXACT, compensated residual sum as the library's)
20 steps into the dam break, then the forward-mode tangent along the uniform inflow direction
twice from that state, with the same float values: once with derivatives in double (precision 32,
the exact derivative of the FP32 program) and once with every derivative operation rounded to
float (precision -32, oracle/dual.hpp). The relative difference of dL/d(inflow) between the two,
L the water's kinetic energy, is printed per horizon.

With --hold, the tangent (derivatives in double) runs once with nothing held and once with
each named quantity held constant (its derivative dropped: py_oracle.TANGENT_HOLD), and the
table gives what each path contributes to dL/d(inflow).  --order sorted takes the state in the
world's own order after the warm-up (the library's, bit for bit), as tests/adjoint_c5.py does.

    python tests/tangent_conditioning.py [--steps 8 16] [--axis 0] [--counts 100 100 100]
    python tests/tangent_conditioning.py --steps 16 --order sorted --hold each
"""
import argparse
import os
import sys
import time

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)

from oracle import py_oracle  # noqa: E402
from solunar_b200 import scenes  # noqa: E402


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--steps", type=int, nargs="+", default=[8, 16])
    ap.add_argument("--warm", type=int, default=20, help="steps into the dam break before the tangent")
    ap.add_argument("--axis", type=int, default=0)
    ap.add_argument("--counts", type=int, nargs=3, default=None, help="block counts (default: the 1M scene's)")
    ap.add_argument("--order", choices=("ids", "sorted"), default="ids",
                    help="the state's rows after the warm-up: by particle id, or in the world's order")
    ap.add_argument("--hold", nargs="*", default=None,
                    help="quantities to hold constant one at a time ('each': all of py_oracle.TANGENT_HOLD)")
    args = ap.parse_args()

    py_oracle.build()
    sc = scenes.dfsph_dam_1m()
    if args.counts:
        import dataclasses

        sc = dataclasses.replace(sc, block_counts=tuple(args.counts))
    w = py_oracle.OracleWorld(sc.settings, precision=32, residual_sum=1)
    sc.build(w)
    t0 = time.perf_counter()
    for _ in range(args.warm):
        w.step(sc.dt)
    order = np.argsort(w.ids()) if args.order == "ids" else np.arange(w.len())
    pos = np.asarray(w.positions(), dtype=np.float32)[order]
    vel = np.asarray(w.velocities(), dtype=np.float32)[order]
    mass = w.particle_mass()
    print(f"{len(pos)} particles, {args.warm} steps in ({time.perf_counter() - t0:.1f} s)", flush=True)

    direction = np.zeros(pos.shape)
    direction[:, args.axis] = 1.0
    tank = ((0.0, 0.0, 0.0), sc.tank)
    if args.hold is not None:
        names = list(py_oracle.TANGENT_HOLD) if args.hold in (["each"], []) else args.hold
        print("| steps | held constant | dL/d inflow | change |")
        print("|---|---|---|---|")
        for steps in args.steps:
            full = None
            for name in [None] + names:
                t0 = time.perf_counter()
                _, V, _, dV, _ = py_oracle.tangent_run(sc.settings, tank, pos, vel, np.zeros(pos.shape), direction,
                                                       steps=steps, dt=sc.dt, precision=32,
                                                       hold=() if name is None else (name,))
                value = mass * float(np.sum(V * dV))
                if name is None:
                    full = value
                change = "" if name is None else f"{value - full:+.6e}"
                print(f"| {steps} | {name or 'nothing'} | {value:.9e} | {change} |", flush=True)
                print(f"  ({time.perf_counter() - t0:.1f} s)", file=sys.stderr, flush=True)
        return
    print("| steps | dL/d inflow, derivatives in double | in float | relative difference |")
    print("|---|---|---|---|")
    for steps in args.steps:
        out = []
        for precision in (32, -32):
            t0 = time.perf_counter()
            _, V, _, dV, _ = py_oracle.tangent_run(sc.settings, tank, pos, vel, np.zeros(pos.shape), direction,
                                                   steps=steps, dt=sc.dt, precision=precision)
            out.append(mass * float(np.sum(V * dV)))
            print(f"  (precision {precision}: {time.perf_counter() - t0:.1f} s)", file=sys.stderr, flush=True)
        exact, single = out
        print(f"| {steps} | {exact:.9e} | {single:.9e} | {abs(single - exact) / abs(exact):.2e} |", flush=True)


if __name__ == "__main__":
    main()
