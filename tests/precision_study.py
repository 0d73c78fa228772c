"""Precision study of the position representations, against the FP64 restatement.

One scene runs through
  * the FP64 restatement of the algorithm (the oracle, on the CPU, compensated residual sums);
  * the GPU, EXACT arithmetic, absolute f32 positions (the reference's own arithmetic);
  * the GPU, FAST arithmetic, absolute f32 positions;
  * the GPU, FAST arithmetic, cell-relative positions (an f32 offset from each particle's cell).
Against the FP64 run it reports the density error (max and mean of |rho - rho64| / rho0 at the
end), the position error, the drift of the centroid, and the solver iterations per substep.

Two parts, because the FP64 run is CPU work and the others need a B200:

    python tests/precision_study.py oracle --scene dfsph_precision_1m --steps 300 --out DIR
    python tests/precision_study.py gpu --scene dfsph_precision_1m --steps 300 --out DIR \\
        --reference DIR/fp64_dfsph_precision_1m.npz

The gpu part writes DIR/precision_<scene>.md and .json.
"""
import argparse
import json
import os
import sys
import time

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)

from solunar_b200 import scenes  # noqa: E402
from solunar_b200.abi import Arithmetic, Positions  # noqa: E402


def make_scene(name, counts=None):
    sc = getattr(scenes, name)(counts=tuple(counts)) if counts else getattr(scenes, name)()
    return sc


def run(world, sc, steps, label):
    """Steps `world` through the scene; per step the iterations and the centroid (float64)."""
    sc.build(world)
    iters, centroid, substeps = [], [], []
    t0 = time.time()
    for k in range(steps):
        r = world.step(sc.dt)
        iters.append(int(r.iterations))
        substeps.append(int(r.substeps))
        centroid.append(world.positions().astype(np.float64).mean(axis=0).tolist())
        if (k + 1) % 50 == 0:
            print(f"{label}: step {k + 1}/{steps}, {time.time() - t0:.0f} s", flush=True)
    order = np.argsort(world.ids())
    return {
        "positions": world.positions()[order].astype(np.float64),
        "densities": world.densities()[order].astype(np.float64),
        "iterations": np.asarray(iters),
        "substeps": np.asarray(substeps),
        "centroid": np.asarray(centroid),
    }


def part_oracle(args):
    from oracle import py_oracle

    sc = make_scene(args.scene, args.counts)
    w = py_oracle.OracleWorld(sc.settings, precision=64, residual_sum=1, threads=os.cpu_count() or 1)
    res = run(w, sc, args.steps, "fp64")
    os.makedirs(args.out, exist_ok=True)
    path = os.path.join(args.out, f"fp64_{sc.name}.npz")
    np.savez_compressed(path, **res)
    print(path)


def part_gpu(args):
    from solunar_b200 import fluid

    ref = dict(np.load(args.reference))
    sc0 = make_scene(args.scene, args.counts)
    rest = float(sc0.settings.rest_density)
    c0 = None
    rows = {}
    for label, arith, positions in (("f32 absolute, EXACT", Arithmetic.EXACT, Positions.ABSOLUTE),
                                    ("f32 absolute, FAST", Arithmetic.FAST, Positions.ABSOLUTE),
                                    ("f32 cell-relative, FAST", Arithmetic.FAST, Positions.CELL_RELATIVE)):
        sc = make_scene(args.scene, args.counts)
        sc.settings.arithmetic = arith
        sc.settings.positions = positions
        res = run(fluid.FluidWorld(sc.settings), sc, args.steps, label)
        if c0 is None:
            c0 = np.asarray(sc.initial_state()[0], dtype=np.float64).mean(axis=0)
        derr = np.abs(res["densities"] - ref["densities"]) / rest
        perr = np.linalg.norm(res["positions"] - ref["positions"], axis=1)
        drift = np.linalg.norm(res["centroid"] - ref["centroid"], axis=1)
        rows[label] = {
            "density_err_max": float(derr.max()),
            "density_err_mean": float(derr.mean()),
            "position_err_max_m": float(perr.max()),
            "position_err_mean_m": float(perr.mean()),
            "centroid_drift_end_m": float(drift[-1]),
            "centroid_drift_max_m": float(drift.max()),
            "iterations_mean": float(res["iterations"].mean()),
            "iterations_total": int(res["iterations"].sum()),
            "iteration_steps_differing_from_fp64": int(np.count_nonzero(res["iterations"] != ref["iterations"])),
            "substeps": int(res["substeps"].sum()),
        }
    fp64 = {"iterations_mean": float(ref["iterations"].mean()), "iterations_total": int(ref["iterations"].sum()),
            "substeps": int(ref["substeps"].sum()),
            "centroid_moved_m": float(np.linalg.norm(ref["centroid"][-1] - c0))}
    out = {"scene": sc0.name, "particles": sc0.particles, "steps": args.steps, "dt": sc0.dt, "origin": sc0.origin,
           "fp64": fp64, "runs": rows}
    os.makedirs(args.out, exist_ok=True)
    with open(os.path.join(args.out, f"precision_{sc0.name}.json"), "w") as f:
        json.dump(out, f, indent=1)
    lines = [f"# precision: {sc0.name}, {sc0.particles} particles, {args.steps} steps of {sc0.dt} s, "
             f"origin {sc0.origin}",
             "",
             f"FP64 restatement: {fp64['substeps']} substeps, {fp64['iterations_mean']:.2f} solver iterations "
             f"per step, centroid moved {fp64['centroid_moved_m']:.4g} m.",
             "",
             "| run | max abs(rho - rho64)/rho0 | mean | max abs(x - x64) m | mean | centroid drift m (end) "
             "| iterations per step | steps whose iterations differ |",
             "|---|---|---|---|---|---|---|---|"]
    for label, r in rows.items():
        lines.append(f"| {label} | {r['density_err_max']:.3e} | {r['density_err_mean']:.3e} | "
                     f"{r['position_err_max_m']:.3e} | {r['position_err_mean_m']:.3e} | "
                     f"{r['centroid_drift_end_m']:.3e} | {r['iterations_mean']:.2f} | "
                     f"{r['iteration_steps_differing_from_fp64']} |")
    with open(os.path.join(args.out, f"precision_{sc0.name}.md"), "w") as f:
        f.write("\n".join(lines) + "\n")
    print("\n".join(lines))


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("part", choices=["oracle", "gpu"])
    ap.add_argument("--scene", default="dfsph_precision_1m")
    ap.add_argument("--counts", type=int, nargs=3, default=None, help="block particle counts (scenes that take them)")
    ap.add_argument("--steps", type=int, default=300)
    ap.add_argument("--out", required=True)
    ap.add_argument("--reference", help="the oracle part's .npz (gpu part)")
    args = ap.parse_args()
    part_oracle(args) if args.part == "oracle" else part_gpu(args)


if __name__ == "__main__":
    main()
