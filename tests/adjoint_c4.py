"""The WCSPH adjoint on its benchmark configuration, against central differences.

40^3 particles at 0.02 m in a 1 m tank, support 4, c = 20 m/s, viscosity 0.01, initial velocities
N(0, 0.1 m/s), 200 steps of 2e-4 s, tape checkpoint every 20 steps.  Loss: |centroid - (start
centroid + 0.3 m along x)|^2.  The adjoint's derivative along 16 seeded directions of the initial
velocities, and its viscosity derivative, are compared with central differences of the same FP32
forward at several step sizes; the forward and the backward are timed with CUDA events.  With
--tangent K the first K directions and the viscosity are also compared with the exact derivative
of the FP32 program itself: the restatement in forward-mode derivative numbers whose values are the
float restatement's, and so the library's, bit for bit (oracle/dual.hpp; about half a minute a
direction on the host cores).  The particles start on the pressure clamp's kink, where the
differences cannot converge; the tangent has no step size.

    python tests/adjoint_c4.py [--directions 16] [--tangent K] [--repeat R] [--out FILE]
"""
import argparse
import os
import sys
import time

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)

from solunar_b200 import fluid, scenes  # noqa: E402


def run(settings, sc, vel0):
    w = fluid.FluidWorld(settings)
    w.add_box_container((0.0, 0.0, 0.0), sc.tank)
    pos, _ = sc.initial_state()
    w.add_particles(pos, vel0)
    return w, pos


def loss_of(w, target):
    c = np.mean(np.asarray(w.positions(), dtype=np.float64), axis=0)
    return float(np.sum((c - target) ** 2)), c


def forward_loss(settings, sc, vel0, target):
    w, _ = run(settings, sc, vel0)
    for _ in range(sc.steps):
        w.step(sc.dt)
    loss = loss_of(w, target)[0]
    w.close()
    return loss


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--directions", type=int, default=16)
    ap.add_argument("--every", type=int, default=20)
    ap.add_argument("--tangent", type=int, default=0, help="directions also checked against the FP32 tangent")
    ap.add_argument("--out", default=None)
    ap.add_argument("--repeat", type=int, default=1,
                    help="tapes timed on the same world, each from the initial state (the later ones reuse the "
                         "tape's device buffers)")
    ap.add_argument("--profile", action="store_true",
                    help="one more tape whose backward is timed kernel by kernel (CUDA events)")
    args = ap.parse_args()
    import torch

    sc = scenes.wcsph_adjoint_64k()
    pos0, vel0 = sc.initial_state()
    target = np.mean(pos0.astype(np.float64), axis=0) + np.array([0.3, 0.0, 0.0])

    w, _ = run(sc.settings, sc, vel0)
    stream = torch.cuda.ExternalStream(w.stream())
    lines = []
    for r in range(max(1, args.repeat)):
        if r:  # the initial state again, in the world's current order
            ids = w.ids()
            w.write_state(pos0[ids], vel0[ids])
        e = [torch.cuda.Event(enable_timing=True) for _ in range(4)]
        w.tape_begin(args.every)
        e[0].record(stream)
        for _ in range(sc.steps):
            w.step(sc.dt)
        e[1].record(stream)
        e[1].synchronize()
        L, c = loss_of(w, target)
        n = w.len()
        dpos = np.tile(2.0 * (c - target) / n, (n, 1)).astype(np.float32)
        e[2].record(stream)
        dp0, dv0, params = w.step_backward(dpos, np.zeros_like(dpos))
        e[3].record(stream)
        e[3].synchronize()
        fwd_ms, bwd_ms = e[0].elapsed_time(e[1]), e[2].elapsed_time(e[3])
        w.tape_end()
        lines.append(f"tape {r}: loss {L:.6e}; forward {fwd_ms:.1f} ms, backward {bwd_ms:.1f} ms "
                     f"(forward+adjoint {1 + bwd_ms / fwd_ms:.2f}x the taped forward), {sc.steps} steps, "
                     f"checkpoint every {args.every}")
        print(lines[-1], flush=True)
    if args.profile:
        ids = w.ids()
        w.write_state(pos0[ids], vel0[ids])
        w.tape_begin(args.every)
        for _ in range(sc.steps):
            w.step(sc.dt)
        L, c = loss_of(w, target)
        dpos = np.tile(2.0 * (c - target) / w.len(), (w.len(), 1)).astype(np.float32)
        w.profile(True)
        w.profile_reset()
        w.step_backward(dpos, np.zeros_like(dpos))
        prof = w.profile_read()
        w.profile(False)
        w.tape_end()
        total = sum(v[1] for v in prof.values())
        lines.append(f"backward kernel by kernel (CUDA events, launch by launch): {total:.1f} ms in all")
        for name, (k, ms, _) in sorted(prof.items(), key=lambda kv: -kv[1][1]):
            lines.append(f"  {name}: {k} launches, {ms:.1f} ms, {1e3 * ms / max(k, 1):.1f} us each")
        print("\n".join(lines[-len(prof) - 1:]), flush=True)
    w.close()
    lines.append("")
    tank = ((0.0, 0.0, 0.0), sc.tank)

    def tangent(dvel, dparams):
        """dL along the direction from the FP32 program's exact derivative."""
        from oracle import py_oracle

        P, _, dP, _, _ = py_oracle.tangent_run(sc.settings, tank, pos0, vel0, np.zeros(pos0.shape), dvel,
                                               dparams=dparams, steps=sc.steps, dt=sc.dt, precision=32)
        c = P.mean(axis=0)
        return float(np.sum((2.0 * (c - target) / len(P)) * dP))

    head = "| direction | adjoint | FD eps 1e-3 | rel | FD eps 3e-3 | rel | FD eps 1e-2 | rel |"
    rule = "|---|---|---|---|---|---|---|---|"
    if args.tangent:
        head += " FP32 tangent | rel |"
        rule += "---|---|"
    lines += [head, rule]
    exact = []
    rng = np.random.default_rng(11)
    worst = []
    for k in range(args.directions):
        d = rng.normal(size=vel0.shape)
        d /= np.sqrt(np.mean(d * d))
        row = [f"{k}"]
        ana = None
        rels = []
        for eps in (1e-3, 3e-3, 1e-2):
            vp = (vel0 + eps * d).astype(np.float32)
            vm = (vel0 - eps * d).astype(np.float32)
            num = (forward_loss(sc.settings, sc, vp, target) - forward_loss(sc.settings, sc, vm, target)) / (2 * eps)
            if ana is None:
                ana = float(np.sum(dv0.astype(np.float64) * (vp.astype(np.float64) - vm.astype(np.float64)) / (2 * eps)))
                row.append(f"{ana:.6e}")
            rel = abs(ana - num) / max(abs(num), 1e-300)
            rels.append(rel)
            row += [f"{num:.6e}", f"{rel:.2e}"]
        worst.append(min(rels))
        if k < args.tangent:
            t = tangent(d, np.zeros(5))
            a = float(np.sum(dv0.astype(np.float64) * d))
            exact.append(abs(a - t) / max(abs(t), 1e-300))
            row += [f"{t:.6e}", f"{exact[-1]:.2e}"]
        lines.append("| " + " | ".join(row) + " |")
        print(lines[-1], flush=True)
    lines.append("")
    if worst:
        lines.append(f"best-of-steps relative error over the {args.directions} directions: median "
                     f"{np.median(worst):.2e}, max {np.max(worst):.2e}")
    if exact:
        lines.append(f"against the FP32 tangent over {len(exact)} directions: median {np.median(exact):.2e}, "
                     f"max {np.max(exact):.2e}")
    s = sc.settings
    vrow = []
    for eps in (1e-4, 1e-3):
        a = dict(vars(s))
        up = fluid.FluidSettings(**{**a, "viscosity": s.viscosity + eps})
        dn = fluid.FluidSettings(**{**a, "viscosity": s.viscosity - eps})
        num = (forward_loss(up, sc, vel0, target) - forward_loss(dn, sc, vel0, target)) / (2 * eps)
        vrow.append(f"eps {eps:g}: FD {num:.6e}, rel {abs(params['viscosity'] - num) / max(abs(num), 1e-300):.2e}")
    if args.tangent:
        t = tangent(np.zeros(pos0.shape), np.array([1.0, 0.0, 0.0, 0.0, 0.0]))
        vrow.append(f"FP32 tangent {t:.6e}, rel {abs(params['viscosity'] - t) / max(abs(t), 1e-300):.2e}")
    lines.append(f"viscosity: adjoint {params['viscosity']:.6e}; " + "; ".join(vrow))
    text = "\n".join(lines) + "\n"
    print(text)
    if args.out:
        with open(args.out, "w") as f:
            f.write(text)


if __name__ == "__main__":
    main()
