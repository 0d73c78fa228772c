"""Prints the WCSPH adjoint's directional derivatives next to central differences (FP32 GPU forward
at three steps, FP64 CPU restatement at two), on the scene of test_gpu_adjoint.py.

    python tests/adjoint_report.py
"""
import os, sys, numpy as np
ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT); sys.path.insert(0, os.path.join(ROOT, "tests"))
from oracle import py_oracle
from solunar_b200 import fluid
import test_gpu_adjoint as T
fluid.load_library()
sc = T.scene()
w, pos, vel = T.run(fluid.FluidWorld, sc)

target = np.mean(pos.astype(np.float64), axis=0) + np.array([0.3, 0.0, 0.0])
w.tape_begin(10)
for _ in range(T.STEPS): w.step(T.DT)
L, c = T.loss(w, target); n = w.len()
dpos = np.tile(2.0 * (c - target) / n, (n, 1)).astype(np.float32)
dp0, dv0, params = w.step_backward(dpos, np.zeros_like(dpos))
print("L", L, "params", params)
make64 = lambda s: py_oracle.OracleWorld(s, precision=64)
rng = np.random.default_rng(7)
for k in range(4):
    d = rng.normal(size=vel.shape); d /= np.sqrt(np.mean(d * d))
    ana = float(np.sum(dv0.astype(np.float64) * d))
    line = f"dir {k}: adjoint {ana:.6e}"
    for eps in (1e-3, 3e-3, 1e-2):
        lp = T.fd(fluid.FluidWorld, sc, target, (vel + eps * d).astype(np.float32))
        lm = T.fd(fluid.FluidWorld, sc, target, (vel - eps * d).astype(np.float32))
        num = (lp - lm) / (2 * eps)
        line += f" | f32 eps {eps:g}: {num:.6e} rel {abs(ana-num)/abs(num):.2e}"
    for eps in (1e-4, 3e-5):
        vp = (vel + eps * d).astype(np.float32); vm = (vel - eps * d).astype(np.float32)
        num = (T.fd(make64, sc, target, vp) - T.fd(make64, sc, target, vm)) / (2 * eps)
        ana2 = float(np.sum(dv0.astype(np.float64) * (vp.astype(np.float64) - vm.astype(np.float64)) / (2 * eps)))
        line += f" | f64 eps {eps:g}: {num:.6e} rel {abs(ana2-num)/abs(num):.2e}"
    print(line, flush=True)
