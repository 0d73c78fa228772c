"""The adjoint through torch.autograd: the test harness's `FluidRun` (tests/fluid_autograd.py)
wraps a taped run and `step_backward` as a torch.autograd.Function.

Its gradients must be `step_backward`'s, called directly on the same run, bit for bit (the
parameter gradients, FP64 sums taken with atomics, to 1e-9), and a loss written in torch must
get central differences' slope: the WCSPH block of the adjoint tests (512 particles, support 4,
30 steps of 2e-4 s), loss the squared distance of the centroid to a point 0.3 m downstream,
differentiated along a seeded direction of the initial velocities (relative error 2e-2, the
better of eps 3e-3 and 1e-2, as for `step_backward` itself).
"""
import numpy as np
import pytest
import torch

from fluid_autograd import FluidRun, to_id_order
from solunar_b200 import scenes
from solunar_b200.abi import FluidSettings, FluidSolver

pytestmark = pytest.mark.gpu

STEPS = 30
DT = 2e-4
TANK = (0.4, 0.4, 0.4)


def setup(gpu_lib, solver=FluidSolver.WCSPH):
    if solver == FluidSolver.WCSPH:
        s = FluidSettings(solver=solver, spacing=0.02, support=4.0, sound_speed=20.0, viscosity=0.01)
    else:
        s = FluidSettings(solver=solver, spacing=0.02, support=2.0)

    def make():
        w = gpu_lib.FluidWorld(s)
        w.add_box_container((0.0, 0.0, 0.0), TANK)
        return w

    pos = scenes.lattice_block((0.02, 0.02, 0.02), (8, 8, 8), 0.98 * s.spacing)
    pos = (pos + scenes.jitter(len(pos), 1e-4)).astype(np.float32)
    vel = np.random.default_rng(3).normal(0.0, 0.1, size=pos.shape).astype(np.float32)
    return make, pos, vel


def centroid_loss(P, target):
    c = P.double().mean(dim=0)
    return ((c - target) ** 2).sum()


@pytest.mark.parametrize("solver,every", [(FluidSolver.WCSPH, 10), (FluidSolver.WCSPH, 0), (FluidSolver.DFSPH, 3)])
def test_autograd_gradients_are_step_backwards(gpu_lib, solver, every):
    make, pos, vel = setup(gpu_lib, solver)
    steps, dt = (STEPS, DT) if solver == FluidSolver.WCSPH else (12, 1e-3)
    rng = np.random.default_rng(11)
    gp = rng.normal(size=pos.shape).astype(np.float32)
    gv = rng.normal(size=pos.shape).astype(np.float32)
    p0 = torch.tensor(pos, requires_grad=True)
    v0 = torch.tensor(vel, requires_grad=True)
    P, V = FluidRun.apply(p0, v0, make, steps, dt, every)
    dp0, dv0 = torch.autograd.grad((P, V), (p0, v0), (torch.from_numpy(gp), torch.from_numpy(gv)))
    auto_params = FluidRun.last_params

    w = make()
    w.add_particles(pos, vel)
    ids0 = w.ids().astype(np.int64)
    w.tape_begin(every)
    for _ in range(steps):
        w.step(dt)
    ids1 = w.ids().astype(np.int64)
    # the forward outputs are the run's final state in id order
    assert np.array_equal(P.detach().numpy(), to_id_order(ids1, np.asarray(w.positions(), np.float32)))
    assert np.array_equal(V.detach().numpy(), to_id_order(ids1, np.asarray(w.velocities(), np.float32)))
    ep, ev, params = w.step_backward(gp[ids1], gv[ids1])
    w.tape_end()
    w.close()
    assert np.array_equal(dp0.numpy(), to_id_order(ids0, ep))
    assert np.array_equal(dv0.numpy(), to_id_order(ids0, ev))
    flat = lambda d: np.array([d["viscosity"], d["sound_speed"], *d["gravity"]])
    np.testing.assert_allclose(flat(auto_params), flat(params), rtol=1e-9, atol=1e-300)


def test_a_torch_loss_gets_the_slope_of_central_differences(gpu_lib):
    make, pos, vel = setup(gpu_lib)
    target = torch.tensor(pos.astype(np.float64).mean(axis=0) + np.array([0.3, 0.0, 0.0]))

    def loss_at(v):
        w = make()
        w.add_particles(pos, v)
        for _ in range(STEPS):
            w.step(DT)
        P = torch.from_numpy(np.asarray(w.positions(), dtype=np.float32))
        w.close()
        return float(centroid_loss(P, target))

    p0 = torch.tensor(pos, requires_grad=True)
    v0 = torch.tensor(vel, requires_grad=True)
    P, V = FluidRun.apply(p0, v0, make, STEPS, DT, 10)
    centroid_loss(P, target).backward()
    d = np.random.default_rng(7).normal(size=vel.shape).astype(np.float32)
    d /= np.sqrt(np.mean(d * d))
    ana = float(np.sum(v0.grad.numpy().astype(np.float64) * d))
    best = np.inf
    for eps in (3e-3, 1e-2):
        num = (loss_at((vel + eps * d).astype(np.float32)) - loss_at((vel - eps * d).astype(np.float32))) / (2 * eps)
        best = min(best, abs(ana - num) / abs(num))
    assert best <= 2e-2, best
    assert p0.grad is not None and np.all(np.isfinite(p0.grad.numpy()))
