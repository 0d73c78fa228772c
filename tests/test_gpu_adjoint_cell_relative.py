"""step_backward with cell-relative positions (SLF_POSITIONS_CELL_RELATIVE, FAST arithmetic).

The adjoint forms each pair's offset as the forward pass does, from the two particles' offsets
and the cell step the list entry carries, (o_i - o_j) - step r, and its tapes keep each
particle's cell beside its offset.  Checked as the absolute-position adjoint is
(tests/test_gpu_adjoint.py): the gradient of the centroid loss along seeded directions of the
initial velocities against central differences of the FP64 restatement (absolute positions in
double), within 1e-3 relative, on the small WCSPH and DFSPH blocks near the origin and 1024 m
away from it, where an f32 coordinate resolves 1.2e-4 m (1/160 of the 0.02 m spacing) and an
adjoint on absolute f32 positions would see the pair geometry through that rounding.  The tape's
modes (every substep recorded, checkpoints) give identical particle gradients.
"""
import numpy as np
import pytest

from solunar_b200 import scenes
from solunar_b200.abi import Arithmetic, FluidSettings, FluidSolver, Positions

pytestmark = pytest.mark.gpu

FAR = np.array([1024.0, 1024.0, 1024.0])


def settings(solver, **kw):
    base = dict(solver=solver, spacing=0.02, support=4.0 if solver == FluidSolver.WCSPH else 2.0,
                sound_speed=20.0, viscosity=0.01)
    base.update(kw)
    return FluidSettings(**base)


def rel(s):
    s.positions = Positions.CELL_RELATIVE
    s.arithmetic = Arithmetic.FAST
    return s


def block(solver):
    counts = (8, 8, 8) if solver == FluidSolver.WCSPH else (10, 10, 10)
    pos = scenes.lattice_block((0.02, 0.02, 0.02), counts, 0.98 * 0.02)
    pos = (pos + scenes.jitter(len(pos), 1e-4)).astype(np.float64)
    vel = np.random.default_rng(3).normal(0.0, 0.1, size=pos.shape).astype(np.float32)
    return pos, vel


def build(make, s, origin, vel0=None):
    solver = s.solver
    pos, vel = block(solver)
    tank = (0.4, 0.4, 0.4) if solver == FluidSolver.WCSPH else (0.5, 0.5, 0.5)
    w = make(s)
    w.add_box_container(tuple(origin), tuple(origin + np.array(tank)))
    w.add_particles((pos + origin).astype(np.float32), vel if vel0 is None else vel0)
    return w, (pos + origin).astype(np.float32), vel


RUNS = {FluidSolver.WCSPH: (20, 2e-4, 5), FluidSolver.DFSPH: (5, 1e-3, 2)}


def centroid_loss(w, target):
    c = np.mean(np.asarray(w.positions(), dtype=np.float64), axis=0)
    return float(np.sum((c - target) ** 2)), c


def adjoint(gpu_lib, solver, origin, every=None):
    steps, dt, default_every = RUNS[solver]
    w, pos, vel = build(gpu_lib.FluidWorld, rel(settings(solver)), origin)
    target = np.mean(pos.astype(np.float64), axis=0) + np.array([0.3, 0.0, 0.0])
    w.tape_begin(default_every if every is None else every)
    for _ in range(steps):
        w.step(dt)
    _, c = centroid_loss(w, target)
    n = w.len()
    dpos = np.tile(2.0 * (c - target) / n, (n, 1)).astype(np.float32)
    dp0, dv0, params = w.step_backward(dpos, np.zeros_like(dpos))
    w.tape_end()
    w.close()
    return vel, target, dp0, dv0


def fp64_loss(oracle_lib, solver, origin, target, vel0):
    steps, dt, _ = RUNS[solver]
    w, _, _ = build(lambda s: oracle_lib.OracleWorld(s, precision=64, residual_sum=1), settings(solver), origin,
                    vel0)
    for _ in range(steps):
        w.step(dt)
    return centroid_loss(w, target)[0]


@pytest.mark.parametrize("solver", [FluidSolver.WCSPH, FluidSolver.DFSPH])
@pytest.mark.parametrize("far", [False, True])
def test_cell_relative_gradient_matches_fp64_differences(gpu_lib, oracle_lib, solver, far):
    origin = FAR if far else np.zeros(3)
    vel, target, dp0, dv0 = adjoint(gpu_lib, solver, origin)
    assert np.isfinite(dv0).all() and np.isfinite(dp0).all()
    rng = np.random.default_rng(17)
    within = []
    for _ in range(4):
        d = rng.normal(size=vel.shape)
        d /= np.sqrt(np.mean(d * d))
        best = np.inf
        for eps in (1e-4, 3e-5):
            # the restatement takes float inputs: the adjoint is projected on the rounded change
            vp = (vel + eps * d).astype(np.float32)
            vm = (vel - eps * d).astype(np.float32)
            num = (fp64_loss(oracle_lib, solver, origin, target, vp) -
                   fp64_loss(oracle_lib, solver, origin, target, vm)) / (2 * eps)
            ana = float(np.sum(dv0.astype(np.float64) * (vp.astype(np.float64) - vm.astype(np.float64)) / (2 * eps)))
            best = min(best, abs(ana - num) / abs(num))
        within.append(best <= 1e-3)
    assert sum(within) >= 3, within


@pytest.mark.parametrize("solver", [FluidSolver.WCSPH, FluidSolver.DFSPH])
def test_cell_relative_tape_modes_give_identical_gradients(gpu_lib, solver):
    _, _, dp_a, dv_a = adjoint(gpu_lib, solver, FAR, every=0)
    _, _, dp_b, dv_b = adjoint(gpu_lib, solver, FAR, every=1)
    assert np.array_equal(dp_a, dp_b) and np.array_equal(dv_a, dv_b)
