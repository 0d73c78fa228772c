"""step_backward through warm-started DFSPH solves (the `warm_start` setting).

The reference cold-starts every solve (src/fluid/dfsph.rs:217-229); with `warm_start` each solve
starts with one push at kappa_w = impulse / (2 dt), the impulse (sum of kappa dt) the particle's
solve of the same kind applied the substep before, and the solve's impulse then restarts from
kappa_w dt.  The impulses are state carried from substep to substep, so the backward pass
carries their adjoint too: every push of a solve adds dt of it to its stiffness adjoint, and the
warm push turns its own stiffness adjoint into the previous substep's impulse adjoint.

Same loss and scene as the DFSPH tests of test_gpu_adjoint.py (a 1000-particle block, 5 steps of
1 ms), compared with central differences of the FP64 restatement running the same warm-started
method (tolerance 1e-3 relative), and across tape modes and solve launches (bit for bit).
"""
import numpy as np
import pytest

from solunar_b200 import scenes
from solunar_b200.abi import FluidSettings, FluidSolver

pytestmark = pytest.mark.gpu

STEPS = 5
DT = 1e-3


def settings(**kw):
    # viscosity 0.01: viscosity(dt) = min(0.01 c r, 0.05 r^2 / dt) is on its free branch here
    base = dict(solver=FluidSolver.DFSPH, spacing=0.02, support=2.0, viscosity=0.01, warm_start=True)
    return FluidSettings(**{**base, **kw})


def run(make, vel0=None, s=None):
    w = make(s or settings())
    pos = scenes.lattice_block((0.02, 0.02, 0.02), (10, 10, 10), 0.98 * 0.02)
    pos = (pos + scenes.jitter(len(pos), 1e-4)).astype(np.float32)
    vel = np.random.default_rng(3).normal(0.0, 0.1, size=pos.shape).astype(np.float32)
    w.add_box_container((0.0, 0.0, 0.0), (0.5, 0.5, 0.5))
    w.add_particles(pos, vel if vel0 is None else vel0)
    return w, pos, vel


def loss(w, target):
    c = np.mean(np.asarray(w.positions(), dtype=np.float64), axis=0)
    return float(np.sum((c - target) ** 2)), c


def fd(make, target, vel0=None, s=None):
    w, _, _ = run(make, vel0, s)
    for _ in range(STEPS):
        w.step(DT)
    return loss(w, target)[0]


def taped(w, every, target):
    w.tape_begin(every)
    for _ in range(STEPS):
        w.step(DT)
    L, c = loss(w, target)
    n = w.len()
    dpos = np.tile(2.0 * (c - target) / n, (n, 1)).astype(np.float32)
    out = w.step_backward(dpos, np.zeros_like(dpos))
    w.tape_end()
    return out


@pytest.fixture(scope="module")
def warm_adjoint(gpu_lib):
    w, pos, vel = run(gpu_lib.FluidWorld)
    target = np.mean(pos.astype(np.float64), axis=0) + np.array([0.3, 0.0, 0.0])
    dp0, dv0, params = taped(w, 2, target)
    return pos, vel, target, dp0, dv0, params


def make64(oracle_lib):
    return lambda s: oracle_lib.OracleWorld(s, precision=64, residual_sum=1)


def test_warm_solves_carry_impulses(gpu_lib):
    # the scene's solves start warm from the second substep on: the run differs from a cold one
    warm, _, _ = run(gpu_lib.FluidWorld)
    cold, _, _ = run(gpu_lib.FluidWorld, s=settings(warm_start=False))
    for _ in range(STEPS):
        warm.step(DT)
        cold.step(DT)
    assert warm.state_hash() != cold.state_hash()


def test_warm_velocity_gradient_matches_the_fp64_reference(oracle_lib, warm_adjoint):
    pos, vel, target, dp0, dv0, params = warm_adjoint
    make = make64(oracle_lib)
    rng = np.random.default_rng(5)
    for _ in range(3):
        d = rng.normal(size=vel.shape)
        d /= np.sqrt(np.mean(d * d))
        eps = 3e-5
        vp = (vel + eps * d).astype(np.float32)
        vm = (vel - eps * d).astype(np.float32)
        num = (fd(make, target, vp) - fd(make, target, vm)) / (2 * eps)
        ana = float(np.sum(dv0.astype(np.float64) * (vp.astype(np.float64) - vm.astype(np.float64)) / (2 * eps)))
        assert abs(ana - num) <= 1e-3 * abs(num), (ana, num)


def test_warm_gravity_gradient_matches_the_fp64_reference(oracle_lib, warm_adjoint):
    pos, vel, target, dp0, dv0, params = warm_adjoint
    make = make64(oracle_lib)
    g = list(settings().gravity)
    eps = 1e-3
    num = (fd(make, target, s=settings(gravity=(g[0] + eps, g[1], g[2]))) -
           fd(make, target, s=settings(gravity=(g[0] - eps, g[1], g[2])))) / (2 * eps)
    assert abs(params["gravity"][0] - num) <= 1e-3 * abs(num), (params["gravity"][0], num)


def same_params(a, b):
    flat = lambda d: np.array([d["viscosity"], d["sound_speed"], *d["gravity"]])
    np.testing.assert_allclose(flat(a), flat(b), rtol=1e-9, atol=1e-300)


@pytest.mark.parametrize("every", [0, 1, 3])
def test_warm_tape_modes_give_identical_gradients(gpu_lib, warm_adjoint, every):
    pos, vel, target, dp0, dv0, params = warm_adjoint
    w, _, _ = run(gpu_lib.FluidWorld)
    dp, dv, pr = taped(w, every, target)
    assert np.array_equal(dp, dp0) and np.array_equal(dv, dv0)
    same_params(pr, params)


def test_warm_gradients_do_not_depend_on_how_solves_launch(gpu_lib, warm_adjoint):
    pos, vel, target, dp0, dv0, params = warm_adjoint
    w, _, _ = run(gpu_lib.FluidWorld)
    w.solver_graphs(False)
    dp, dv, pr = taped(w, 2, target)
    assert np.array_equal(dp, dp0) and np.array_equal(dv, dv0)
    same_params(pr, params)


def test_the_backward_pass_leaves_the_warm_state_as_it_was(gpu_lib, warm_adjoint):
    # the impulses are part of the state: the step after a backward pass is the untaped one
    pos, vel, target, *_ = warm_adjoint
    a, _, _ = run(gpu_lib.FluidWorld)
    taped(a, 2, target)
    b, _, _ = run(gpu_lib.FluidWorld)
    for _ in range(STEPS):
        b.step(DT)
    a.step(DT)
    b.step(DT)
    assert a.state_hash() == b.state_hash()
