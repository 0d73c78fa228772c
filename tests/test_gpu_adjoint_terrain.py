"""step_backward with terrain ground (src/fluid/terrain.rs), WCSPH.

A block of water thrown down at 1.5 m/s into the reference's test trench (tests/trench.py): its
lowest layer starts 3 cm above the bed, within reach of the ground's density, and with a soft
fluid (sound speed 2 m/s; at 20 m/s the ground's pressure stops the block 4 cm above the bed) the
whole layer reaches the contact distance (half a spacing) and stays there.  The adjoint takes the
ground's four terms:

  * its density (terrain.rs:144-171, mod.rs:657-663), whose derivative is the slope the density
    pass keeps;
  * the push it gives with each particle's own pressure, -slope (s_i + p_i / rho_0^2)
    (step.rs:203-205), through the trilinear field's second derivatives;
  * its damping in the wall viscosity (step.rs:281-296), through the damping table's slope and
    the unit normal;
  * terrain contact after the advance (terrain.rs:314-333), reversed region by region.

Checked as the other adjoints are (tests/test_gpu_adjoint.py): along seeded directions of the
initial velocities against central differences of the FP64 restatement with the same terrain
(eps 1e-4 and 3e-5, the better of the two), within 1e-3 relative on at least three of four
directions; the viscosity and sound-speed gradients against central differences of the FP64
restatement, within 1e-3 (differences of the library's FP32 forward sit at the loss's FP32
resolution here: 3.6 % off for the viscosity, where the FP64 ones agree with the adjoint to
1e-6); and the tape's modes (every substep recorded, checkpoints) give identical gradients.
"""
import numpy as np
import pytest

import trench
from solunar_b200 import scenes
from solunar_b200.abi import FluidSettings, FluidSolver

pytestmark = pytest.mark.gpu

STEPS = 15
DT = 2e-3
SETTINGS = dict(solver=FluidSolver.WCSPH, spacing=0.05, support=4.0, sound_speed=2.0, viscosity=0.01)


def initial():
    pos = scenes.lattice_block((0.6, -0.37, -0.13), (6, 3, 6), 0.98 * SETTINGS["spacing"])
    pos = (pos + scenes.jitter(len(pos), 1e-4)).astype(np.float32)
    vel = np.random.default_rng(5).normal(0.0, 0.1, size=pos.shape)
    vel[:, 1] -= 1.5
    return pos, vel.astype(np.float32)


def build(make, settings, vel0=None):
    w = make(settings)
    trench.add_trench(w, SETTINGS["spacing"])
    pos, vel = initial()
    w.add_particles(pos, vel if vel0 is None else vel0)
    return w, pos, vel


def centroid_loss(w, target):
    c = np.mean(np.asarray(w.positions(), dtype=np.float64), axis=0)
    return float(np.sum((c - target) ** 2)), c


def target_of(pos):
    return np.mean(pos.astype(np.float64), axis=0) + np.array([0.3, 0.0, 0.0])


def adjoint_run(gpu_lib, every):
    w, pos, vel = build(gpu_lib.FluidWorld, FluidSettings(**SETTINGS))
    target = target_of(pos)
    w.tape_begin(every)
    for _ in range(STEPS):
        w.step(DT)
    low = float(np.min(np.asarray(w.positions())[:, 1]))
    _, c = centroid_loss(w, target)
    n = w.len()
    dpos = np.tile(2.0 * (c - target) / n, (n, 1)).astype(np.float32)
    dp0, dv0, params = w.step_backward(dpos, np.zeros_like(dpos))
    w.tape_end()
    w.close()
    return pos, vel, target, dp0, dv0, params, low


@pytest.fixture(scope="module")
def adjoint(gpu_lib):
    return adjoint_run(gpu_lib, 4)


def fp64_loss(oracle_lib, target, vel0=None, **settings):
    w, _, _ = build(lambda s: oracle_lib.OracleWorld(s, precision=64), FluidSettings(**{**SETTINGS, **settings}),
                    vel0)
    for _ in range(STEPS):
        w.step(DT)
    return centroid_loss(w, target)[0]


def test_the_run_reaches_the_ground(adjoint):
    # the lowest particle ends at the contact distance of the bed at y = -0.4
    low = adjoint[-1]
    assert low < -0.4 + SETTINGS["spacing"] / 2 + 1e-4


def test_velocity_gradient_matches_fp64_differences(oracle_lib, adjoint):
    pos, vel, target, dp0, dv0, params, _ = adjoint
    assert np.isfinite(dv0).all() and np.isfinite(dp0).all()
    rng = np.random.default_rng(23)
    within = []
    for _ in range(4):
        d = rng.normal(size=vel.shape)
        d /= np.sqrt(np.mean(d * d))
        best = np.inf
        for eps in (1e-4, 3e-5):
            # the restatement takes float inputs: the adjoint is projected on the rounded change
            vp = (vel + eps * d).astype(np.float32)
            vm = (vel - eps * d).astype(np.float32)
            num = (fp64_loss(oracle_lib, target, vp) - fp64_loss(oracle_lib, target, vm)) / (2 * eps)
            ana = float(np.sum(dv0.astype(np.float64) * (vp.astype(np.float64) - vm.astype(np.float64)) / (2 * eps)))
            best = min(best, abs(ana - num) / abs(num))
        within.append(best <= 1e-3)
    assert sum(within) >= 3, within


def test_parameter_gradients_match_fp64_differences(oracle_lib, adjoint):
    pos, vel, target, dp0, dv0, params, _ = adjoint
    for name, eps in [("viscosity", 1e-4), ("sound_speed", 2e-3)]:
        hi = fp64_loss(oracle_lib, target, **{name: SETTINGS[name] + eps})
        lo = fp64_loss(oracle_lib, target, **{name: SETTINGS[name] - eps})
        num = (hi - lo) / (2 * eps)
        assert abs(params[name] - num) <= 1e-3 * abs(num), (name, params[name], num)


def test_tape_modes_give_identical_gradients(gpu_lib, adjoint):
    _, _, _, dp_a, dv_a, _, _ = adjoint
    for every in (0, 1):
        _, _, _, dp_b, dv_b, _, _ = adjoint_run(gpu_lib, every)
        assert np.array_equal(dp_a, dp_b) and np.array_equal(dv_a, dv_b), every
