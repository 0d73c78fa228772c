"""step_backward: the hand-written WCSPH adjoint against finite differences.

Loss: the squared distance of the fluid's centroid after the run to a point 0.3 m downstream
of where it started (the differentiable WCSPH configuration, on a smaller block).  Gradients with
respect to the initial velocities (along seeded random directions), the viscosity, the sound
speed and gravity are compared with central differences.

The reference's model is not smooth everywhere: pressure is clamped at zero below rest density
(src/fluid/step.rs:156), where a jittered lattice at rest sits; viscosity acts only on approach
(step.rs:192); walls clamp positions (step.rs:311-328).  A difference whose interval straddles
one of these kinks measures a different slope, and at eps = 1e-3 m/s many do.  Stated tolerances:
  * against central differences of the FP64 restatement at eps 1e-4 and 3e-5 (the better of the
    two): relative error 1e-3, on at least three of four directions;
  * against central differences of the GPU forward in FP32 (the better of eps 3e-3 and 1e-2;
    smaller steps drown in the FP32 resolution of the loss, larger ones in its curvature):
    relative error 2e-2;
  * parameters (viscosity, sound speed, gravity): relative error 2e-2 against FP32 differences.
"""
import numpy as np
import pytest

from solunar_b200 import scenes
from solunar_b200.abi import FluidSettings, FluidSolver

pytestmark = pytest.mark.gpu

STEPS = 30
DT = 2e-4


def scene():
    s = FluidSettings(solver=FluidSolver.WCSPH, spacing=0.02, support=4.0, sound_speed=20.0, viscosity=0.01)
    sc = scenes.Scene("adjoint_dam", s, (0.4, 0.4, 0.4), (8, 8, 8), jitter=1e-4, velocity_sigma=0.1,
                      dt=DT, steps=STEPS)
    return sc


def initial(sc):
    # the block starts 2 % denser than rest (lattice at 0.98 of the spacing): its pressures are
    # clearly positive inside and clearly clamped at the free surface, so few particles sit on
    # the pressure clamp's kink at rest density
    pos = scenes.lattice_block((0.02, 0.02, 0.02), sc.block_counts, 0.98 * sc.settings.spacing)
    pos = (pos + scenes.jitter(len(pos), sc.jitter)).astype(np.float32)
    vel = np.random.default_rng(3).normal(0.0, sc.velocity_sigma, size=pos.shape).astype(np.float32)
    return pos, vel


def run(make, sc, vel0=None, settings=None):
    w = make(settings or sc.settings)
    pos, vel = initial(sc)
    w.add_box_container((0.0, 0.0, 0.0), sc.tank)
    w.add_particles(pos, vel if vel0 is None else vel0)
    return w, pos, vel


def loss(w, target):
    c = np.mean(np.asarray(w.positions(), dtype=np.float64), axis=0)
    return float(np.sum((c - target) ** 2)), c


@pytest.fixture(scope="module")
def adjoint(gpu_lib):
    sc = scene()
    w, pos, vel = run(gpu_lib.FluidWorld, sc)
    target = np.mean(pos.astype(np.float64), axis=0) + np.array([0.3, 0.0, 0.0])
    w.tape_begin(10)
    for _ in range(STEPS):
        w.step(DT)
    L, c = loss(w, target)
    n = w.len()
    dpos = np.tile(2.0 * (c - target) / n, (n, 1)).astype(np.float32)
    dp0, dv0, params = w.step_backward(dpos, np.zeros_like(dpos))
    # the state is left where the run ended
    L2, _ = loss(w, target)
    assert L2 == L
    return sc, pos, vel, target, dp0, dv0, params


def fd(make, sc, target, vel0=None, settings=None):
    w, _, _ = run(make, sc, vel0, settings)
    for _ in range(STEPS):
        w.step(DT)
    return loss(w, target)[0]


def test_velocity_gradient_matches_central_differences(gpu_lib, adjoint):
    sc, pos, vel, target, dp0, dv0, params = adjoint
    rng = np.random.default_rng(7)
    for _ in range(3):
        d = rng.normal(size=vel.shape).astype(np.float32)
        d /= np.sqrt(np.mean(d * d))
        ana = float(np.sum(dv0.astype(np.float64) * d))
        best = np.inf
        for eps in (3e-3, 1e-2):
            lp = fd(gpu_lib.FluidWorld, sc, target, (vel + eps * d).astype(np.float32))
            lm = fd(gpu_lib.FluidWorld, sc, target, (vel - eps * d).astype(np.float32))
            num = (lp - lm) / (2 * eps)
            best = min(best, abs(ana - num) / abs(num))
        assert best <= 2e-2, best


def test_parameter_gradients_match_central_differences(gpu_lib, adjoint):
    sc, pos, vel, target, dp0, dv0, params = adjoint
    s = sc.settings
    for name, eps in [("viscosity", 1e-3), ("sound_speed", 2e-2)]:
        base = getattr(s, name)
        hi = FluidSettings(**{**s.__dict__, name: base + eps})
        lo = FluidSettings(**{**s.__dict__, name: base - eps})
        num = (fd(gpu_lib.FluidWorld, sc, target, settings=hi) - fd(gpu_lib.FluidWorld, sc, target, settings=lo)) / (2 * eps)
        assert abs(params[name] - num) <= 2e-2 * abs(num) + 1e-7, (name, params[name], num)
    g = list(s.gravity)
    eps = 1e-2
    hi = FluidSettings(**{**s.__dict__, "gravity": (g[0] + eps, g[1], g[2])})
    lo = FluidSettings(**{**s.__dict__, "gravity": (g[0] - eps, g[1], g[2])})
    num = (fd(gpu_lib.FluidWorld, sc, target, settings=hi) - fd(gpu_lib.FluidWorld, sc, target, settings=lo)) / (2 * eps)
    assert abs(params["gravity"][0] - num) <= 1e-2 * abs(num) + 1e-9, (params["gravity"][0], num)


def test_velocity_gradient_matches_the_fp64_reference(oracle_lib, adjoint):
    sc, pos, vel, target, dp0, dv0, params = adjoint
    make64 = lambda s: oracle_lib.OracleWorld(s, precision=64)
    rng = np.random.default_rng(11)
    within = []
    for _ in range(4):
        d = rng.normal(size=vel.shape)
        d /= np.sqrt(np.mean(d * d))
        best = np.inf
        for eps in (1e-4, 3e-5):
            # the FP64 restatement takes float inputs: the perturbed velocities are rounded to
            # f32, so the adjoint is projected on the difference actually applied
            vp = (vel + eps * d).astype(np.float32)
            vm = (vel - eps * d).astype(np.float32)
            num = (fd(make64, sc, target, vp) - fd(make64, sc, target, vm)) / (2 * eps)
            ana = float(np.sum(dv0.astype(np.float64) * (vp.astype(np.float64) - vm.astype(np.float64)) / (2 * eps)))
            best = min(best, abs(ana - num) / abs(num))
        within.append(best <= 1e-3)
    assert sum(within) >= 3, within


# ---- DFSPH: the same loss through 5 substeps (25 solver iterations), tape checkpoint every 2 ----

DFSPH_STEPS = 5
DFSPH_DT = 1e-3


def dfsph_settings(**kw):
    # viscosity 0.01: viscosity(dt) = min(0.01 c r, 0.05 r^2 / dt) is on its free branch here
    return FluidSettings(**{**dict(solver=FluidSolver.DFSPH, spacing=0.02, support=2.0, viscosity=0.01), **kw})


def dfsph_run(make, vel0=None, settings=None):
    w = make(settings or dfsph_settings())
    pos = scenes.lattice_block((0.02, 0.02, 0.02), (10, 10, 10), 0.98 * 0.02)
    pos = (pos + scenes.jitter(len(pos), 1e-4)).astype(np.float32)
    vel = np.random.default_rng(3).normal(0.0, 0.1, size=pos.shape).astype(np.float32)
    w.add_box_container((0.0, 0.0, 0.0), (0.5, 0.5, 0.5))
    w.add_particles(pos, vel if vel0 is None else vel0)
    return w, pos, vel


def dfsph_fd(make, target, vel0=None, settings=None):
    w, _, _ = dfsph_run(make, vel0, settings)
    for _ in range(DFSPH_STEPS):
        w.step(DFSPH_DT)
    return loss(w, target)[0]


@pytest.fixture(scope="module")
def dfsph_adjoint(gpu_lib):
    w, pos, vel = dfsph_run(gpu_lib.FluidWorld)
    target = np.mean(pos.astype(np.float64), axis=0) + np.array([0.3, 0.0, 0.0])
    w.tape_begin(2)
    for _ in range(DFSPH_STEPS):
        w.step(DFSPH_DT)
    L, c = loss(w, target)
    n = w.len()
    dpos = np.tile(2.0 * (c - target) / n, (n, 1)).astype(np.float32)
    dp0, dv0, params = w.step_backward(dpos, np.zeros_like(dpos))
    return pos, vel, target, dp0, dv0, params


def test_dfsph_velocity_gradient_matches_the_fp64_reference(oracle_lib, dfsph_adjoint):
    # the solves' iteration counts are the forward's; at these small steps they do not change
    pos, vel, target, dp0, dv0, params = dfsph_adjoint
    make64 = lambda s: oracle_lib.OracleWorld(s, precision=64, residual_sum=1)
    rng = np.random.default_rng(5)
    for _ in range(3):
        d = rng.normal(size=vel.shape)
        d /= np.sqrt(np.mean(d * d))
        eps = 3e-5
        vp = (vel + eps * d).astype(np.float32)
        vm = (vel - eps * d).astype(np.float32)
        num = (dfsph_fd(make64, target, vp) - dfsph_fd(make64, target, vm)) / (2 * eps)
        ana = float(np.sum(dv0.astype(np.float64) * (vp.astype(np.float64) - vm.astype(np.float64)) / (2 * eps)))
        assert abs(ana - num) <= 1e-3 * abs(num), (ana, num)


def test_dfsph_parameter_gradients_match_the_fp64_reference(oracle_lib, dfsph_adjoint):
    # the loss moves by about 1e-10 for a 1e-3 change of the viscosity: below what FP32 positions
    # resolve, so the differences are taken on the FP64 restatement
    pos, vel, target, dp0, dv0, params = dfsph_adjoint
    make64 = lambda s: oracle_lib.OracleWorld(s, precision=64, residual_sum=1)
    s = dfsph_settings()
    eps = 1e-4
    num = (dfsph_fd(make64, target, settings=dfsph_settings(viscosity=s.viscosity + eps)) -
           dfsph_fd(make64, target, settings=dfsph_settings(viscosity=s.viscosity - eps))) / (2 * eps)
    assert abs(params["viscosity"] - num) <= 1e-2 * abs(num), (params["viscosity"], num)
    g = list(s.gravity)
    eps = 1e-3
    num = (dfsph_fd(make64, target, settings=dfsph_settings(gravity=(g[0] + eps, g[1], g[2]))) -
           dfsph_fd(make64, target, settings=dfsph_settings(gravity=(g[0] - eps, g[1], g[2])))) / (2 * eps)
    assert abs(params["gravity"][0] - num) <= 1e-3 * abs(num), (params["gravity"][0], num)


# ---- tape modes: keeping every substep's record, or checkpoints at any spacing, feed the
# backward pass the same forward values (recomputation is bit-identical), so the particle
# gradients agree bit for bit; the parameter gradients are FP64 sums taken with atomics, whose
# order varies, so they agree to 1e-9 ----

def same_params(a, b):
    flat = lambda d: np.array([d["viscosity"], d["sound_speed"], *d["gravity"]])
    np.testing.assert_allclose(flat(a), flat(b), rtol=1e-9, atol=1e-300)

def taped_gradients(w, steps, dt, every, target):
    w.tape_begin(every)
    for _ in range(steps):
        w.step(dt)
    L, c = loss(w, target)
    n = w.len()
    dpos = np.tile(2.0 * (c - target) / n, (n, 1)).astype(np.float32)
    out = w.step_backward(dpos, np.zeros_like(dpos))
    w.tape_end()
    return out


@pytest.mark.parametrize("every", [0, 1, 3])
def test_dfsph_tape_modes_give_identical_gradients(gpu_lib, dfsph_adjoint, every):
    pos, vel, target, dp0, dv0, params = dfsph_adjoint
    w, _, _ = dfsph_run(gpu_lib.FluidWorld)
    dp, dv, pr = taped_gradients(w, DFSPH_STEPS, DFSPH_DT, every, target)
    assert np.array_equal(dp, dp0) and np.array_equal(dv, dv0)
    same_params(pr, params)


@pytest.mark.parametrize("warm", [False, True])
def test_dfsph_kept_segments_give_identical_gradients(gpu_lib, warm):
    # 40 checkpoints, one a substep: enough segments that the backward keeps each segment's
    # substeps in their records with the solves as graphs, against a tape that recorded every
    # substep as it ran (the same records, the lists from the world's replay of each substep)
    steps = 40
    target = np.array([0.4, 0.1, 0.1])
    out = []
    for every in (0, 1):
        w, _, _ = dfsph_run(gpu_lib.FluidWorld, settings=dfsph_settings(warm_start=warm))
        out.append(taped_gradients(w, steps, DFSPH_DT, every, target))
        w.close()
    (dp0, dv0, p0), (dp1, dv1, p1) = out
    assert np.isfinite(dv0).all() and np.abs(dv0).max() > 0
    assert np.array_equal(dp1, dp0) and np.array_equal(dv1, dv0)
    same_params(p1, p0)


def test_wcsph_recorded_tape_gives_identical_gradients(gpu_lib, adjoint):
    sc, pos, vel, target, dp0, dv0, params = adjoint
    w, _, _ = run(gpu_lib.FluidWorld, sc)
    dp, dv, pr = taped_gradients(w, STEPS, DT, 0, target)
    assert np.array_equal(dp, dp0) and np.array_equal(dv, dv0)
    same_params(pr, params)


@pytest.mark.parametrize("every", [0, 2])
def test_dfsph_gradients_do_not_depend_on_how_solves_launch(gpu_lib, dfsph_adjoint, every):
    # the fixture's world ran its solves as CUDA graphs (the default); here they run in batches of
    # launches with host checks between them, forward and recorded alike
    pos, vel, target, dp0, dv0, params = dfsph_adjoint
    w, _, _ = dfsph_run(gpu_lib.FluidWorld)
    w.solver_graphs(False)
    dp, dv, pr = taped_gradients(w, DFSPH_STEPS, DFSPH_DT, every, target)
    assert np.array_equal(dp, dp0) and np.array_equal(dv, dv0)
    same_params(pr, params)


# ---- against the FP64 tangent: the restatement run in forward-mode derivative numbers
# (oracle/dual.hpp, oracle/oracle_tangent.cpp) gives the exact derivative of the FP64 method along a
# direction d, with no step size; the adjoint (J^T g) must meet it through <g, J d> = <J^T g, d>.
# What separates the two is the FP32 trajectory and arithmetic of the adjoint against the FP64 ones
# of the tangent: relative error 1e-5 on the velocity directions and 1e-4 on the parameters
# (measured on B200: at most 4.5e-7 and 2.0e-5) ----

def tangent_projections(oracle_lib, settings, tank, pos, vel, target, steps, dt, directions, dparams, precision=64):
    """<g, dP> of the tangent for each velocity direction, then each parameter seed."""
    n = len(pos)
    zero = np.zeros(pos.shape)
    out = []
    for d, dq in [(d, np.zeros(5)) for d in directions] + [(zero, q) for q in dparams]:
        P, _, dP, _, _ = oracle_lib.tangent_run(settings, ((0.0, 0.0, 0.0), tank), pos, vel, zero, d, dparams=dq,
                                                steps=steps, dt=dt, precision=precision)
        c = P.mean(axis=0)
        out.append(float(np.sum((2.0 * (c - target) / n) * dP)))
    return out


def seeds(which):
    out = []
    for k in which:
        q = np.zeros(5)
        q[k] = 1.0
        out.append(q)
    return out


def test_wcsph_gradients_match_the_fp64_tangent(oracle_lib, adjoint):
    sc, pos, vel, target, dp0, dv0, params = adjoint
    rng = np.random.default_rng(13)
    directions = [rng.normal(size=vel.shape) for _ in range(3)]
    tan = tangent_projections(oracle_lib, sc.settings, sc.tank, pos, vel, target, STEPS, DT, directions,
                              seeds([0, 1, 2]))
    ana = [float(np.sum(dv0.astype(np.float64) * d)) for d in directions]
    ana += [params["viscosity"], params["sound_speed"], params["gravity"][0]]
    rel = [abs(a - t) / abs(t) for a, t in zip(ana, tan)]
    print("WCSPH adjoint vs FP64 tangent, relative:", rel)
    assert max(rel[:3]) <= 1e-5 and max(rel[3:]) <= 1e-4, (rel, ana, tan)


def test_dfsph_gradients_match_the_fp64_tangent(oracle_lib, dfsph_adjoint):
    pos, vel, target, dp0, dv0, params = dfsph_adjoint
    rng = np.random.default_rng(17)
    directions = [rng.normal(size=vel.shape) for _ in range(3)]
    tan = tangent_projections(oracle_lib, dfsph_settings(), (0.5, 0.5, 0.5), pos, vel, target, DFSPH_STEPS, DFSPH_DT,
                              directions, seeds([0, 2]))
    ana = [float(np.sum(dv0.astype(np.float64) * d)) for d in directions]
    ana += [params["viscosity"], params["gravity"][0]]
    rel = [abs(a - t) / abs(t) for a, t in zip(ana, tan)]
    print("DFSPH adjoint vs FP64 tangent, relative:", rel)
    assert max(rel[:3]) <= 1e-5 and max(rel[3:]) <= 1e-4, (rel, ana, tan)


# ---- against the FP32 program's own derivative: the restatement in derivative numbers whose
# values are the float restatement's (and so the library's) bit for bit, derivatives in double; it
# takes every branch the library's forward takes, so what remains is the adjoint's own FP32
# arithmetic ----

@pytest.mark.parametrize("solver", ["wcsph", "dfsph"])
def test_gradients_match_the_fp32_programs_tangent(oracle_lib, adjoint, dfsph_adjoint, solver):
    if solver == "wcsph":
        sc, pos, vel, target, dp0, dv0, params = adjoint
        settings, tank, steps, dt, which = sc.settings, sc.tank, STEPS, DT, [0, 1, 2]
        names = [params["viscosity"], params["sound_speed"], params["gravity"][0]]
    else:
        pos, vel, target, dp0, dv0, params = dfsph_adjoint
        settings, tank, steps, dt, which = dfsph_settings(), (0.5, 0.5, 0.5), DFSPH_STEPS, DFSPH_DT, [0, 2]
        names = [params["viscosity"], params["gravity"][0]]
    rng = np.random.default_rng(19)
    directions = [rng.normal(size=vel.shape) for _ in range(3)]
    tan = tangent_projections(oracle_lib, settings, tank, pos, vel, target, steps, dt, directions, seeds(which),
                              precision=32)
    ana = [float(np.sum(dv0.astype(np.float64) * d)) for d in directions] + names
    rel = [abs(a - t) / abs(t) for a, t in zip(ana, tan)]
    print(solver, "adjoint vs FP32 tangent, relative:", rel)
    assert max(rel[:3]) <= 1e-5 and max(rel[3:]) <= 1e-4, (rel, ana, tan)
