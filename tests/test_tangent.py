"""The FP64 forward-mode restatement (oracle/dual.hpp, oracle/oracle_tangent.cpp) against central
differences of the FP64 restatement itself.

`tangent_run` carries the derivative of every quantity along one direction of the inputs.  Its
values must be the FP64 world's bit for bit, and its tangents the FP64 world's central differences
at eps 1e-6, where the model's kinks (the pressure clamp, approach-only viscosity, wall clamps)
are crossed by few pairs: relative error 1e-5.  The inputs are float32, so each difference is
divided by the perturbation the float32 inputs actually got.  The GPU adjoint is checked against
these tangents in tests/test_gpu_adjoint.py.
"""
import dataclasses

import numpy as np
import pytest

from solunar_b200 import scenes
from solunar_b200.abi import FluidSettings, FluidSolver

TANK = ((0.0, 0.0, 0.0), (0.4, 0.4, 0.4))


def case(solver):
    if solver == FluidSolver.WCSPH:
        s = FluidSettings(solver=solver, spacing=0.02, support=4.0, sound_speed=20.0, viscosity=0.01)
        steps, dt = 10, 2e-4
    else:
        s = FluidSettings(solver=solver, spacing=0.02, support=2.0)
        steps, dt = 6, 1e-3
    pos = scenes.lattice_block((0.02, 0.02, 0.02), (8, 8, 8), 0.98 * s.spacing)
    pos = (pos + scenes.jitter(len(pos), 1e-4)).astype(np.float32)
    vel = np.random.default_rng(3).normal(0.0, 0.1, size=pos.shape).astype(np.float32)
    return s, steps, dt, pos, vel


def run64(oracle_lib, s, steps, dt, pos, vel):
    w = oracle_lib.OracleWorld(s, precision=64, residual_sum=1)
    w.add_box_container(*TANK)
    w.add_particles(pos, vel)
    for _ in range(steps):
        w.step(dt)
    order = np.argsort(w.ids())
    return np.asarray(w.positions())[order], np.asarray(w.velocities())[order]


@pytest.mark.parametrize("solver,warm", [(FluidSolver.WCSPH, False), (FluidSolver.DFSPH, False),
                                         (FluidSolver.DFSPH, True)])
def test_tangent_values_are_the_fp64_restatements_and_tangents_its_differences(oracle_lib, solver, warm):
    # warm: warm-started solves, whose impulses carry derivatives from substep to substep
    s, steps, dt, pos, vel = case(solver)
    s = dataclasses.replace(s, warm_start=warm)
    d = np.random.default_rng(7).normal(size=vel.shape)
    P, V, dP, dV, ids = oracle_lib.tangent_run(s, TANK, pos, vel, np.zeros_like(d), d, steps=steps, dt=dt)
    assert np.array_equal(ids, np.arange(len(pos)))
    P64, V64 = run64(oracle_lib, s, steps, dt, pos, vel)
    assert np.array_equal(P, P64) and np.array_equal(V, V64)
    eps = 1e-6
    vp = (vel.astype(np.float64) + eps * d).astype(np.float32)
    vm = (vel.astype(np.float64) - eps * d).astype(np.float32)
    moved = (vp.astype(np.float64) - vm.astype(np.float64)) / 2.0
    _, _, dPm, dVm, _ = oracle_lib.tangent_run(s, TANK, pos, vel, np.zeros_like(d), moved, steps=steps, dt=dt)
    (Pp, Vp), (Pm, Vm) = run64(oracle_lib, s, steps, dt, pos, vp), run64(oracle_lib, s, steps, dt, pos, vm)
    assert np.linalg.norm((Pp - Pm) / 2.0 - dPm) <= 1e-5 * np.linalg.norm(dPm)
    assert np.linalg.norm((Vp - Vm) / 2.0 - dVm) <= 1e-5 * np.linalg.norm(dVm)


@pytest.mark.parametrize("solver,name,which", [(FluidSolver.WCSPH, "viscosity", 0), (FluidSolver.WCSPH, "sound_speed", 1),
                                               (FluidSolver.WCSPH, "gravity", 2), (FluidSolver.DFSPH, "viscosity", 0),
                                               (FluidSolver.DFSPH, "gravity", 2)])
def test_parameter_tangents_are_the_fp64_restatements_differences(oracle_lib, solver, name, which):
    s, steps, dt, pos, vel = case(solver)
    dq = np.zeros(5)
    dq[which] = 1.0
    zero = np.zeros(pos.shape)
    _, _, dP, _, _ = oracle_lib.tangent_run(s, TANK, pos, vel, zero, zero, dparams=dq, steps=steps, dt=dt)

    def with_value(delta):
        if name == "gravity":
            g = list(s.gravity)
            g[0] = float(np.float32(g[0] + delta))
            return dataclasses.replace(s, gravity=tuple(g)), g[0]
        v = float(np.float32(getattr(s, name) + delta))
        return dataclasses.replace(s, **{name: v}), v

    base = s.gravity[0] if name == "gravity" else getattr(s, name)
    eps = 1e-5 * max(abs(base), 1.0)
    (sp, hi), (sm, lo) = with_value(eps), with_value(-eps)
    num = (run64(oracle_lib, sp, steps, dt, pos, vel)[0] - run64(oracle_lib, sm, steps, dt, pos, vel)[0]) / (hi - lo)
    assert np.linalg.norm(num - dP) <= 1e-4 * np.linalg.norm(dP), (np.linalg.norm(num - dP), np.linalg.norm(dP))


def test_a_run_held_to_its_own_solver_iterations_is_the_same_run(oracle_lib):
    # forced iteration counts (the counts another run's solves took) change nothing when they are
    # the counts this run takes anyway, and change the run when they are not
    s, steps, dt, pos, vel = case(FluidSolver.DFSPH)
    w = oracle_lib.OracleWorld(s, precision=64, residual_sum=1)
    w.add_box_container(*TANK)
    w.add_particles(pos, vel)
    counts = []
    for _ in range(steps):
        r = w.step(dt)
        assert r.substeps == 1
        counts += list(w.last_iterations())
    d = np.random.default_rng(7).normal(size=vel.shape)
    free = oracle_lib.tangent_run(s, TANK, pos, vel, np.zeros_like(d), d, steps=steps, dt=dt)
    held = oracle_lib.tangent_run(s, TANK, pos, vel, np.zeros_like(d), d, steps=steps, dt=dt, forced_iterations=counts)
    for a, b in zip(free, held):
        assert np.array_equal(a, b)
    more = oracle_lib.tangent_run(s, TANK, pos, vel, np.zeros_like(d), d, steps=steps, dt=dt,
                                  forced_iterations=[c + 1 for c in counts])
    assert not np.array_equal(more[0], free[0])


@pytest.mark.parametrize("solver", [FluidSolver.WCSPH, FluidSolver.DFSPH])
def test_fp32_tangent_values_are_the_float_restatements_bit_for_bit(oracle_lib, solver):
    # precision 32: every value operation is the float restatement's, so the run is the FP32
    # program the CUDA library runs (and takes its branches); its derivative, in double, is close
    # to the FP64 method's on this short run
    s, steps, dt, pos, vel = case(solver)
    d = np.random.default_rng(7).normal(size=vel.shape)
    P, V, dP, dV, ids = oracle_lib.tangent_run(s, TANK, pos, vel, np.zeros_like(d), d, steps=steps, dt=dt,
                                               precision=32)
    w = oracle_lib.OracleWorld(s, precision=32, residual_sum=1)
    w.add_box_container(*TANK)
    w.add_particles(pos, vel)
    for _ in range(steps):
        w.step(dt)
    order = np.argsort(w.ids())
    assert np.array_equal(P.astype(np.float32), np.asarray(w.positions(), dtype=np.float32)[order])
    assert np.array_equal(V.astype(np.float32), np.asarray(w.velocities(), dtype=np.float32)[order])
    _, _, dP64, _, _ = oracle_lib.tangent_run(s, TANK, pos, vel, np.zeros_like(d), d, steps=steps, dt=dt)
    assert np.linalg.norm(dP - dP64) <= 1e-3 * np.linalg.norm(dP64)


def test_float_derivatives_stay_near_the_exact_ones_on_a_short_run(oracle_lib):
    # precision -32: the float restatement's values, each derivative operation rounded to float
    # (tests/tangent_conditioning.py measures the same on the 1M dam)
    s, steps, dt, pos, vel = case(FluidSolver.DFSPH)
    d = np.random.default_rng(11).normal(size=vel.shape)
    zero = np.zeros_like(d)
    P32, V32, dP32, dV32, _ = oracle_lib.tangent_run(s, TANK, pos, vel, zero, d, steps=steps, dt=dt, precision=32)
    Pf, Vf, dPf, dVf, _ = oracle_lib.tangent_run(s, TANK, pos, vel, zero, d, steps=steps, dt=dt, precision=-32)
    assert np.array_equal(P32, Pf) and np.array_equal(V32, Vf)
    assert np.linalg.norm(dVf - dV32) <= 1e-5 * np.linalg.norm(dV32)
    assert np.linalg.norm(dPf - dP32) <= 1e-5 * np.linalg.norm(dP32)
