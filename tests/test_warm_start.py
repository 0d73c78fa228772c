"""Warm-started DFSPH solves (the `warm_start` setting), against both implementations.

The reference cold-starts every solve (src/fluid/dfsph.rs:217-229); a warm start is this
library's opt-in setting, written the same way in the CUDA library and in the CPU restatement:
each solve starts with one push at half the stiffness impulse (sum of kappa dt) the particle's
solve of the same kind applied the substep before.  The reference's note is that a half-pressure
start sped a dam-break front up, so the dam tests here check the front against a cold start as
well as the iteration savings, and the density error against the FP64 restatement of the same
warm-started method.
"""
import numpy as np
import pytest

from solunar_b200 import scenes
from solunar_b200.abi import Arithmetic, FluidSettings, FluidSolver

TICK = np.float32(1.0 / 60.0)


@pytest.fixture(params=["oracle", pytest.param("gpu", marks=pytest.mark.gpu)])
def backend(request):
    """A factory of worlds: the CPU restatement, or the CUDA library."""
    if request.param == "oracle":
        from oracle import py_oracle

        py_oracle.build()
        return lambda s: py_oracle.OracleWorld(s, residual_sum=1)
    gpu = request.getfixturevalue("gpu_lib")
    return lambda s: gpu.FluidWorld(s)


def dam(make, warm, counts=(15, 30, 15), **kw):
    s = FluidSettings(solver=FluidSolver.DFSPH, spacing=0.02, support=2.0, warm_start=warm, **kw)
    sc = scenes.Scene("warm_dam", s, (2.0, 1.0, 1.0), counts, jitter=1e-5, dt=1e-3)
    w = make(s)
    sc.build(w)
    return w


def front(w):
    return float(np.percentile(np.asarray(w.positions(), dtype=np.float64)[:, 0], 99.5))


def test_the_first_warm_substep_is_a_cold_one(backend):
    # no impulse yet: the warm push moves nothing, bit for bit
    cold, warm = dam(backend, False), dam(backend, True)
    a, b = cold.step(1e-3), warm.step(1e-3)
    assert a.iterations == b.iterations
    assert cold.state_hash() == warm.state_hash()


def test_warm_start_leaves_wcsph_alone(backend):
    def run(warm):
        w = backend(FluidSettings(warm_start=warm))
        w.add_box_container((0.0, 0.0, 0.0), (0.5, 0.5, 0.3))
        w.fill_box((0.0, 0.0, 0.0), (0.2, 0.3, 0.3))
        for _ in range(5):
            w.step(TICK)
        return w.state_hash()

    assert run(True) == run(False)


@pytest.mark.slow
def test_a_warm_dam_break_takes_fewer_iterations_and_keeps_its_front(backend):
    cold, warm = dam(backend, False), dam(backend, True)
    its = {False: 0, True: 0}
    for k in range(300):
        its[False] += cold.step(1e-3).iterations
        its[True] += warm.step(1e-3).iterations
    # the solves start nearer their answer ...
    assert its[True] < 0.85 * its[False], its
    # ... and the front runs as a cold start's does (0.3 s in, it has moved about 0.5 m)
    assert abs(front(warm) - front(cold)) < 0.01, (front(warm), front(cold))
    assert front(cold) > 0.55


@pytest.mark.slow
def test_warm_f32_densities_stay_within_a_tenth_of_a_percent_of_fp64(oracle_lib):
    # the same warm-started method in f32 and in f64: the density error the precision makes
    def run(precision):
        w = dam(lambda s: oracle_lib.OracleWorld(s, precision=precision, residual_sum=1), True)
        for _ in range(100):
            w.step(1e-3)
        order = np.argsort(w.ids())
        return np.asarray(w.densities(), dtype=np.float64)[order]

    single, double = run(32), run(64)
    error = np.abs(single - double) / 1000.0
    assert error.mean() < 1e-3, error.mean()


def test_a_loaded_snapshot_starts_cold(backend):
    from oracle import py_oracle

    warm = dam(backend, True)
    for _ in range(3):
        warm.step(1e-3)
    s = FluidSettings(solver=FluidSolver.DFSPH, spacing=0.02, support=2.0, warm_start=True)
    saved = warm.save_snapshot()
    if isinstance(warm, py_oracle.OracleWorld):
        loaded = py_oracle.OracleWorld.load_snapshot(saved, s, residual_sum=1)
        cold = py_oracle.OracleWorld.load_snapshot(saved, FluidSettings(solver=FluidSolver.DFSPH), residual_sum=1)
    else:
        loaded = type(warm).load_snapshot(saved, s)
        cold = type(warm).load_snapshot(saved, FluidSettings(solver=FluidSolver.DFSPH))
    loaded.step(1e-3)
    cold.step(1e-3)
    assert loaded.state_hash() == cold.state_hash()


@pytest.mark.gpu
def test_a_warm_taped_forward_is_the_untaped_one(gpu_lib):
    # a tape records the impulses with the state (the adjoint is tests/test_gpu_adjoint_warm.py)
    taped = dam(lambda s: gpu_lib.FluidWorld(s), True, counts=(4, 4, 4))
    plain = dam(lambda s: gpu_lib.FluidWorld(s), True, counts=(4, 4, 4))
    for every in (0, 2):
        taped.tape_begin(every)
        for _ in range(3):
            taped.step(1e-3)
            plain.step(1e-3)
        taped.tape_end()
        assert taped.state_hash() == plain.state_hash()


@pytest.mark.gpu
def test_a_warm_river_matches_the_restatement_bit_for_bit(gpu_lib, oracle_lib):
    # EXACT arithmetic: the impulses ride through sorts, emissions, drains and the domain's
    # compaction exactly as the restatement's do
    s = FluidSettings(solver=FluidSolver.DFSPH, arithmetic=Arithmetic.EXACT, warm_start=True)
    g, o = gpu_lib.FluidWorld(s), oracle_lib.OracleWorld(s, residual_sum=1)
    for w in (g, o):
        w.add_box_container((0.0, 0.0, 0.0), (2.0, 0.6, 0.3))
        w.add_emitter((0.0, 0.0, 0.0), (0.15, 0.3, 0.3), (1.0, 0.0, 0.0))
        w.add_drain((0.9, 0.0, 0.0), (2.0, 0.6, 0.3))
        w.set_domain(((-1.0, -1.0, -1.0), (3.0, 0.25, 1.0)))
    for tick in range(40):
        a, b = g.step(TICK), o.step(TICK)
        assert (a.emitted, a.drained, a.lost, a.substeps, a.iterations) == (
            b.emitted, b.drained, b.lost, b.substeps, b.iterations), tick
    assert g.state_hash() == o.state_hash()
    np.testing.assert_array_equal(g.densities(), o.densities().astype(np.float32))


@pytest.mark.gpu
def test_a_warm_dam_matches_the_restatement_bit_for_bit(gpu_lib, oracle_lib):
    s = FluidSettings(solver=FluidSolver.DFSPH, spacing=0.02, support=2.0, arithmetic=Arithmetic.EXACT,
                      warm_start=True)
    g = dam(lambda _: gpu_lib.FluidWorld(s), True)
    o = dam(lambda _: oracle_lib.OracleWorld(s, residual_sum=1), True)
    for k in range(60):
        a, b = g.step(1e-3), o.step(1e-3)
        assert a.iterations == b.iterations, k
    assert g.state_hash() == o.state_hash()


@pytest.mark.gpu
def test_fast_warm_densities_stay_within_a_tenth_of_a_percent_of_fp64(gpu_lib, oracle_lib):
    s = FluidSettings(solver=FluidSolver.DFSPH, spacing=0.02, support=2.0, arithmetic=Arithmetic.FAST,
                      warm_start=True)
    g = dam(lambda _: gpu_lib.FluidWorld(s), True)
    o = dam(lambda _: oracle_lib.OracleWorld(s, precision=64, residual_sum=1), True)
    for _ in range(100):
        g.step(1e-3)
        o.step(1e-3)
    a = np.asarray(g.densities(), dtype=np.float64)[np.argsort(g.ids())]
    b = np.asarray(o.densities(), dtype=np.float64)[np.argsort(o.ids())]
    assert (np.abs(a - b) / 1000.0).mean() < 1e-3
