"""FAST arithmetic (SLF_ARITHMETIC_FAST) against the CPU restatement and the FP64 oracle.

FAST keeps the reference's cells, neighbour sets, list order and sums, and changes only the
rounding (fused multiply-adds, a reciprocal square root per pair).  Stated tolerances:
  * cell order and neighbour lists: identical (bit for bit);
  * densities of one pass: relative 2e-6 of the float restatement's;
  * six ticks of a dam break: positions within 1e-4 m (1/200 of the spacing), densities within
    1e-4 of rest density, DFSPH iteration counts within 2 a tick;
  * density error against the FP64 restatement of the same run: at most 0.1 % of rest density.
"""
import numpy as np
import pytest

from solunar_b200 import scenes
from solunar_b200.abi import Arithmetic, FluidSolver

pytestmark = pytest.mark.gpu


def by_id(w, arr):
    return arr[np.argsort(w.ids())]


def fast_scene(solver, support=2.0):
    sc = scenes.small_dam(solver, counts=(10, 12, 6), support=support)
    sc.settings.arithmetic = Arithmetic.FAST
    return sc


@pytest.mark.parametrize("solver", [FluidSolver.WCSPH, FluidSolver.DFSPH])
@pytest.mark.parametrize("support", [2.0, 4.0])
def test_fast_lists_are_exact_and_densities_within_tolerance(gpu_lib, oracle_lib, solver, support):
    sc = fast_scene(solver, support)
    g, o = gpu_lib.FluidWorld(sc.settings), oracle_lib.OracleWorld(sc.settings, residual_sum=1)
    for w in (g, o):
        sc.build(w)
        w.update_neighbors()
        w.compute_densities()
    assert np.array_equal(g.ids(), o.ids())
    gs, gi = g.neighbor_lists()
    os_, oi = o.neighbor_lists()
    assert np.array_equal(gs, os_) and np.array_equal(gi, oi)
    np.testing.assert_allclose(g.densities(), o.densities(), rtol=2e-6)


@pytest.mark.parametrize("solver", [FluidSolver.WCSPH, FluidSolver.DFSPH])
def test_fast_ticks_track_the_restatement(gpu_lib, oracle_lib, solver):
    sc = fast_scene(solver)
    g, o = gpu_lib.FluidWorld(sc.settings), oracle_lib.OracleWorld(sc.settings, residual_sum=1)
    for w in (g, o):
        sc.build(w)
    for _ in range(6):
        a, b = g.step(sc.dt), o.step(sc.dt)
        assert a.substeps == b.substeps
        assert abs(a.iterations - b.iterations) <= 2
    assert np.max(np.abs(by_id(g, g.positions()) - by_id(o, o.positions()))) < 1e-4
    assert np.max(np.abs(by_id(g, g.densities()) - by_id(o, o.densities()))) / 1000.0 < 1e-4


@pytest.mark.parametrize("arithmetic", [Arithmetic.EXACT, Arithmetic.FAST])
@pytest.mark.parametrize("solver", [FluidSolver.WCSPH, FluidSolver.DFSPH])
def test_density_error_against_the_fp64_oracle_is_under_a_tenth_of_a_percent(gpu_lib, oracle_lib, solver,
                                                                             arithmetic):
    sc = scenes.small_dam(solver, counts=(10, 12, 6))
    sc.settings.arithmetic = arithmetic
    g, d = gpu_lib.FluidWorld(sc.settings), oracle_lib.OracleWorld(sc.settings, precision=64, residual_sum=1)
    for w in (g, d):
        sc.build(w)
    for _ in range(8):
        g.step(sc.dt)
        d.step(sc.dt)
    err = np.abs(by_id(g, g.densities()) - by_id(d, d.densities())) / 1000.0
    assert np.max(err) < 1e-3, np.max(err)
