"""Cell-relative positions (SLF_POSITIONS_CELL_RELATIVE) against the CPU restatements.

Each position is held as an f32 offset from its cell's corner plus an integer cell, so a pair's
offset is formed from small numbers; arithmetic is FAST.  Stated tolerances:
  * near the origin it tracks the float restatement as FAST does: positions within 1e-4 m after
    six ticks, densities within 1e-4 of rest density, DFSPH iterations within 2 a tick;
  * neighbour sets equal the restatement's except for pairs whose distance is within 1e-5 of
    the kernel radius (the two round the distance differently);
  * far from the origin (1024 m, where an f32 coordinate resolves 1.2e-4 m) its densities stay
    within 0.1 % of rest density of the FP64 restatement and its positions within 2e-4 m,
    while absolute f32 positions there cannot follow slow motion at all.
"""
import numpy as np
import pytest

from solunar_b200 import scenes
from solunar_b200.abi import Arithmetic, FluidSolver, Positions, PhysicsError

pytestmark = pytest.mark.gpu


def by_id(w, arr):
    return arr[np.argsort(w.ids())]


def rel(sc):
    sc.settings.arithmetic = Arithmetic.FAST
    sc.settings.positions = Positions.CELL_RELATIVE
    return sc


def test_positions_round_trip_and_match_the_absolute_world(gpu_lib):
    sc = rel(scenes.small_dam(FluidSolver.DFSPH))
    g = gpu_lib.FluidWorld(sc.settings)
    pos, vel = sc.build(g)
    assert np.array_equal(g.positions(), pos)
    assert np.array_equal(g.velocities(), vel)
    a = scenes.small_dam(FluidSolver.DFSPH)
    a.settings.arithmetic = Arithmetic.FAST
    w = gpu_lib.FluidWorld(a.settings)
    a.build(w)
    assert g.state_hash() == w.state_hash()
    moved = (pos + np.float32(0.003)).astype(np.float32)
    g.write_state(moved, vel)
    assert np.array_equal(g.positions(), moved)


def test_cell_relative_needs_fast_arithmetic(gpu_lib):
    sc = scenes.small_dam(FluidSolver.DFSPH)
    sc.settings.positions = Positions.CELL_RELATIVE
    with pytest.raises(PhysicsError):
        gpu_lib.FluidWorld(sc.settings)


@pytest.mark.parametrize("solver", [FluidSolver.WCSPH, FluidSolver.DFSPH])
def test_neighbour_sets_match_up_to_the_radius_rounding(gpu_lib, oracle_lib, solver):
    sc = rel(scenes.small_dam(solver))
    g, o = gpu_lib.FluidWorld(sc.settings), oracle_lib.OracleWorld(sc.settings, residual_sum=1)
    for w in (g, o):
        sc.build(w)
        w.update_neighbors()
        w.compute_densities()
    assert np.array_equal(g.ids(), o.ids())
    gs, gi = g.neighbor_lists()
    os_, oi = o.neighbor_lists()
    p = o.positions().astype(np.float64)
    r = float(o.kernel()[0])
    for i in range(len(p)):
        a, b = set(gi[gs[i]:gs[i + 1]].tolist()), set(oi[os_[i]:os_[i + 1]].tolist())
        for j in a ^ b:
            d = np.linalg.norm(p[i] - p[j])
            assert abs(d - r) < 1e-5 * r, (i, j, d, r)
    np.testing.assert_allclose(g.densities(), o.densities(), rtol=2e-5)


@pytest.mark.parametrize("solver", [FluidSolver.WCSPH, FluidSolver.DFSPH])
def test_cell_relative_ticks_track_the_restatement(gpu_lib, oracle_lib, solver):
    sc = rel(scenes.small_dam(solver))
    g, o = gpu_lib.FluidWorld(sc.settings), oracle_lib.OracleWorld(sc.settings, residual_sum=1)
    for w in (g, o):
        sc.build(w)
    for _ in range(6):
        a, b = g.step(sc.dt), o.step(sc.dt)
        assert a.substeps == b.substeps
        assert abs(a.iterations - b.iterations) <= 2
    assert np.max(np.abs(by_id(g, g.positions()) - by_id(o, o.positions()))) < 1e-4
    assert np.max(np.abs(by_id(g, g.densities()) - by_id(o, o.densities()))) / 1000.0 < 1e-4


def test_domain_keeps_cell_relative_particles_inside(gpu_lib, oracle_lib):
    sc = rel(scenes.small_dam(FluidSolver.WCSPH))
    g, o = gpu_lib.FluidWorld(sc.settings), oracle_lib.OracleWorld(sc.settings, residual_sum=1)
    for w in (g, o):
        sc.build(w)
        w.set_domain(((0.0, 0.0, 0.0), (0.6, 0.1, 0.2)))
    a, b = g.step(sc.dt), o.step(sc.dt)
    assert a.lost == b.lost > 0
    assert np.array_equal(np.sort(g.ids()), np.sort(o.ids()))


def far_run(world, sc, steps):
    sc.build(world)
    for _ in range(steps):
        world.step(sc.dt)
    return by_id(world, world.positions()).astype(np.float64), by_id(world, world.densities())


def test_far_from_the_origin_cell_relative_keeps_fp64_accuracy(gpu_lib, oracle_lib):
    steps = 40
    sc = scenes.dfsph_precision_far(counts=(10, 12, 6))
    d = oracle_lib.OracleWorld(sc.settings, precision=64, residual_sum=1)
    pd, rd = far_run(d, sc, steps)
    sc_rel = rel(scenes.dfsph_precision_far(counts=(10, 12, 6)))
    pr, rr = far_run(gpu_lib.FluidWorld(sc_rel.settings), sc_rel, steps)
    sc_abs = scenes.dfsph_precision_far(counts=(10, 12, 6))
    sc_abs.settings.arithmetic = Arithmetic.FAST
    pa, ra = far_run(gpu_lib.FluidWorld(sc_abs.settings), sc_abs, steps)
    rel_pos = np.max(np.abs(pr - pd))
    abs_pos = np.max(np.abs(pa - pd))
    assert rel_pos < 2e-4, rel_pos
    assert np.max(np.abs(rr - rd)) / 1000.0 < 1e-3
    # 40 ms at 0.05 m/s is 2 mm of motion, most of which absolute f32 at 1024 m cannot represent
    assert abs_pos > 5 * rel_pos, (abs_pos, rel_pos)
