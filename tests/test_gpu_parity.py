"""Parity of the CUDA library with the CPU restatement, through the C ABI.

EXACT arithmetic is the default: kernels round every operation as the reference's scalar f32
code does, and sum each particle's neighbours in the reference's list order, so cell order,
neighbour lists, densities, velocities and positions must agree bit for bit with the float
restatement (`residual_sum=1`: the DFSPH stop test on the same compensated FP64 sum of the
solver error that the library takes).
"""
import numpy as np
import pytest

from solunar_b200 import scenes
from solunar_b200.abi import FluidSettings, FluidSolver, PhysicsError

pytestmark = pytest.mark.gpu


def bits(a):
    return np.ascontiguousarray(np.asarray(a, dtype=np.float32)).view(np.uint32)


def assert_same_particles(g, o):
    assert g.len() == o.len()
    assert np.array_equal(g.ids(), o.ids())
    assert np.array_equal(bits(g.positions()), bits(o.positions()))
    assert np.array_equal(bits(g.velocities()), bits(o.velocities()))
    assert g.state_hash() == o.state_hash()


def assert_same_lists(g, o):
    gs, gi = g.neighbor_lists()
    os_, oi = o.neighbor_lists()
    assert np.array_equal(gs, os_)
    assert np.array_equal(gi, oi)
    gs, gi = g.wall_neighbor_lists()
    os_, oi = o.wall_neighbor_lists()
    assert np.array_equal(gs, os_)
    assert np.array_equal(gi, oi)


def both(gpu_lib, oracle_lib, settings, residual_sum=1):
    return gpu_lib.FluidWorld(settings), oracle_lib.OracleWorld(settings, residual_sum=residual_sum)


def assert_same_report(a, b):
    assert (a.substeps, a.capped, a.held_back, a.iterations, a.lost) == (
        b.substeps, b.capped, b.held_back, b.iterations, b.lost)
    assert bits(a.max_speed) == bits(b.max_speed)
    assert bits(a.max_compression) == bits(b.max_compression)


@pytest.mark.parametrize("count", [1, 100, 3000])
def test_sort_lists_and_densities_of_a_shaken_lattice(gpu_lib, oracle_lib, count):
    g, o = both(gpu_lib, oracle_lib, FluidSettings())
    pts = scenes.shaken(count)
    g.add_particles(pts)
    o.add_particles(pts)
    for w in (g, o):
        w.update_neighbors()
        w.compute_densities()
    assert_same_particles(g, o)
    assert_same_lists(g, o)
    assert np.array_equal(bits(g.densities()), bits(o.densities()))


@pytest.mark.parametrize("support", [1.5, 2.0, 3.3, 4.0])
def test_walls_lists_and_densities_in_a_tank(gpu_lib, oracle_lib, support):
    sc = scenes.small_dam(support=support, counts=(9, 11, 5))
    g, o = both(gpu_lib, oracle_lib, sc.settings)
    sc.build(g)
    sc.build(o)
    assert np.array_equal(bits(g.wall_positions()), bits(o.wall_positions()))
    for w in (g, o):
        w.update_neighbors()
        w.compute_densities()
    assert_same_particles(g, o)
    assert_same_lists(g, o)
    assert np.array_equal(bits(g.densities()), bits(o.densities()))


def test_an_empty_world_steps(gpu_lib, oracle_lib):
    g, o = both(gpu_lib, oracle_lib, FluidSettings())
    assert_same_report(g.step(1 / 60), o.step(1 / 60))
    g.update_neighbors()
    assert g.len() == 0


@pytest.mark.parametrize("support", [2.0, 4.0])
def test_wcsph_ticks_match_bit_for_bit(gpu_lib, oracle_lib, support):
    sc = scenes.small_dam(FluidSolver.WCSPH, support=support, counts=(10, 12, 6))
    g, o = both(gpu_lib, oracle_lib, sc.settings)
    sc.build(g)
    sc.build(o)
    for _ in range(8):
        assert_same_report(g.step(sc.dt), o.step(sc.dt))
    assert_same_particles(g, o)
    assert np.array_equal(bits(g.densities()), bits(o.densities()))
    assert_same_lists(g, o)


def test_dfsph_ticks_match_bit_for_bit(gpu_lib, oracle_lib):
    sc = scenes.small_dam(FluidSolver.DFSPH, counts=(10, 12, 6))
    g, o = both(gpu_lib, oracle_lib, sc.settings)
    sc.build(g)
    sc.build(o)
    for _ in range(6):
        assert_same_report(g.step(sc.dt), o.step(sc.dt))
        assert g.last_iterations() == o.last_iterations()
    assert_same_particles(g, o)
    assert np.array_equal(bits(g.densities()), bits(o.densities()))


def test_the_wcsph_dam_of_8000_particles_matches_for_its_1000_steps(gpu_lib, oracle_lib):
    # the 20^3 WCSPH dam at 0.02 m, support 4 (~250 neighbours), dt 2e-4, 1000 steps: reports
    # every step, particles and densities every 100, and at the end the cell order and the
    # neighbour sets of the final state
    sc = scenes.wcsph_dam_8k()
    g, o = both(gpu_lib, oracle_lib, sc.settings)
    sc.build(g)
    sc.build(o)
    for k in range(sc.steps):
        assert_same_report(g.step(sc.dt), o.step(sc.dt))
        if k % 100 == 99:
            assert_same_particles(g, o)
            assert np.array_equal(bits(g.densities()), bits(o.densities()))
    for w in (g, o):
        w.update_neighbors()
    assert_same_particles(g, o)
    assert_same_lists(g, o)


def test_a_domain_takes_out_what_leaves_it(gpu_lib, oracle_lib):
    sc = scenes.small_dam(FluidSolver.WCSPH, counts=(10, 12, 6))
    g, o = both(gpu_lib, oracle_lib, sc.settings)
    for w in (g, o):
        sc.build(w)
        w.set_domain(((0.0, 0.0, 0.0), (0.15, 1.0, 1.0)))
    lost = 0
    for _ in range(6):
        a, b = g.step(sc.dt), o.step(sc.dt)
        assert_same_report(a, b)
        lost += a.lost
    assert lost > 0
    assert_same_particles(g, o)


def test_a_skipped_job_is_reported_and_changes_nothing(gpu_lib):
    # the GPU counterpart of SkipsJobs (src/dispatch.rs:50-65, src/fluid/mod.rs:965-971)
    w = gpu_lib.FluidWorld(FluidSettings())
    w.fill_box((0, 0, 0), (0.6, 0.6, 0.6))
    before = (w.ids().copy(), w.positions().copy())
    w.debug_skip_job(0)
    with pytest.raises(PhysicsError) as e:
        w.update_neighbors()
    assert e.value.kind == "DispatchIncomplete"
    assert np.array_equal(w.ids(), before[0]) and np.array_equal(w.positions(), before[1])
    with pytest.raises(PhysicsError) as e:
        w.compute_densities()
    assert e.value.kind == "OutOfRange"
    w.update_neighbors()
    w.compute_densities()


def test_repeated_runs_give_the_same_bits(gpu_lib):
    # the determinism the reference pins across thread counts (src/fluid/step.rs:534-550)
    def run(solver):
        sc = scenes.small_dam(solver, counts=(8, 10, 5))
        w = gpu_lib.FluidWorld(sc.settings)
        sc.build(w)
        for _ in range(5):
            w.step(sc.dt)
        return w.state_hash()

    for solver in (FluidSolver.WCSPH, FluidSolver.DFSPH):
        assert run(solver) == run(solver)


def test_particles_added_between_steps_join_the_next_one(gpu_lib, oracle_lib):
    sc = scenes.small_dam(FluidSolver.WCSPH, counts=(6, 8, 4))
    g, o = both(gpu_lib, oracle_lib, sc.settings)
    for w in (g, o):
        sc.build(w)
        w.step(sc.dt)
        w.add_particle((0.3, 0.3, 0.1), (0.5, 0.0, 0.0))
        w.fill_box((0.4, 0.1, 0.02), (0.48, 0.2, 0.1))
    for _ in range(3):
        assert_same_report(g.step(sc.dt), o.step(sc.dt))
    assert_same_particles(g, o)
