"""The reference's own fluid tests, restated against both implementations.

The reference stores no golden vectors for this path apart from the Martin & Moyce front table
its dam-break test embeds (tests/golden/martin_moyce.json); its tests are properties.  Each test
here restates one of them (src/fluid/mod.rs:742-973, src/fluid/step.rs:342-584) with the
reference's thresholds.  Tests that take `backend` run against the CPU restatement (pinning the
oracle) and, marked `gpu`, against the CUDA library; the rest probe parts only the restatement
exposes (kernel samples, the cell table, thread counts).
"""
import json
import math
import os

import numpy as np
import pytest

from solunar_b200.abi import FluidSettings, FluidSolver, PhysicsError
from solunar_b200 import scenes


TICK = np.float32(1.0 / 60.0)


def world(oracle_lib, **kw):
    return oracle_lib.OracleWorld(FluidSettings(**kw))


def shaken_world(oracle_lib, count, **kw):
    w = world(oracle_lib, **kw)
    w.add_particles(scenes.shaken(count))
    return w


@pytest.fixture(params=["oracle", pytest.param("gpu", marks=pytest.mark.gpu)])
def backend(request):
    """A factory of worlds: the CPU restatement, or the CUDA library."""
    if request.param == "oracle":
        from oracle import py_oracle

        py_oracle.build()
        return lambda **kw: py_oracle.OracleWorld(FluidSettings(**kw))
    gpu = request.getfixturevalue("gpu_lib")
    return lambda **kw: gpu.FluidWorld(FluidSettings(**kw))


def test_kernel_holds_unit_mass_and_its_slope_matches(oracle_lib):
    # src/fluid/mod.rs:776-801
    steps = 4000
    dr = np.float32(0.1) / np.float32(steps)
    rs = (np.arange(steps, dtype=np.float32) + np.float32(0.5)) * dr
    offsets = np.stack([rs, np.zeros_like(rs), np.zeros_like(rs)], axis=1)
    value, _, _ = oracle_lib.kernel_eval(0.1, offsets)
    total = np.float32(0.0)
    four_pi = np.float32(4.0) * np.float32(math.pi)
    for r, v in zip(rs, value):
        total = np.float32(total + np.float32(np.float32(np.float32(np.float32(four_pi * r) * r) * v) * dr))
    assert abs(float(total) - 1.0) < 1e-3
    v, _, _ = oracle_lib.kernel_eval(0.1, [[0.1, 0, 0], [0.5, 0, 0]])
    assert v[0] == 0.0 and v[1] == 0.0
    for r in [0.01, 0.03, 0.05, 0.08, 0.099]:
        h = np.float32(1e-4)
        vals, slopes, _ = oracle_lib.kernel_eval(0.1, [[r + h, 0, 0], [r - h, 0, 0], [r, 0, 0]])
        numeric = (float(vals[0]) - float(vals[1])) / (2 * float(h))
        slope = float(slopes[2])
        assert abs(numeric - slope) < 1e-2 * max(abs(slope), 1.0), r
        assert slope <= 0.0
    _, _, g = oracle_lib.kernel_eval(0.1, [[0.03, 0, 0], [0, 0, 0]])
    assert g[0, 0] < 0.0 and g[0, 1] == 0.0
    assert np.all(g[1] == 0.0)


def test_the_dense_table_and_the_search_find_the_same_cells(oracle_lib):
    # src/fluid/mod.rs:803-828
    keys = sorted([(-3, 0, 2), (-3, 0, 2), (-1, 4, 0), (0, 0, 0), (5, -2, 1)])
    queries = [(x, y, z) for x in range(-5, 7) for y in range(-4, 6) for z in range(-2, 4)]
    dense, had_dense = oracle_lib.grid_ranges(keys, queries, force_search=False)
    search, _ = oracle_lib.grid_ranges(keys, queries, force_search=True)
    assert had_dense
    assert np.array_equal(dense, search)
    far, had_dense = oracle_lib.grid_ranges([(-100_000, 0, 0), (100_000, 0, 0)],
                                            [(100_000, 0, 0), (2**31 - 1, -2**31, 0)], force_search=False)
    assert not had_dense
    assert tuple(far[0]) == (1, 2)
    assert tuple(far[1]) == (0xFFFFFFFF, 0xFFFFFFFF)


def brute_force_sets(pos32: np.ndarray, reach: np.float32):
    out = []
    for i in range(len(pos32)):
        d = pos32 - pos32[i]
        l2 = (d[:, 0] * d[:, 0] + d[:, 1] * d[:, 1]) + d[:, 2] * d[:, 2]
        out.append(np.nonzero(l2 < reach)[0])
    return out


def test_neighbors_are_exactly_the_brute_force_ones(backend):
    # src/fluid/mod.rs:830-845
    w = backend()
    w.add_particles(scenes.shaken(900))
    w.update_neighbors()
    pos = w.positions().astype(np.float32)
    r = np.float32(w.settings().radius())
    brute = brute_force_sets(pos, np.float32(r * r))
    start, items = w.neighbor_lists()
    for i in range(len(pos)):
        found = np.sort(items[start[i]:start[i + 1]])
        assert np.array_equal(found, brute[i]), i


def test_any_thread_count_gives_the_same_lists_densities_and_hash(oracle_lib):
    # src/fluid/mod.rs:847-864
    def run(threads):
        w = shaken_world(oracle_lib, 3000)
        w.set_threads(threads)
        w.update_neighbors()
        w.compute_densities()
        return (w.neighbor_lists()[1].tobytes(), w.densities().astype(np.float32).tobytes(),
                w.ids().tobytes(), w.state_hash())

    one = run(1)
    assert run(4) == one
    assert run(7) == one


def test_a_lattice_inside_is_at_rest_density(backend):
    # src/fluid/mod.rs:866-895
    w = backend()
    assert w.fill_box((0, 0, 0), (0.6, 0.6, 0.6)) == 12 ** 3
    w.update_neighbors()
    w.compute_densities()
    rest = 1000.0
    margin = w.settings().radius()
    checked = 0
    for at, d in zip(w.positions(), w.densities()):
        if all(margin < v < 0.6 - margin for v in at):
            assert abs(d - rest) / rest < 1e-4
            checked += 1
        else:
            assert d <= rest * (1 + 1e-4)
    assert checked > 100
    cell = rest * 0.05 ** 3
    assert abs(w.particle_mass() / cell - 1.0) < 0.1


def test_ids_follow_particles_through_the_sort(backend):
    # src/fluid/mod.rs:897-913
    w = backend()
    w.add_particles(scenes.shaken(700))
    before = dict(zip(w.ids().tolist(), w.positions().tolist()))
    h = w.state_hash()
    w.update_neighbors()
    for i, at in zip(w.ids().tolist(), w.positions().tolist()):
        assert before[i] == at
    assert w.state_hash() == h


def test_bad_input_is_refused_and_changes_nothing(backend):
    # src/fluid/mod.rs:915-972 (the dispatcher case has no CPU-restatement counterpart; the
    # CUDA library's fault-injection test covers DispatchIncomplete)
    for kw in [dict(spacing=0.0), dict(rest_density=float("nan")), dict(support=9.0), dict(max_particles=0)]:
        with pytest.raises(PhysicsError) as e:
            backend(**kw)
        assert e.value.kind == "InvalidSettings"
    w = backend(max_particles=100)
    nan = (float("nan"), 0.0, 0.0)
    with pytest.raises(PhysicsError):
        w.add_particle(nan, (0, 0, 0))
    with pytest.raises(PhysicsError):
        w.add_particle((0, 0, 0), nan)
    with pytest.raises(PhysicsError):
        w.fill_box((1, 1, 1), (0, 0, 0))
    with pytest.raises(PhysicsError):
        w.fill_box((0, 0, 0), nan)
    with pytest.raises(PhysicsError) as e:
        w.fill_box((0, 0, 0), (1, 1, 1))
    assert e.value.kind == "FluidFull"
    with pytest.raises(PhysicsError) as e:
        w.fill_box((0, 0, 0), (1e30, 1e30, 1e30))
    assert e.value.kind == "FluidFull"
    assert w.len() == 0
    assert w.fill_box((0, 0, 0), (0.2, 0.2, 0.2)) == 64
    with pytest.raises(PhysicsError) as e:
        w.compute_densities()
    assert e.value.kind == "OutOfRange"


# ---- step.rs tests ---------------------------------------------------------------------------

def tank(make, water, size, solver=FluidSolver.WCSPH, **kw):
    w = make(solver=solver, **kw)
    w.add_box_container((0, 0, 0), size)
    w.fill_box((0, 0, 0), water)
    return w


def inside(w, size):
    p = w.positions()
    return bool(np.all(p >= 0) and np.all(p <= np.asarray(size)))


def test_still_water_stays_still_and_presses_by_its_depth(backend):
    # src/fluid/step.rs:377-411
    size = (0.5, 0.6, 0.5)
    depth = 0.4
    w = tank(backend, (0.5, depth, 0.5), size)
    count = w.len()
    held = 0
    last = None
    for _ in range(180):
        last = w.step(TICK)
        held += last.held_back
        assert not last.capped
    assert w.len() == count
    assert inside(w, size)
    assert held == 0
    mean = float(np.mean(np.linalg.norm(w.velocities(), axis=1)))
    assert last.max_speed < 0.2 and mean < 0.03, (last, mean)
    stiffness = 1000.0 * 20.0 ** 2 / 7.0
    bottom = 1000.0 * 9.81 * depth
    expected = (1.0 + bottom / stiffness) ** (1.0 / 7.0) - 1.0
    assert expected * 0.5 < last.max_compression < expected * 2.0
    top = float(np.max(w.positions()[:, 1]))
    assert abs(top - (depth - 0.025)) < 0.05


def test_a_column_collapses_but_never_outruns_the_ideal_front(backend):
    # src/fluid/step.rs:413-445
    size = (1.6, 0.6, 0.2)
    height = 0.4
    w = tank(backend, (0.4, height, 0.2), size)
    start = float(np.max(w.positions()[:, 0]))
    ideal = 2.0 * math.sqrt(9.81 * height)
    held = 0
    time = 0.0
    last = start
    for _ in range(24):
        held += w.step(TICK).held_back
        time += float(TICK)
        now = float(np.max(w.positions()[:, 0]))
        assert now - start <= ideal * time + 0.05
        assert now >= last - 0.01
        last = now
    assert last - start > 0.4
    assert inside(w, size)
    assert held == 0


def martin_moyce_table():
    """The digitised Martin & Moyce (1952) front table embedded in the reference's own test
    (src/fluid/step.rs:447-460), extracted into tests/golden/martin_moyce.json by
    tests/golden/make_martin_moyce.py."""
    with open(os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "martin_moyce.json")) as f:
        return [(float(a), float(b)) for a, b in json.load(f)["pairs"]]


@pytest.mark.slow
def test_the_dam_break_front_follows_martin_and_moyce(backend):
    # src/fluid/step.rs:462-507
    table = martin_moyce_table()
    assert len(table) == 10
    width = 0.3
    spacing = np.float32(0.3) / np.float32(18.0)
    w = backend(spacing=float(spacing))
    size = (3.2, 0.8, 0.1)
    w.add_box_container((0, 0, 0), size)
    w.fill_box((0, 0, 0), (width, 2 * width, 0.1))
    count = w.len()
    scale = math.sqrt(2 * 9.81 / width)
    tick = np.float32(1.0 / 240.0)
    time = np.float32(0.0)
    errors = []
    held = 0
    for when, measured in table:
        while float(time) * scale < when:
            held += w.step(tick).held_back
            time = np.float32(time + tick)
        edge = float(np.max(w.positions()[:, 0]))
        front = (edge + float(spacing) / 2) / width
        error = (front - measured) / measured
        assert -0.03 < error < 0.16, (when, front, measured)
        errors.append(error)
    assert sum(errors) / len(errors) < 0.10
    assert w.len() == count
    assert held == 0
    assert inside(w, size)


def test_a_gate_holds_until_it_is_taken_away(backend):
    # src/fluid/step.rs:509-532
    w = tank(backend, (0.4, 0.4, 0.2), (1.2, 0.6, 0.2))
    gate = w.add_wall((0.4, 0.0, 0.0), (0.5, 0.6, 0.2))
    for _ in range(30):
        w.step(TICK)
    assert float(np.max(w.positions()[:, 0])) < 0.45
    assert w.remove_boundary(gate)
    assert not w.remove_boundary(gate)
    for _ in range(20):
        w.step(TICK)
    assert float(np.max(w.positions()[:, 0])) > 0.7


@pytest.mark.parametrize("solver", [FluidSolver.WCSPH, FluidSolver.DFSPH])
def test_any_thread_count_ends_on_the_same_state(oracle_lib, solver):
    # src/fluid/step.rs:534-550
    def run(threads):
        w = tank(lambda **kw: world(oracle_lib, **kw), (0.3, 0.3, 0.2), (0.9, 0.5, 0.2), solver=solver)
        w.set_threads(threads)
        for _ in range(12):
            w.step(TICK)
        return w.state_hash()

    one = run(1)
    assert run(4) == one
    assert run(3) == one
    assert run(1) == one


def test_bad_steps_are_refused_and_a_cap_is_reported(backend):
    # src/fluid/step.rs:552-583
    w = tank(backend, (0.2, 0.2, 0.2), (0.3, 0.3, 0.3))
    with pytest.raises(PhysicsError):
        w.step(-1.0)
    with pytest.raises(PhysicsError):
        w.step(float("nan"))
    assert w.step(0.0).substeps == 0
    tight = backend(max_substeps=2)
    tight.fill_box((0, 0, 0), (0.1, 0.1, 0.1))
    r = tight.step(TICK)
    assert r.capped and r.substeps == 2
    for kw in [dict(sound_speed=0.0), dict(courant=1.5), dict(viscosity=-1.0)]:
        with pytest.raises(PhysicsError):
            backend(**kw)


def test_the_double_restatement_agrees_with_the_float_one_on_a_short_dam(oracle_lib):
    # the precision oracle runs the same method: a few steps of a small dam stay within f32 noise
    sc = scenes.small_dam(counts=(8, 10, 5))
    a = oracle_lib.OracleWorld(sc.settings, precision=32)
    b = oracle_lib.OracleWorld(sc.settings, precision=64)
    sc.build(a)
    sc.build(b)
    for _ in range(3):
        a.step(sc.dt)
        b.step(sc.dt)
    assert np.array_equal(a.ids(), b.ids())
    assert np.max(np.abs(a.positions() - b.positions())) < 1e-4
    assert np.max(np.abs(a.densities() - b.densities()) / 1000.0) < 1e-3


@pytest.mark.parametrize("counts", [(10, 12, 6), (14, 10, 8)])
def test_the_compensated_residual_stops_the_solves_where_the_reference_sum_does(oracle_lib, counts):
    # The CUDA library sums the DFSPH solver error in compensated FP64; the reference sums it in
    # f32, sequentially (src/fluid/dfsph.rs:266-267).  On these dams both stop every solve at
    # the same iteration, so the two runs stay bit-identical.
    sc = scenes.small_dam(FluidSolver.DFSPH, counts=counts)
    ref = oracle_lib.OracleWorld(sc.settings, residual_sum=0)
    comp = oracle_lib.OracleWorld(sc.settings, residual_sum=1)
    sc.build(ref)
    sc.build(comp)
    for _ in range(6):
        a, b = ref.step(sc.dt), comp.step(sc.dt)
        assert a.iterations == b.iterations
        assert ref.last_iterations() == comp.last_iterations()
    assert ref.state_hash() == comp.state_hash()


@pytest.mark.slow
@pytest.mark.parametrize("name", ["dfsph_dam_250k", "dfsph_dam_250k_c2"])
def test_the_compensated_residual_stops_where_the_reference_sum_does_at_250k(oracle_lib, name):
    # The same check on the 250,000-particle dams, solve by solve, through the steps where the
    # falling column drives the density solve to 10-15 iterations: the reference's f32 sum over
    # a quarter of a million errors and the compensated FP64 sum stop at the same iteration.
    # (tests/test_gpu_parity_at_scale.py makes the same comparison at one million particles.)
    sc = getattr(scenes, name)()
    ref = oracle_lib.OracleWorld(sc.settings, residual_sum=0)
    comp = oracle_lib.OracleWorld(sc.settings, residual_sum=1)
    sc.build(ref)
    sc.build(comp)
    counts = []
    for _ in range(12):
        ref.step(sc.dt)
        comp.step(sc.dt)
        assert ref.last_iterations() == comp.last_iterations()
        counts.append(comp.last_iterations()[1])
    assert ref.state_hash() == comp.state_hash()
    assert max(counts) >= 4
