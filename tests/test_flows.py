"""Emitters and drains (src/fluid/flow.rs), against both implementations.

The reference's flow tests (flow.rs:243-337), restated with its thresholds, run on the CPU
restatement and, marked `gpu`, on the CUDA library; a river run then checks that the library's
emitted and drained particles, ids, positions and velocities are the restatement's bit for bit.
"""
import numpy as np
import pytest

from solunar_b200.abi import Arithmetic, FluidSettings, FluidSolver, PhysicsError

TICK = np.float32(1.0 / 60.0)


@pytest.fixture(params=["oracle", pytest.param("gpu", marks=pytest.mark.gpu)])
def backend(request):
    """A factory of worlds: the CPU restatement, or the CUDA library."""
    if request.param == "oracle":
        from oracle import py_oracle

        py_oracle.build()
        return lambda **kw: py_oracle.OracleWorld(FluidSettings(**kw))
    gpu = request.getfixturevalue("gpu_lib")
    return lambda **kw: gpu.FluidWorld(FluidSettings(**kw))


def channel(make, **kw):
    # flow.rs:235-241
    w = make(**kw)
    w.add_box_container((0.0, 0.0, 0.0), (2.0, 0.6, 0.3))
    return w


def test_an_emitter_fills_its_box_once_and_tops_it_up(backend):
    # flow.rs:243-257
    w = channel(backend)
    w.add_emitter((0.0, 0.0, 0.0), (0.2, 0.3, 0.3), (0.0, 0.0, 0.0))
    r = w.step(TICK)
    assert r.emitted == 4 * 6 * 6
    assert w.len() == 4 * 6 * 6
    total = r.emitted
    for _ in range(30):
        total += w.step(TICK).emitted
    assert w.len() == total
    assert total > 4 * 6 * 6


def test_a_river_from_an_emitter_to_a_drain_keeps_its_count_and_books(backend):
    # flow.rs:259-287
    w = channel(backend)
    w.add_emitter((0.0, 0.0, 0.0), (0.15, 0.3, 0.3), (1.0, 0.0, 0.0))
    w.add_drain((1.8, 0.0, 0.0), (2.0, 0.6, 0.3))
    emitted = drained = 0
    counts = []
    for _ in range(240):
        r = w.step(TICK)
        emitted += r.emitted
        drained += r.drained
        assert r.held_back == 0
        counts.append(w.len())
    assert w.len() == emitted - drained
    assert drained > 0, "water reached the drain"
    late = counts[180:]
    spread = (max(late) - min(late)) / max(late)
    assert spread < 0.15, (min(late), max(late))
    assert np.all(w.positions()[:, 0] < 1.8 + 0.1)


def test_an_emitter_never_puts_water_on_top_of_water(backend):
    # flow.rs:289-307: a particle a little past the first slot's edge.  The reference calls
    # run_flows directly; here a step of 1e-6 s runs it after a substep that moves nothing
    # measurable.
    w = channel(backend)
    s = FluidSettings().spacing
    w.add_particle((s * 1.05, s * 0.5, s * 0.5), (0.0, 0.0, 0.0))
    w.add_emitter((0.0, 0.0, 0.0), (0.1, 0.05, 0.05), (0.0, 0.0, 0.0))
    w.step(1e-6)
    p = w.positions().astype(np.float64)
    d = np.linalg.norm(p[:, None, :] - p[None, :, :], axis=2)
    d[np.diag_indices(len(p))] = np.inf
    assert np.all(d > 0.5 * s)


def test_flows_refuse_bad_boxes_and_go_away(backend):
    # flow.rs:309-320
    w = channel(backend)
    with pytest.raises(PhysicsError):
        w.add_drain((1.0, 1.0, 1.0), (0.0, 0.0, 0.0))
    with pytest.raises(PhysicsError):
        w.add_emitter((0.0, 0.0, 0.0), (1.0, 1.0, 1.0), (float("nan"), 0.0, 0.0))
    with pytest.raises(PhysicsError):
        w.add_drain((float("nan"), 0.0, 0.0), (1.0, 1.0, 1.0))
    drain = w.add_drain((0.0, 0.0, 0.0), (1.0, 1.0, 1.0))
    assert w.remove_flow(drain)
    assert not w.remove_flow(drain)


def test_a_full_world_stops_the_emitter_with_an_error(backend):
    # flow.rs:322-337
    w = backend(max_particles=10)
    w.add_emitter((0.0, 0.0, 0.0), (0.2, 0.2, 0.2), (0.0, 0.0, 0.0))
    with pytest.raises(PhysicsError) as e:
        w.step(TICK)
    assert e.value.kind == "FluidFull"
    assert w.len() == 10


def by_id(w):
    order = np.argsort(w.ids())
    return w.ids()[order], w.positions()[order], w.velocities()[order]


@pytest.mark.gpu
@pytest.mark.parametrize("solver", [FluidSolver.WCSPH, FluidSolver.DFSPH])
def test_a_river_matches_the_restatement_bit_for_bit(gpu_lib, oracle_lib, solver):
    # EXACT arithmetic: what the emitter adds and the drain takes, and the water between them,
    # equal the float restatement's after every tick
    s = FluidSettings(solver=solver, arithmetic=Arithmetic.EXACT)
    g, o = gpu_lib.FluidWorld(s), oracle_lib.OracleWorld(s, residual_sum=1)
    for w in (g, o):
        w.add_box_container((0.0, 0.0, 0.0), (2.0, 0.6, 0.3))
        w.add_emitter((0.0, 0.0, 0.0), (0.15, 0.3, 0.3), (1.0, 0.0, 0.0))
        w.add_drain((0.9, 0.0, 0.0), (2.0, 0.6, 0.3))
    for tick in range(40):
        a, b = g.step(TICK), o.step(TICK)
        assert (a.emitted, a.drained, a.substeps) == (b.emitted, b.drained, b.substeps), tick
    ig, pg, vg = by_id(g)
    io, po, vo = by_id(o)
    assert np.array_equal(ig, io)
    assert np.array_equal(pg, po.astype(np.float32)) and np.array_equal(vg, vo.astype(np.float32))
    assert g.state_hash() == o.state_hash()
