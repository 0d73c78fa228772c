"""DFSPH substeps and solves run as CUDA graphs against the same solves launched in host-checked
batches.

Mode 2 runs a whole substep as one graph launch (sort, density, both solves, viscosity, advance);
mode 1 runs each solve as one graph launch whose while node the stopping check ends on the
device; mode 0 queues the same kernels with a host check between batches.  All must give the
same state bit for bit, the same iteration counts, and (EXACT) the CPU restatement's state.
"""
import numpy as np
import pytest

from solunar_b200 import scenes
from solunar_b200.abi import Arithmetic, FluidSettings, FluidSolver, PhysicsError

TICK = np.float32(1.0 / 60.0)

pytestmark = pytest.mark.gpu


def pair(gpu_lib, settings, build, mode=2):
    worlds = []
    for m in (mode, 0):
        w = gpu_lib.FluidWorld(settings)
        w.solver_graphs(m)
        build(w)
        worlds.append(w)
    return worlds


def dam_build(counts=(12, 20, 12), spacing=0.02):
    """A jittered block in the corner of a 1 x 0.6 x 0.5 m tank."""
    def build(w):
        w.add_box_container((0.0, 0.0, 0.0), (1.0, 0.6, 0.5))
        pos = scenes.lattice_block((0.0, 0.0, 0.0), counts, spacing)
        pos = (pos + scenes.jitter(len(pos), 1e-5)).astype(np.float32)
        w.add_particles(pos, np.zeros_like(pos))
    return build


@pytest.mark.parametrize("mode", [1, 2])
@pytest.mark.parametrize("arithmetic", [Arithmetic.EXACT, Arithmetic.FAST])
@pytest.mark.parametrize("warm", [False, True])
def test_graph_solves_equal_batched_solves(gpu_lib, arithmetic, warm, mode):
    s = FluidSettings(solver=FluidSolver.DFSPH, spacing=0.02, support=2.0, arithmetic=arithmetic, warm_start=warm)
    g, e = pair(gpu_lib, s, dam_build(), mode)
    subs = 0
    for k in range(40):
        a, b = g.step(1e-3), e.step(1e-3)
        assert (a.substeps, a.iterations, a.held_back) == (b.substeps, b.iterations, b.held_back), k
        subs += a.substeps
    assert g.state_hash() == e.state_hash()
    # every substep ran as one graph (recorded when first met, then reused)
    assert g.graph_substeps() == (subs if mode == 2 else 0)
    assert e.graph_substeps() == 0


def test_graph_solves_match_the_restatement(gpu_lib, oracle_lib):
    s = FluidSettings(solver=FluidSolver.DFSPH, spacing=0.02, support=2.0, arithmetic=Arithmetic.EXACT)
    g = gpu_lib.FluidWorld(s)
    o = oracle_lib.OracleWorld(s, residual_sum=1)
    for w in (g, o):
        dam_build()(w)
    for k in range(30):
        a, b = g.step(1e-3), o.step(1e-3)
        assert a.iterations == b.iterations, k
    assert g.state_hash() == o.state_hash()
    assert g.graph_substeps() > 0


def test_a_solve_that_hits_max_iterations_stops_there(gpu_lib):
    # a density tolerance no compressed water meets: the density solve runs to max_iterations on
    # both paths (the divergence solve of water at rest has no error and stops at min_iterations)
    s = FluidSettings(solver=FluidSolver.DFSPH, spacing=0.02, support=2.0, arithmetic=Arithmetic.EXACT,
                      divergence_tolerance=1e-12, density_tolerance=1e-12, max_iterations=5)
    g, e = pair(gpu_lib, s, dam_build())
    for _ in range(16):
        a, b = g.step(1e-3), e.step(1e-3)
        assert a.iterations == b.iterations
        assert 7 * a.substeps <= a.iterations <= 10 * a.substeps
    assert g.state_hash() == e.state_hash()
    assert g.graph_substeps() > 0


def test_graphs_follow_a_changing_particle_count(gpu_lib):
    # an emitter and a drain change the count every tick: new graphs, same results
    s = FluidSettings(solver=FluidSolver.DFSPH, arithmetic=Arithmetic.EXACT)

    def river(w):
        w.add_box_container((0.0, 0.0, 0.0), (2.0, 0.6, 0.3))
        w.add_emitter((0.0, 0.0, 0.0), (0.15, 0.3, 0.3), (1.0, 0.0, 0.0))
        w.add_drain((0.9, 0.0, 0.0), (2.0, 0.6, 0.3))

    g, e = pair(gpu_lib, s, river)
    subs = 0
    for k in range(30):
        a, b = g.step(TICK), e.step(TICK)
        assert (a.emitted, a.drained, a.substeps, a.iterations) == (b.emitted, b.drained, b.substeps, b.iterations), k
        subs += a.substeps
    assert g.state_hash() == e.state_hash()
    # graphs recorded for counts that never recur stop being recorded at first sight
    assert g.graph_substeps() < subs // 2, (g.graph_substeps(), subs)


def test_whole_substep_graphs_count_the_kernels_eager_launches_count(gpu_lib):
    # the same step in modes 2 and 1 (identical worlds): the same kernels, counted the same
    s = FluidSettings(solver=FluidSolver.DFSPH, spacing=0.02, support=2.0)
    worlds = []
    for mode in (2, 1):
        w = gpu_lib.FluidWorld(s)
        w.solver_graphs(mode)
        dam_build()(w)
        worlds.append(w)
    for k in range(20):
        ran = []
        for w in worlds:
            before = gpu_lib.kernel_launches()
            r = w.step(1e-3)
            ran.append((gpu_lib.kernel_launches() - before, r.iterations))
        assert ran[0] == ran[1], k
    assert worlds[0].graph_substeps() > 0
    assert worlds[0].state_hash() == worlds[1].state_hash()


def test_graph_modes_outside_0_to_2_are_refused(gpu_lib):
    w = gpu_lib.FluidWorld(FluidSettings(solver=FluidSolver.DFSPH))
    for bad in (-1, 3):
        with pytest.raises(PhysicsError) as e:
            w.solver_graphs(bad)
        assert e.value.kind == "InvalidSettings"


def test_graph_solves_count_the_kernels_they_run(gpu_lib):
    s = FluidSettings(solver=FluidSolver.DFSPH, spacing=0.02, support=2.0)
    w = gpu_lib.FluidWorld(s)
    dam_build()(w)
    w.step(1e-3)
    before = gpu_lib.kernel_launches()
    r = w.step(1e-3)
    ran = gpu_lib.kernel_launches() - before
    # per substep at least: sort and lists, density, two first checks, a push and a check per
    # iteration, viscosity, advance
    assert ran >= 2 * r.iterations + 2 + 3 * r.substeps
    # and not the capture's launches on top: well under twice that
    assert ran < 2 * (2 * r.iterations + 30 * r.substeps)


@pytest.mark.parametrize("solver,mode", [(FluidSolver.WCSPH, 2), (FluidSolver.DFSPH, 0), (FluidSolver.DFSPH, 1),
                                         (FluidSolver.DFSPH, 2)])
def test_a_substep_whose_lists_outgrow_their_room_runs_again_as_the_restatement(gpu_lib, oracle_lib, solver, mode):
    # the rerun sorts the committed state again (its own cell box, not the failed substep's)
    s = FluidSettings(solver=solver, spacing=0.02, support=2.0, arithmetic=Arithmetic.EXACT)
    g = gpu_lib.FluidWorld(s)
    g.solver_graphs(mode)
    o = oracle_lib.OracleWorld(s, residual_sum=1)
    for w in (g, o):
        dam_build()(w)
    for k in range(24):
        if k in (14, 20):
            g.debug_list_room(8)
        a, b = g.step(1e-3), o.step(1e-3)
        assert (a.substeps, a.iterations, a.held_back) == (b.substeps, b.iterations, b.held_back), k
        assert g.state_hash() == o.state_hash(), k


@pytest.mark.parametrize("arithmetic", [Arithmetic.EXACT, Arithmetic.FAST])
def test_whole_wcsph_substeps_equal_eager_substeps_and_the_restatement(gpu_lib, oracle_lib, arithmetic):
    # a WCSPH substep as one graph (sort, density, force and advance) against the same launches
    # queued one by one, and (EXACT) against the restatement
    s = FluidSettings(solver=FluidSolver.WCSPH, spacing=0.02, support=2.0, arithmetic=arithmetic)
    g, e = pair(gpu_lib, s, dam_build())
    subs = 0
    for k in range(30):
        a, b = g.step(1e-3), e.step(1e-3)
        assert (a.substeps, a.held_back) == (b.substeps, b.held_back), k
        subs += a.substeps
    assert g.state_hash() == e.state_hash()
    assert g.graph_substeps() == subs and e.graph_substeps() == 0
    if arithmetic == Arithmetic.EXACT:
        o = oracle_lib.OracleWorld(s)
        dam_build()(o)
        for _ in range(30):
            o.step(1e-3)
        assert g.state_hash() == o.state_hash()
