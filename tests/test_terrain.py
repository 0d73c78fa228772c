"""Terrain ground (src/fluid/terrain.rs), against both implementations.

The reference's terrain tests (terrain.rs:392-535) restated over its test trench
(`tests/trench.py`: the same shape as a closed-form distance field, where the reference samples
a 10 cm voxel field).  Tests that take `backend` run on the CPU restatement and, marked `gpu`, on
the CUDA library; probes of the field and of the ground a particle sees read the restatement,
as the reference's own tests read its internals.  A trench run then checks that the library
matches the restatement bit for bit.
"""
import numpy as np
import pytest

import trench
from solunar_b200.abi import Arithmetic, FluidSettings, FluidSolver, PhysicsError

TICK = np.float32(1.0 / 60.0)


@pytest.fixture(params=["oracle", pytest.param("gpu", marks=pytest.mark.gpu)])
def backend(request):
    """(make, load): new worlds and loaded snapshots, of the CPU restatement or the CUDA library."""
    if request.param == "oracle":
        from oracle import py_oracle

        py_oracle.build()
        return (lambda **kw: py_oracle.OracleWorld(FluidSettings(**kw)), py_oracle.OracleWorld.load_snapshot)
    gpu = request.getfixturevalue("gpu_lib")
    return (lambda **kw: gpu.FluidWorld(FluidSettings(**kw)), gpu.FluidWorld.load_snapshot)


def in_trench(make, **kw):
    w = make(**kw)
    trench.add_trench(w)
    return w


def test_terrain_fields_come_back_from_a_snapshot(backend):
    # terrain.rs:392-408
    make, load = backend
    w = in_trench(make)
    w.fill_box((0.6, 0.85, 0.8), (1.0, 1.2, 1.2))
    for _ in range(10):
        w.step(TICK)
    loaded = load(w.save_snapshot())
    for _ in range(20):
        w.step(TICK)
        loaded.step(TICK)
    assert loaded.state_hash() == w.state_hash()


def test_the_field_matches_the_terrain_between_nodes(oracle_lib):
    # terrain.rs:410-428
    w = in_trench(oracle_lib.OracleWorld)
    for at in [(0.5, -0.3, 0.0), (1.03, 0.07, 0.41), (0.2, -0.5, 0.2)]:
        distance = w.terrain_probe(0, at)[0]
        assert abs(distance - trench.distance([at])[0]) < 0.02, at
    # on the trench bed the way out is up, on its side wall it is across
    assert w.terrain_probe(0, (1.0, -0.38, 0.0))[1][1] > 0.9
    assert w.terrain_probe(0, (1.0, -0.2, 0.28))[1][2] < -0.9
    assert w.terrain_probe(0, (9.0, 0.0, 0.0)) is None


def test_ground_gives_what_a_box_wall_gives(oracle_lib):
    # terrain.rs:430-464: the trench bed seen from a particle resting on it gives about what a box
    # wall gives.  The gradient is probed 3 cm above the bed: exactly at rest height (2.5 cm) the
    # exact field leaves every ground site wholly solid or wholly open, so no site is partly
    # solid and the gradient is zero (the reference's voxel field is off by a little there).
    box = oracle_lib.OracleWorld(FluidSettings())
    box.add_box_container((0.0, 0.0, 0.0), (0.5, 0.5, 0.5))
    at = np.array([0.225, 0.025, 0.225])
    r = box.kernel()[0]
    d = np.linalg.norm(box.wall_positions() - at, axis=1)
    d = d[d * d < r * r]
    value, _, _ = oracle_lib.kernel_eval(r, np.stack([d, 0 * d, 0 * d], axis=1))
    wall = box.particle_mass() * float(np.sum(value))
    w = in_trench(oracle_lib.OracleWorld)
    bed = w.terrain_probe(0, (1.0, -0.375, 0.0))
    assert abs(bed[2] - wall) / wall < 0.05, (bed[2], wall)
    lifted = w.terrain_probe(0, (1.0, -0.37, 0.0))
    assert lifted[3][1] < 0.0 and abs(lifted[3][0]) < abs(lifted[3][1]) * 0.1, lifted[3]
    corner = w.terrain_probe(0, (1.0, -0.375, 0.275))
    assert corner[2] > bed[2] * 1.2, (corner[2], bed[2])


def test_water_set_down_in_a_trench_does_not_jump(backend):
    # terrain.rs:466-476
    make, _ = backend
    w = in_trench(make)
    w.fill_box((-0.1, -0.4, -0.3), (0.5, -0.1, 0.3))
    r = w.step(TICK)
    assert r.max_speed < 0.5, r
    assert r.max_compression < 0.05, r


def test_water_rests_in_a_trench_and_does_not_sink_into_it(backend):
    # terrain.rs:478-508
    make, _ = backend
    w = in_trench(make)
    w.fill_box((0.0, -0.4, -0.3), (0.6, -0.1, 0.3))
    count = w.len()
    held = 0
    for _ in range(150):
        held += w.step(TICK).held_back
    assert w.len() == count
    assert held == 0, "water got under the ground"
    p = w.positions()
    assert p[:, 1].min() > -0.4
    assert p[:, 0].max() > 1.0
    assert np.all(np.abs(p[:, 2]) < 0.35)


def test_a_terrain_region_is_checked_and_can_go_away(backend):
    # terrain.rs:510-535
    make, _ = backend
    w = make()
    with pytest.raises(PhysicsError):
        w.terrain_nodes((1.0, 1.0, 1.0), (0.0, 0.0, 0.0))
    with pytest.raises(PhysicsError):
        w.terrain_nodes((float("nan"), 0.0, 0.0), (1.0, 1.0, 1.0))
    with pytest.raises(PhysicsError) as e:
        w.terrain_nodes((0.0, 0.0, 0.0), (1e6, 1e6, 1e6))
    assert e.value.kind == "FluidFull"
    low, high = (0.0, 0.0, 0.0), (1.0, 1.0, 1.0)
    nodes = w.terrain_nodes(low, high)
    boundary = w.add_terrain(low, high, trench.sample(low, nodes, np.float32(0.025)))
    assert w.remove_boundary(boundary)
    assert not w.remove_boundary(boundary)


def test_dfsph_takes_no_terrain(backend):
    # dfsph.rs:52-55
    make, _ = backend
    w = in_trench(make, solver=FluidSolver.DFSPH)
    w.fill_box((0.0, -0.4, -0.3), (0.2, -0.2, 0.0))
    with pytest.raises(PhysicsError) as e:
        w.step(TICK)
    assert e.value.kind == "InvalidSettings"


@pytest.mark.gpu
def test_water_in_a_trench_matches_the_restatement_bit_for_bit(gpu_lib, oracle_lib):
    s = FluidSettings(arithmetic=Arithmetic.EXACT)
    g, o = gpu_lib.FluidWorld(s), oracle_lib.OracleWorld(s)
    for w in (g, o):
        trench.add_trench(w)
        w.fill_box((0.0, -0.4, -0.3), (0.6, -0.1, 0.3))
    for tick in range(30):
        a, b = g.step(TICK), o.step(TICK)
        assert (a.substeps, a.held_back) == (b.substeps, b.held_back), tick
    assert g.state_hash() == o.state_hash()
    np.testing.assert_array_equal(g.densities(), o.densities().astype(np.float32))
