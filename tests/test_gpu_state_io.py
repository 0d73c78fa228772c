"""Host-owned state through the C ABI: slf_write_state and slf_read_state.

A host that owns the particle arrays uploads them before each step and reads them back after;
the round trip must leave the step bit-identical to one on resident state, and a state with a
non finite value must be refused without touching the world.
"""
import numpy as np
import pytest

from solunar_b200.abi import Arithmetic, FluidSettings, FluidSolver, PhysicsError, Positions

pytestmark = pytest.mark.gpu

TICK = np.float32(1.0 / 60.0)


def world(gpu_lib, **kw):
    w = gpu_lib.FluidWorld(FluidSettings(solver=FluidSolver.DFSPH, **kw))
    w.add_box_container((0.0, 0.0, 0.0), (0.6, 0.5, 0.3))
    w.fill_box((0.0, 0.0, 0.0), (0.25, 0.3, 0.3))
    return w


def read_state(w):
    import torch

    n = w.len()
    p = torch.empty((n, 3), dtype=torch.float32).pin_memory()
    v = torch.empty((n, 3), dtype=torch.float32).pin_memory()
    w.read_state_ptr(p.data_ptr(), v.data_ptr(), n)
    return p.numpy().copy(), v.numpy().copy()


def test_a_host_round_trip_each_step_changes_nothing(gpu_lib):
    a = world(gpu_lib, arithmetic=Arithmetic.EXACT)
    b = world(gpu_lib, arithmetic=Arithmetic.EXACT)
    for _ in range(10):
        p, v = read_state(b)
        np.testing.assert_array_equal(p, b.positions())
        np.testing.assert_array_equal(v, b.velocities())
        b.write_state(p, v)
        a.step(TICK)
        b.step(TICK)
    assert a.state_hash() == b.state_hash()


def test_cell_relative_state_reads_as_the_absolute_positions(gpu_lib):
    # offsets and cells come back as absolute f32 positions, the same ones positions() gives
    w = world(gpu_lib, arithmetic=Arithmetic.FAST, positions=Positions.CELL_RELATIVE)
    for _ in range(3):
        w.step(TICK)
    p, v = read_state(w)
    np.testing.assert_array_equal(p, w.positions())
    np.testing.assert_array_equal(v, w.velocities())
    w.write_state(p, v)
    np.testing.assert_array_equal(w.positions(), p)


def test_a_non_finite_state_is_refused_and_the_world_kept(gpu_lib):
    w = world(gpu_lib, arithmetic=Arithmetic.EXACT)
    w.step(TICK)
    before = w.state_hash()
    p, v = w.positions().copy(), w.velocities().copy()
    for bad in (np.nan, np.inf, -np.inf):
        q = p.copy()
        q[len(q) // 2, 1] = bad
        with pytest.raises(PhysicsError) as e:
            w.write_state(q, v)
        assert e.value.kind == "NonFinite"
        u = v.copy()
        u[-1, 2] = bad
        with pytest.raises(PhysicsError):
            w.write_state(p, u)
        assert w.state_hash() == before
    # and the world steps on as if nothing had been offered
    ref = world(gpu_lib, arithmetic=Arithmetic.EXACT)
    ref.step(TICK)
    ref.step(TICK)
    w.step(TICK)
    assert w.state_hash() == ref.state_hash()
