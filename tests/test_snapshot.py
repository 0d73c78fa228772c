"""Fluid snapshots (src/fluid/save.rs, SLFL version 3), against both implementations.

The reference's snapshot tests (save.rs:229-313), restated, run on the CPU restatement and,
marked `gpu`, on the CUDA library; snapshots then cross between the two: the library's bytes
load into the restatement and step on to the same state, and the other way round.
"""
import numpy as np
import pytest

from solunar_b200.abi import Arithmetic, FluidSettings, PhysicsError

TICK = np.float32(1.0 / 60.0)
CHECKSUM_BYTES = 8


@pytest.fixture(params=["oracle", pytest.param("gpu", marks=pytest.mark.gpu)])
def backend(request):
    """(make, load): new worlds and loaded snapshots, of the CPU restatement or the CUDA library."""
    if request.param == "oracle":
        from oracle import py_oracle

        py_oracle.build()
        return (lambda **kw: py_oracle.OracleWorld(FluidSettings(**kw)), py_oracle.OracleWorld.load_snapshot)
    gpu = request.getfixturevalue("gpu_lib")
    return (lambda **kw: gpu.FluidWorld(FluidSettings(**kw)), gpu.FluidWorld.load_snapshot)


def fnv1a(data: bytes) -> int:
    h = 0xCBF29CE484222325
    for b in data:
        h = ((h ^ b) * 0x00000100000001B3) & 0xFFFFFFFFFFFFFFFF
    return h


def pool(make):
    # save.rs:199-221
    w = make()
    w.add_box_container((0.0, 0.0, 0.0), (1.0, 1.0, 0.6))
    w.add_wall((0.45, 0.0, 0.0), (0.55, 0.3, 0.6))
    w.fill_box((0.0, 0.0, 0.0), (0.4, 0.5, 0.6))
    w.add_emitter((0.05, 0.7, 0.2), (0.2, 0.8, 0.4), (1.0, 0.0, 0.0))
    w.add_drain((0.8, 0.0, 0.0), (1.0, 0.1, 0.6))
    return w


def steps(w, count):
    for _ in range(count):
        w.step(TICK)


def test_water_past_the_domain_is_taken_out_and_the_domain_kept(backend):
    # save.rs:229-255
    make, load = backend
    w = pool(make)
    low, high = (-1.0, -1.0, -1.0), (2.0, 0.3, 2.0)
    w.set_domain((low, high))
    before = w.len()
    r = w.step(TICK)
    assert r.lost > 0
    assert np.all(w.positions()[:, 1] <= 0.3)
    assert w.len() + r.lost <= before + r.emitted
    loaded = load(w.save_snapshot())
    # the domain survives the round trip: the loaded world saves the same bytes
    assert loaded.save_snapshot() == w.save_snapshot()
    with pytest.raises(PhysicsError):
        w.set_domain((high, low))
    with pytest.raises(PhysicsError):
        w.set_domain((low, (float("nan"),) * 3))


def test_a_loaded_fluid_steps_on_exactly_as_the_saved_one(backend):
    # save.rs:257-270
    make, load = backend
    w = pool(make)
    steps(w, 20)
    saved = w.save_snapshot()
    loaded = load(saved)
    assert loaded.save_snapshot() == saved
    assert loaded.state_hash() == w.state_hash()
    steps(w, 30)
    steps(loaded, 30)
    assert loaded.state_hash() == w.state_hash()
    assert loaded.len() == w.len()


def test_a_cut_or_flipped_fluid_snapshot_is_refused_without_a_panic(backend):
    # save.rs:272-313
    make, load = backend
    w = make()
    w.add_box_container((0.0, 0.0, 0.0), (0.3, 0.3, 0.3))
    w.fill_box((0.0, 0.0, 0.0), (0.15, 0.15, 0.15))
    w.add_drain((0.0, 0.0, 0.0), (0.05, 0.05, 0.05))
    saved = w.save_snapshot()
    for end in range(len(saved)):
        with pytest.raises(PhysicsError):
            load(saved[:end])
    for at in range(len(saved)):
        flipped = bytearray(saved)
        flipped[at] ^= 0x41
        with pytest.raises(PhysicsError):
            load(bytes(flipped))
    # a good checksum over bad content is still refused
    bad = bytearray(saved[:-CHECKSUM_BYTES])
    bad[8] = 7  # the solver tag, right after magic and version
    bad += fnv1a(bytes(bad)).to_bytes(8, "little")
    with pytest.raises(PhysicsError, match="invalid snapshot: fluid solver"):
        load(bytes(bad))
    later = bytearray(saved[:-CHECKSUM_BYTES])
    later[4:8] = (3 + 1).to_bytes(4, "little")
    later += fnv1a(bytes(later)).to_bytes(8, "little")
    with pytest.raises(PhysicsError, match="unsupported snapshot version 4"):
        load(bytes(later))


@pytest.mark.gpu
def test_snapshots_cross_between_the_library_and_the_restatement(gpu_lib, oracle_lib):
    # EXACT arithmetic: the same bytes, and either side steps on to the other's state
    s = FluidSettings(arithmetic=Arithmetic.EXACT)
    g = pool(lambda: gpu_lib.FluidWorld(s))
    steps(g, 10)
    saved = g.save_snapshot()
    o = oracle_lib.OracleWorld.load_snapshot(saved, s, residual_sum=1)
    assert o.save_snapshot() == saved
    steps(g, 15)
    steps(o, 15)
    assert g.state_hash() == o.state_hash()
    back = gpu_lib.FluidWorld.load_snapshot(o.save_snapshot(), s)
    steps(back, 5)
    steps(o, 5)
    assert back.state_hash() == o.state_hash()
