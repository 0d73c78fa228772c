"""Coupled bodies (src/fluid/couple.rs, lift.rs), against both implementations.

The reference's coupling tests (couple.rs:519-811) restated with their thresholds.  The caller
owns the rigid bodies: here `tests/rigid.py`, a small integrator standing in for the reference's
PhysicsWorld (gravity, the water's pushes, a floor).  Tests that take `backend` run on the CPU
restatement and, marked `gpu`, on the CUDA library; a run with bodies on prescribed paths then
checks that the library's water and pushes are the restatement's bit for bit.
"""
import numpy as np
import pytest

import rigid
from solunar_b200.abi import Arithmetic, BodyPose, FluidSettings, FluidSolver, PhysicsError, Shape, body_handle

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


def pool(make, **kw):
    # couple.rs:519-530: a 1 x 1.2 x 1 m tank, water 0.6 m deep
    w = make(**kw)
    w.add_box_container((0.0, 0.0, 0.0), (1.0, 1.2, 1.0))
    w.fill_box((0.0, 0.0, 0.0), (1.0, 0.6, 1.0))
    return w


def drop_box(w, density):
    # couple.rs:532-540
    body = rigid.Body(1, Shape.CUBOID, (0.15, 0.15, 0.15), density, (0.5, 0.9, 0.5))
    w.couple(body.handle, Shape.CUBOID, body.dims)
    return body


def test_shapes_sample_and_bad_ones_are_refused(backend):
    # couple.rs:786-810
    make, _ = backend
    w = pool(make)
    body = body_handle(3)
    for shape, dims in ((Shape.SPHERE, (0.2,)), (Shape.CAPSULE, (0.1, 0.2)), (Shape.CUBOID, (0.3, 0.1, 0.1))):
        w.couple(body, shape, dims)
        assert len(w.coupled()) == 1
    for dims in ((0.001,), (-1.0,)):
        with pytest.raises(PhysicsError) as e:
            w.couple(body, Shape.SPHERE, dims)
        assert e.value.kind == "InvalidShape"
    assert w.uncouple(body)
    assert not w.uncouple(body)
    # a body the caller no longer has is dropped
    w.couple(body, Shape.SPHERE, (0.2,))
    w.step_with_bodies(TICK, [])
    assert w.coupled() == []


def test_a_light_box_floats_and_a_heavy_one_sinks(backend):
    # couple.rs:726-742
    make, _ = backend
    light_water = pool(make)
    light = drop_box(light_water, 400.0)
    rigid.run(light_water, [light], 180)
    heavy_water = pool(make)
    heavy = drop_box(heavy_water, 3000.0)
    rigid.run(heavy_water, [heavy], 180)
    floats, sinks = light.x[1], heavy.x[1]
    assert floats > 0.45, floats
    assert sinks < 0.3, sinks
    assert floats < 0.9, floats
    assert light_water.len() == 20 * 12 * 20


def test_a_box_floats_as_deep_as_its_density_says(backend):
    # couple.rs:672-696
    make, _ = backend
    w = pool(make)
    body = drop_box(w, 850.0)
    rigid.run(w, [body], 240)
    p = w.positions()
    tops = np.sort(p[(p[:, 0] < 0.2) & (p[:, 2] < 0.2)][:, 1])
    level = tops[-1] + FluidSettings().spacing / 2.0
    expected = level - 0.35 * 0.3
    assert abs(body.x[1] - expected) < FluidSettings().spacing, (body.x[1], expected)
    assert np.linalg.norm(body.w) < 0.05


def test_a_falling_box_lifts_the_water_and_is_slowed_by_it(backend):
    # couple.rs:743-766
    make, _ = backend
    w = pool(make)
    rigid.run(w, [], 30)
    still = float(w.positions()[:, 1].max())
    body = drop_box(w, 3000.0)
    slowest, free = 0.0, 0.0
    for tick in range(40):
        rigid.run(w, [body], 1)
        slowest = max(slowest, -body.v[1])
        free = 9.81 * float(TICK) * (tick + 1)
    assert slowest < free * 0.8, (slowest, free)
    assert float(w.positions()[:, 1].max()) > still + 0.01


def test_a_ball_faster_than_the_water_sound_speed_does_not_blow_it_apart(backend):
    # couple.rs:542-575
    make, _ = backend
    w = pool(make)
    w.set_domain(((-5.0, -5.0, -5.0), (6.0, 6.0, 6.0)))
    speed = 24.0
    ball = rigid.Body(1, Shape.SPHERE, (0.1,), 7800.0, (0.5, 0.75, 0.5), velocity=(0.0, -speed, 0.0))
    w.couple(ball.handle, Shape.SPHERE, ball.dims)
    assert FluidSettings().sound_speed < speed
    reports = rigid.run(w, [ball], 30)
    louder = max(r.sound_speed for r in reports)
    squeeze = max(r.max_compression for r in reports)
    fastest = max(r.max_speed for r in reports)
    assert louder >= 4.0 * speed, louder
    assert squeeze < 0.2, squeeze
    assert fastest < 2.0 * speed, fastest


def test_a_body_added_inside_the_water_pushes_it_aside_without_throwing_it(backend):
    # couple.rs:577-603
    make, _ = backend
    w = pool(make)
    ball = rigid.Body(1, Shape.SPHERE, (0.2,), 7800.0, (0.5, 0.6, 0.5))
    w.couple(ball.handle, Shape.SPHERE, ball.dims)
    reports = rigid.run(w, [ball], 90)
    fastest = max(r.max_speed for r in reports)
    assert fastest < 12.0, fastest
    assert reports[-1].max_speed < 2.0, reports[-1].max_speed


def test_a_floating_box_and_its_water_step_on_the_same_after_snapshots(backend):
    # couple.rs:698-708: the body's rigid state is copied with the water's snapshot
    make, load = backend
    w = pool(make)
    body = drop_box(w, 500.0)
    rigid.run(w, [body], 20)
    loaded = load(w.save_snapshot())
    assert loaded.coupled() == w.coupled()
    twin = rigid.Body(1, Shape.CUBOID, body.dims, 500.0, body.x)
    twin.v, twin.q, twin.w = body.v.copy(), body.q.copy(), body.w.copy()
    rigid.run(w, [body], 30)
    rigid.run(loaded, [twin], 30)
    assert loaded.state_hash() == w.state_hash()
    assert np.array_equal(twin.x, body.x)


def test_the_divergence_free_solver_does_not_couple(backend):
    # couple.rs:225-227
    make, _ = backend
    w = pool(make, solver=FluidSolver.DFSPH)
    body = drop_box(w, 500.0)
    with pytest.raises(PhysicsError) as e:
        w.step_with_bodies(TICK, [body.pose()])
    assert e.value.kind == "InvalidSettings"


def test_coupling_is_the_same_on_any_thread_count(oracle_lib):
    # couple.rs:768-784, on the restatement's OpenMP threads
    def go(threads):
        w = pool(lambda **kw: oracle_lib.OracleWorld(FluidSettings(**kw), threads=threads))
        body = drop_box(w, 800.0)
        rigid.run(w, [body], 20)
        return w.state_hash(), body.x[1]

    assert go(1) == go(4)


def paths(tick):
    """Prescribed poses: a ball driven down through the surface and a box turning as it slides."""
    t = float(tick) * float(TICK)
    ball = BodyPose(body_handle(1), (0.3, 0.75 - 1.5 * t, 0.4), linear_velocity=(0.0, -1.5, 0.0))
    angle = 0.8 * t
    box = BodyPose(body_handle(2, 7), (0.7 - 0.5 * t, 0.55, 0.6),
                   rotation=(0.0, np.sin(angle / 2.0), 0.0, np.cos(angle / 2.0)),
                   linear_velocity=(-0.5, 0.0, 0.0), angular_velocity=(0.0, 0.8, 0.0), dynamic=(tick % 2 == 0))
    return [ball, box]


@pytest.mark.gpu
def test_coupled_water_and_pushes_match_the_restatement_bit_for_bit(gpu_lib, oracle_lib):
    s = FluidSettings(arithmetic=Arithmetic.EXACT)
    g, o = pool(lambda: gpu_lib.FluidWorld(s)), pool(lambda: oracle_lib.OracleWorld(s))
    for w in (g, o):
        w.couple(body_handle(1), Shape.SPHERE, (0.12,))
        w.couple(body_handle(2, 7), Shape.CUBOID, (0.15, 0.08, 0.1))
    assert g.coupled() == o.coupled()
    for tick in range(40):
        (a, pa), (b, pb) = g.step_with_bodies(TICK, paths(tick)), o.step_with_bodies(TICK, paths(tick))
        assert (a.substeps, a.held_back, a.sound_speed) == (b.substeps, b.held_back, b.sound_speed), tick
        assert pa == pb, tick
    assert g.state_hash() == o.state_hash()
    assert g.save_snapshot() == o.save_snapshot()


@pytest.mark.gpu
def test_fast_arithmetic_does_not_couple(gpu_lib):
    w = pool(lambda: gpu_lib.FluidWorld(FluidSettings(arithmetic=Arithmetic.FAST)))
    body = drop_box(w, 500.0)
    with pytest.raises(PhysicsError) as e:
        w.step_with_bodies(TICK, [body.pose()])
    assert e.value.kind == "Unsupported"
