"""The cell sort for hosts that cannot allocate device memory, checked against the oracle.

Some callers of this library cannot allocate GPU memory themselves: an engine that hands out all
device memory from its own pool, or a plugin that only ever receives buffers from its host.
slf_sort_by_cell_noalloc sorts arrays such a caller owns and keeps its own scratch in a fixed
device array, so it allocates nothing.  Its permutation must be the (cell, id) order of
update_neighbors (src/fluid/mod.rs:541-550) as the oracle computes it, and the one
slf_update_neighbors applies, call after call: every call finds the scratch array as the one
before left it.  The cases reach the array's limits: exactly 262,144 particles, and a bounding
box of exactly 1,048,576 cells, whose last cell ends at the scan's grand total.
"""
import numpy as np
import pytest

from solunar_b200 import scenes
from solunar_b200.abi import FluidSettings, PhysicsError

pytestmark = pytest.mark.gpu

MAX_PARTICLES = 1 << 18
MAX_CELLS = 1 << 20


def scene(count: int, seed: int) -> np.ndarray:
    side = int(np.ceil(count ** (1.0 / 3.0)))
    lattice = scenes.lattice_block((0.0, 0.0, 0.0), (side, side, side), 0.05)[:count]
    return (lattice + scenes.jitter(count, 0.01, seed)).astype(np.float32)


def flat_sheet(count: int, radius: float, seed: int) -> np.ndarray:
    """Particles at cell centres over a 1024 x 1024 x 1 cell box, its two far corners occupied."""
    rng = np.random.default_rng(seed)
    r = np.float32(radius)
    pos = np.empty((count, 3), np.float32)
    pos[:, 0] = rng.integers(0, 1024, count).astype(np.float32) * r + np.float32(0.5) * r
    pos[:, 1] = rng.integers(0, 1024, count).astype(np.float32) * r + np.float32(0.5) * r
    pos[:, 2] = np.float32(0.5) * r
    pos[0] = (np.float32(0.5) * r, np.float32(0.5) * r, np.float32(0.5) * r)
    pos[1] = (np.float32(1023.5) * r, np.float32(1023.5) * r, np.float32(0.5) * r)
    return pos


def cells_of(pos: np.ndarray, radius: float) -> np.ndarray:
    return np.floor(pos / np.float32(radius)).astype(np.int64)


def sort_on_device(gpu_lib, pos: np.ndarray, ids: np.ndarray, radius: float) -> np.ndarray:
    import torch

    count = len(pos)
    d_pos = torch.from_numpy(np.ascontiguousarray(pos, np.float32)).cuda()
    d_ids = torch.from_numpy(np.ascontiguousarray(ids, np.uint32).view(np.int32)).cuda()
    order = torch.full((count,), -1, dtype=torch.int32, device="cuda")
    torch.cuda.synchronize()
    gpu_lib.sort_by_cell_noalloc(d_pos.data_ptr(), d_ids.data_ptr(), count, radius, order.data_ptr())
    return order.cpu().numpy().view(np.uint32)


def oracle_order(oracle_lib, settings: FluidSettings, pos: np.ndarray):
    """Input indexes and positions in the oracle's (cell, id) order after update_neighbors (the
    oracle numbers particles 0..n-1 in input order)."""
    world = oracle_lib.OracleWorld(settings)
    world.add_particles(pos)
    world.update_neighbors()
    return world.ids(), world.positions().astype(np.float32)


def test_the_no_alloc_sort_orders_particles_as_the_oracle_and_update_neighbors(gpu_lib, oracle_lib):
    settings = FluidSettings()
    radius = settings.radius()
    for count, seed in [(3000, scenes.SEED), (50000, 12345), (MAX_PARTICLES, 777)]:
        pos = scene(count, seed)
        ids = np.arange(count, dtype=np.uint32)
        perm = sort_on_device(gpu_lib, pos, ids, radius)
        assert np.array_equal(np.sort(perm), np.arange(count, dtype=np.uint32))
        ref_ids, ref_pos = oracle_order(oracle_lib, settings, pos)
        assert np.array_equal(ids[perm], ref_ids)
        assert np.array_equal(pos[perm], ref_pos)
        world = gpu_lib.FluidWorld(settings)
        world.add_particles(pos)
        world.update_neighbors()
        assert np.array_equal(ids[perm], world.ids())
        assert np.array_equal(pos[perm], world.positions())
        world.close()


def test_a_box_of_exactly_the_scratch_cells_sorts_to_its_last_cell(gpu_lib, oracle_lib):
    settings = FluidSettings()
    radius = settings.radius()
    pos = flat_sheet(MAX_PARTICLES, radius, 4242)
    cells = cells_of(pos, radius)
    span = cells.max(axis=0) - cells.min(axis=0) + 1
    assert int(np.prod(span)) == MAX_CELLS
    # ids in input order, as the oracle numbers them: the two orders must be equal
    perm = sort_on_device(gpu_lib, pos, np.arange(len(pos), dtype=np.uint32), radius)
    ref_ids, ref_pos = oracle_order(oracle_lib, settings, pos)
    assert np.array_equal(perm, ref_ids)
    assert np.array_equal(pos[perm], ref_pos)
    assert tuple(cells[perm[-1]]) == (1023, 1023, 0)
    # ids against the input order, on the scratch array the first call left: the same cells in
    # the same order, ids ascending within each cell
    ids = np.arange(len(pos), dtype=np.uint32)[::-1].copy()
    perm = sort_on_device(gpu_lib, pos, ids, radius)
    assert np.array_equal(np.sort(perm), np.arange(len(pos), dtype=np.uint32))
    key = cells[perm]
    assert np.array_equal(key, cells[ref_ids])
    order_ids = ids[perm]
    same_cell = np.all(key[1:] == key[:-1], axis=1)
    assert np.all(order_ids[1:][same_cell] > order_ids[:-1][same_cell])


def test_repeated_ids_still_give_a_permutation_in_cell_order(gpu_lib):
    radius = FluidSettings().radius()
    pos = scene(5000, 99)
    ids = np.zeros(len(pos), dtype=np.uint32)
    ids[::3] = 7
    perm = sort_on_device(gpu_lib, pos, ids, radius)
    assert np.array_equal(np.sort(perm), np.arange(len(pos), dtype=np.uint32))
    key = cells_of(pos, radius)[perm]
    lo = key.min(axis=0)
    span = key.max(axis=0) - lo + 1
    lin = ((key[:, 0] - lo[0]) * span[1] + (key[:, 1] - lo[1])) * span[2] + (key[:, 2] - lo[2])
    assert np.all(np.diff(lin) >= 0)
    order_ids = ids[perm]
    same_cell = lin[1:] == lin[:-1]
    assert np.all(order_ids[1:][same_cell] >= order_ids[:-1][same_cell])


def test_the_no_alloc_sort_refuses_what_its_scratch_cannot_hold(gpu_lib):
    import torch

    radius = FluidSettings().radius()
    far = torch.tensor([[0.0, 0.0, 0.0], [1000.0, 1000.0, 1000.0]], dtype=torch.float32, device="cuda")
    ids = torch.tensor([0, 1], dtype=torch.int32, device="cuda")
    order = torch.zeros(2, dtype=torch.int32, device="cuda")
    torch.cuda.synchronize()
    with pytest.raises(PhysicsError) as e:
        gpu_lib.sort_by_cell_noalloc(far.data_ptr(), ids.data_ptr(), 2, 0.1, order.data_ptr())
    assert e.value.kind == "OutOfRange"
    # refused on the host before any launch: more particles than the array holds
    with pytest.raises(PhysicsError) as e:
        gpu_lib.sort_by_cell_noalloc(far.data_ptr(), ids.data_ptr(), MAX_PARTICLES + 1, 0.1, order.data_ptr())
    assert e.value.kind == "OutOfRange"
    # one cell column more than the array holds: 1025 x 1024 x 1 cells
    r = np.float32(radius)
    sheet = flat_sheet(4096, radius, 5)
    sheet[2] = (np.float32(1024.5) * r, np.float32(0.5) * r, np.float32(0.5) * r)
    with pytest.raises(PhysicsError) as e:
        sort_on_device(gpu_lib, sheet, np.arange(len(sheet), dtype=np.uint32), radius)
    assert e.value.kind == "OutOfRange"


def test_cells_that_saturate_are_refused_not_written_outside_the_array(gpu_lib, oracle_lib):
    # 64 particles (two whole warps) whose x cell saturates to the i32 maximum, beside a few near
    # the origin: the box spans 2^31 cells along x and the call must refuse it
    settings = FluidSettings()
    radius = settings.radius()
    pos = np.zeros((72, 3), np.float32)
    pos[:64, 0] = np.float32(1e30)
    pos[64:] = np.float32(0.01) * np.arange(8, dtype=np.float32)[:, None]
    with pytest.raises(PhysicsError) as e:
        sort_on_device(gpu_lib, pos, np.arange(72, dtype=np.uint32), radius)
    assert e.value.kind == "OutOfRange"
    # the array is intact: the next call sorts as the oracle does
    pos = scene(2000, 31)
    perm = sort_on_device(gpu_lib, pos, np.arange(len(pos), dtype=np.uint32), radius)
    ref_ids, _ = oracle_order(oracle_lib, settings, pos)
    assert np.array_equal(perm, ref_ids)
