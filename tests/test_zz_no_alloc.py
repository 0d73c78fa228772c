"""The cell sort for hosts that cannot allocate device memory, checked against update_neighbors.

Some callers of this library cannot allocate GPU memory themselves: an engine that hands out all
device memory from its own pool, or a plugin that only ever receives buffers from its host.
slf_sort_by_cell_noalloc sorts arrays such a caller owns and keeps its own scratch in a fixed
device array, so it allocates nothing.  Its permutation must be the one slf_update_neighbors
applies to the same particles, call after call: the second call finds the scratch array as the
first one left it.
"""
import numpy as np
import pytest

from solunar_b200 import scenes
from solunar_b200.abi import FluidSettings, PhysicsError

pytestmark = pytest.mark.gpu


def scene(count: int, seed: int) -> np.ndarray:
    side = int(np.ceil(count ** (1.0 / 3.0)))
    lattice = scenes.lattice_block((0.0, 0.0, 0.0), (side, side, side), 0.05)[:count]
    return (lattice + scenes.jitter(count, 0.01, seed)).astype(np.float32)


def test_the_no_alloc_sort_orders_particles_as_update_neighbors(gpu_lib):
    import torch

    settings = FluidSettings()
    for count, seed in [(3000, scenes.SEED), (50000, 12345)]:
        world = gpu_lib.FluidWorld(settings)
        world.add_particles(scene(count, seed))
        ids = world.ids()
        pos = world.positions()
        d_pos = torch.from_numpy(pos.copy()).cuda()
        d_ids = torch.from_numpy(ids.view(np.int32).copy()).cuda()
        order = torch.full((count,), -1, dtype=torch.int32, device="cuda")
        torch.cuda.synchronize()
        gpu_lib.sort_by_cell_noalloc(d_pos.data_ptr(), d_ids.data_ptr(), count, settings.radius(), order.data_ptr())
        perm = order.cpu().numpy().view(np.uint32)
        world.update_neighbors()
        assert np.array_equal(np.sort(perm), np.arange(count, dtype=np.uint32))
        assert np.array_equal(ids[perm], world.ids())
        assert np.array_equal(pos[perm], world.positions())
        world.close()


def test_the_no_alloc_sort_refuses_what_its_scratch_cannot_hold(gpu_lib):
    import torch

    far = torch.tensor([[0.0, 0.0, 0.0], [1000.0, 1000.0, 1000.0]], dtype=torch.float32, device="cuda")
    ids = torch.tensor([0, 1], dtype=torch.int32, device="cuda")
    order = torch.zeros(2, dtype=torch.int32, device="cuda")
    torch.cuda.synchronize()
    with pytest.raises(PhysicsError) as e:
        gpu_lib.sort_by_cell_noalloc(far.data_ptr(), ids.data_ptr(), 2, 0.1, order.data_ptr())
    assert e.value.kind == "OutOfRange"
    with pytest.raises(PhysicsError) as e:
        gpu_lib.sort_by_cell_noalloc(far.data_ptr(), ids.data_ptr(), 1 << 20, 0.1, order.data_ptr())
    assert e.value.kind == "OutOfRange"
