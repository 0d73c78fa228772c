"""Test-harness wrapper of the fluid step and its adjoint as a torch.autograd.Function.

The library's adjoint is `step_backward` through the C ABI; this wrapper lets a test write its
loss in torch and get the gradients with `torch.autograd`.  It is test scaffolding: the library
itself has no torch dependency on its path.

`FluidRun.apply(pos0, vel0, make, steps, dt, every)` builds a world with `make()` (walls, no
particles), adds the particles (rows of pos0/vel0, which become ids 0..n-1), records `steps` calls
of `step(dt)` on a tape (`every`: the checkpoint interval, 0 keeps every substep), and returns the
final positions and velocities in id order.  Backward hands the output gradients to
`step_backward` in the world's current order and returns the gradients of pos0 and vel0 in id
order; the parameter gradients (viscosity, sound speed, gravity) of the last backward are kept on
`FluidRun.last_params`.
"""
import numpy as np
import torch


def to_id_order(ids, rows):
    out = np.empty_like(rows)
    out[ids] = rows
    return out


class FluidRun(torch.autograd.Function):
    last_params = None

    @staticmethod
    def forward(ctx, pos0, vel0, make, steps, dt, every):
        w = make()
        w.add_particles(pos0.detach().cpu().numpy(), vel0.detach().cpu().numpy())
        ids0 = w.ids().astype(np.int64)
        w.tape_begin(every)
        for _ in range(steps):
            w.step(dt)
        ids1 = w.ids().astype(np.int64)
        p = to_id_order(ids1, np.asarray(w.positions(), dtype=np.float32))
        v = to_id_order(ids1, np.asarray(w.velocities(), dtype=np.float32))
        ctx.world, ctx.ids0, ctx.ids1 = w, ids0, ids1
        ctx.device = pos0.device
        return torch.from_numpy(p).to(pos0.device), torch.from_numpy(v).to(pos0.device)

    @staticmethod
    def backward(ctx, gp, gv):
        w = ctx.world
        n = len(ctx.ids1)
        gp = np.zeros((n, 3), np.float32) if gp is None else gp.detach().cpu().numpy().astype(np.float32)
        gv = np.zeros((n, 3), np.float32) if gv is None else gv.detach().cpu().numpy().astype(np.float32)
        # row k of the world's current order is particle ids1[k]
        dp0, dv0, params = w.step_backward(gp[ctx.ids1], gv[ctx.ids1])
        w.tape_end()
        w.close()
        ctx.world = None
        FluidRun.last_params = params
        dp0 = torch.from_numpy(to_id_order(ctx.ids0, dp0)).to(ctx.device)
        dv0 = torch.from_numpy(to_id_order(ctx.ids0, dv0)).to(ctx.device)
        return dp0, dv0, None, None, None, None
