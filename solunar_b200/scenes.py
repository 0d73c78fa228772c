"""Seeded synthetic scenes: the dam breaks and lattices the fluid is measured and tested on.

Positions are built in float32 exactly as `FluidWorld::fill_box` builds its lattice
(src/fluid/mod.rs:493-524: start = low + spacing/2, then start + (x, y, z) * spacing, filled in
y, z, x order with sequential ids), then nudged by a seeded jitter.  The jitter generator is
the xorshift32 of the reference's `shaken` test fixture (src/fluid/mod.rs:752-774, seed
0x9E3779B9): u = seed / u32::MAX - 0.5, scaled by twice the jitter amplitude, drawn x, y, z per
particle in id order.  Every function takes any object with the FluidWorld methods it calls,
so the same scene feeds the CUDA library and the CPU restatement.
"""
from __future__ import annotations

import dataclasses

import numpy as np

from .abi import FluidSettings, FluidSolver

SEED = 0x9E3779B9


class XorShift32:
    """xorshift32 as in src/fluid/mod.rs:755-761."""

    def __init__(self, seed: int = SEED):
        self.state = seed & 0xFFFFFFFF

    def next_u32(self) -> int:
        s = self.state
        s ^= (s << 13) & 0xFFFFFFFF
        s ^= s >> 17
        s ^= (s << 5) & 0xFFFFFFFF
        self.state = s
        return s

    def uniform_block(self, count: int) -> np.ndarray:
        """count draws of (seed as f32 / u32::MAX as f32 - 0.5) in float32."""
        out = np.empty(count, dtype=np.float32)
        s = self.state
        vals = np.empty(count, dtype=np.uint32)
        for i in range(count):
            s ^= (s << 13) & 0xFFFFFFFF
            s ^= s >> 17
            s ^= (s << 5) & 0xFFFFFFFF
            vals[i] = s
        self.state = s
        f = vals.astype(np.float32)
        out[:] = f / np.float32(4294967295.0) - np.float32(0.5)
        return out


def jitter(count: int, amplitude: float, seed: int = SEED) -> np.ndarray:
    """(count, 3) float32 offsets uniform in +-amplitude, xorshift32 draws x, y, z per particle."""
    g = XorShift32(seed)
    u = g.uniform_block(3 * count).reshape(count, 3)
    return (u * np.float32(2.0 * amplitude)).astype(np.float32)


def shaken(count: int, seed: int = SEED) -> np.ndarray:
    """The reference's `shaken` fixture positions (src/fluid/mod.rs:753-774), float32."""
    g = XorShift32(seed)
    side = int(np.ceil(np.cbrt(np.float32(count))))
    out = np.empty((count, 3), dtype=np.float32)
    for index in range(count):
        lattice = np.array([index % side, index // side % side, index // side // side], dtype=np.float32)
        lattice = lattice * np.float32(0.05)
        j = np.array([g.uniform_block(1)[0] for _ in range(3)], dtype=np.float32) * np.float32(0.02)
        out[index] = lattice + j
    return out


def lattice_block(low, counts, spacing: float) -> np.ndarray:
    """fill_box's lattice (mod.rs:514-521) with counts (nx, ny, nz), in fill order, float32."""
    nx, ny, nz = (int(c) for c in counts)
    s = np.float32(spacing)
    start = np.asarray(low, dtype=np.float32) + np.float32(s * np.float32(0.5))
    y, z, x = np.meshgrid(np.arange(ny), np.arange(nz), np.arange(nx), indexing="ij")
    grid = np.stack([x.ravel(), y.ravel(), z.ravel()], axis=1).astype(np.float32)
    return (start[None, :] + grid * s).astype(np.float32)


@dataclasses.dataclass
class Scene:
    """A fluid block in a box container."""

    name: str
    settings: FluidSettings
    tank: tuple
    block_counts: tuple
    block_low: tuple = (0.0, 0.0, 0.0)
    jitter: float = 0.0
    velocity_sigma: float = 0.0
    dt: float = 1e-3
    steps: int = 1
    seed: int = SEED
    origin: tuple = (0.0, 0.0, 0.0)  # the whole scene moved by this much
    container: bool = True

    @property
    def particles(self) -> int:
        return int(np.prod(self.block_counts))

    def initial_state(self):
        low = tuple(float(b) + float(o) for b, o in zip(self.block_low, self.origin))
        pos = lattice_block(low, self.block_counts, self.settings.spacing)
        if self.jitter:
            pos = (pos + jitter(len(pos), self.jitter, self.seed)).astype(np.float32)
        vel = np.zeros_like(pos)
        if self.velocity_sigma:
            rng = np.random.default_rng(self.seed)
            vel = rng.normal(0.0, self.velocity_sigma, size=pos.shape).astype(np.float32)
        return pos, vel

    def build(self, world):
        """Adds the container and the particles to `world`; returns (positions, velocities)."""
        if self.container:
            world.add_box_container(self.origin, tuple(float(o) + float(t) for o, t in zip(self.origin, self.tank)))
        pos, vel = self.initial_state()
        world.add_particles(pos, vel)
        return pos, vel


def wcsph_dam_8k() -> Scene:
    """WCSPH dam break: 20^3 particles at 0.02 m in the corner of a 1 m tank, support 4,
    c = 20 m/s, viscosity 0.01, dt = 2e-4 s, jitter +-1e-4 m."""
    s = FluidSettings(solver=FluidSolver.WCSPH, spacing=0.02, support=4.0, sound_speed=20.0,
                      viscosity=0.01, rest_density=1000.0)
    return Scene("wcsph_dam_8k", s, (1.0, 1.0, 1.0), (20, 20, 20), jitter=1e-4, dt=2e-4, steps=1000)


def dfsph_dam_250k() -> Scene:
    """DFSPH dam break: 50 x 100 x 50 particles at 0.01 m in a 2 x 1 x 1 m tank, jitter +-1e-5 m,
    step(1e-3) x 500."""
    s = FluidSettings(solver=FluidSolver.DFSPH, spacing=0.01, support=2.0)
    return Scene("dfsph_dam_250k", s, (2.0, 1.0, 1.0), (50, 100, 50), jitter=1e-5, dt=1e-3, steps=500)


def dfsph_dam_250k_c2() -> Scene:
    """The 250k DFSPH dam with both solver tolerances at 0.1 % and warm-started solves (the
    library's opt-in settings; the reference's constants are 5e-4 / 1e-3 and cold starts),
    step(1e-3) x 500."""
    s = FluidSettings(solver=FluidSolver.DFSPH, spacing=0.01, support=2.0, divergence_tolerance=1e-3,
                      density_tolerance=1e-3, warm_start=True)
    return Scene("dfsph_dam_250k_c2", s, (2.0, 1.0, 1.0), (50, 100, 50), jitter=1e-5, dt=1e-3, steps=500)


def dfsph_precision_1m() -> Scene:
    """DFSPH precision study: 100^3 particles at 0.01 m in a 4 x 2 x 2 m tank, initial velocity
    N(0, 0.05 m/s) per component, 300 substeps."""
    s = FluidSettings(solver=FluidSolver.DFSPH, spacing=0.01, support=2.0)
    return Scene("dfsph_precision_1m", s, (4.0, 2.0, 2.0), (100, 100, 100), jitter=1e-5, velocity_sigma=0.05,
                 dt=1e-3, steps=300)


def dfsph_precision_far(counts=(100, 100, 100), origin=(1024.0, 1024.0, 1024.0)) -> Scene:
    """The precision study's block moved far from the origin, where an f32 coordinate resolves
    1.2e-4 m, about 1/80 of the spacing: no container, no gravity, velocities N(0, 0.05 m/s)."""
    s = FluidSettings(solver=FluidSolver.DFSPH, spacing=0.01, support=2.0, gravity=(0.0, 0.0, 0.0))
    return Scene("dfsph_precision_far", s, (4.0, 2.0, 2.0), counts, jitter=1e-5, velocity_sigma=0.05, dt=1e-3,
                 steps=300, origin=origin, container=False)


def dfsph_dam_1m() -> Scene:
    """DFSPH dam break at one million particles: 100^3 at 0.01 m in a 2 x 1 x 1 m tank."""
    s = FluidSettings(solver=FluidSolver.DFSPH, spacing=0.01, support=2.0)
    return Scene("dfsph_dam_1m", s, (2.0, 1.0, 1.0), (100, 100, 100), jitter=1e-5, dt=1e-3, steps=500)


def wcsph_adjoint_64k() -> Scene:
    """Differentiable WCSPH: 40^3 particles at 0.02 m in a 1 m tank, support 4, v0 ~ N(0, 0.1),
    200 steps of 2e-4 s."""
    s = FluidSettings(solver=FluidSolver.WCSPH, spacing=0.02, support=4.0, sound_speed=20.0,
                      viscosity=0.01)
    return Scene("wcsph_adjoint_64k", s, (1.0, 1.0, 1.0), (40, 40, 40), jitter=1e-4, velocity_sigma=0.1,
                 dt=2e-4, steps=200)


def small_dam(solver=FluidSolver.WCSPH, counts=(10, 12, 6), spacing=0.02, support=2.0,
              tank=(0.6, 0.4, 0.2), jitter_amp=1e-4, **settings) -> Scene:
    """A small dam break for parity tests that the CPU restatement finishes in seconds."""
    s = FluidSettings(solver=solver, spacing=spacing, support=support, **settings)
    return Scene(f"small_dam_{int(solver)}", s, tank, counts, jitter=jitter_amp, dt=1.0 / 60.0)
