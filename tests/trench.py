"""The reference's test trench (src/fluid/terrain.rs:360-381) as a closed-form distance field.

Flat ground at y = 0 (solid below) with a trench dug along x from -0.1 to 1.9, its bed at
y = -0.4 and 0.6 m wide (z from -0.3 to 0.3): the plane minus a box.  The reference samples the
same shape from a 10 cm voxel field; here the distance is exact to the CSG bound
max(plane, -box).  `sample` evaluates it at a terrain region's nodes, in the order add_terrain
reads them.
"""
import numpy as np

LOW = (-0.4, -0.7, -0.5)
HIGH = (2.2, 0.3, 0.5)
BOX_CENTER = np.array([0.9, -0.2, 0.0])
BOX_HALF = np.array([1.0, 0.2, 0.3])


def distance(points) -> np.ndarray:
    p = np.asarray(points, dtype=np.float64).reshape(-1, 3)
    q = np.abs(p - BOX_CENTER) - BOX_HALF
    box = np.linalg.norm(np.maximum(q, 0.0), axis=1) + np.minimum(q.max(axis=1), 0.0)
    return np.maximum(p[:, 1], -box)


def sample(low, nodes, step) -> np.ndarray:
    """f32 distances at low + (x, y, z) step, (y, z, x) order with x fastest (terrain.rs:284-291)."""
    nx, ny, nz = nodes
    y, z, x = np.meshgrid(np.arange(ny), np.arange(nz), np.arange(nx), indexing="ij")
    idx = np.stack([x.ravel(), y.ravel(), z.ravel()], axis=1).astype(np.float32)
    at = np.asarray(low, dtype=np.float32)[None, :] + idx * np.float32(step)
    return distance(at).astype(np.float32)


def add_trench(world, spacing=0.05):
    nodes = world.terrain_nodes(LOW, HIGH)
    return world.add_terrain(LOW, HIGH, sample(LOW, nodes, np.float32(spacing) / np.float32(2)))
