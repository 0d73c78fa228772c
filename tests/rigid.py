"""A small rigid-body integrator that stands in for the reference's PhysicsWorld in the coupling
tests: dynamic bodies under gravity and the pushes the water hands back, a floor at y = 0, and
symplectic Euler.  It is test scaffolding for driving bodies, not a restatement of src/world.rs:
the tests check what the reference's coupling tests check (a box floats or sinks, a fall is
slowed), not the rigid world's own numbers.
"""
import numpy as np

from solunar_b200.abi import BodyPose, Shape, body_handle


def quat_mul(a, b):
    ax, ay, az, aw = a
    bx, by, bz, bw = b
    return np.array([aw * bx + ax * bw + ay * bz - az * by,
                     aw * by - ax * bz + ay * bw + az * bx,
                     aw * bz + ax * by - ay * bx + az * bw,
                     aw * bw - ax * bx - ay * by - az * bz])


def rotation_matrix(q):
    x, y, z, w = q
    return np.array([[1 - 2 * (y * y + z * z), 2 * (x * y - z * w), 2 * (x * z + y * w)],
                     [2 * (x * y + z * w), 1 - 2 * (x * x + z * z), 2 * (y * z - x * w)],
                     [2 * (x * z - y * w), 2 * (y * z + x * w), 1 - 2 * (x * x + y * y)]])


class Body:
    def __init__(self, index, shape, dims, density, position, velocity=(0.0, 0.0, 0.0), dynamic=True):
        self.handle = body_handle(index)
        self.shape, self.dims = shape, tuple(dims)
        self.dynamic = dynamic
        if shape == Shape.CUBOID:
            hx, hy, hz = dims
            volume = 8.0 * hx * hy * hz
            self.mass = density * volume
            self.inertia = self.mass / 3.0 * np.array([hy * hy + hz * hz, hx * hx + hz * hz, hx * hx + hy * hy])
            self.corners = np.array([[sx * hx, sy * hy, sz * hz] for sx in (-1, 1) for sy in (-1, 1) for sz in (-1, 1)])
        elif shape == Shape.SPHERE:
            r = dims[0]
            self.mass = density * 4.0 / 3.0 * np.pi * r ** 3
            self.inertia = np.full(3, 0.4 * self.mass * r * r)
            self.corners = np.array([[0.0, -r, 0.0]])
        else:
            raise ValueError("cuboids and spheres only")
        self.x = np.array(position, dtype=np.float64)
        self.v = np.array(velocity, dtype=np.float64)
        self.q = np.array([0.0, 0.0, 0.0, 1.0])
        self.w = np.zeros(3)
        self.force = np.zeros(3)
        self.torque = np.zeros(3)

    def pose(self) -> BodyPose:
        return BodyPose(self.handle, tuple(self.x), tuple(self.q), tuple(self.v), tuple(self.w), self.dynamic)

    def take(self, push, dt):
        """The water's pushes over a step of dt, as force and torque for the next rigid step."""
        if not self.dynamic:
            return
        self.force = (np.array(push.lift, dtype=np.float64) + np.array(push.damping, dtype=np.float64)) / dt
        self.torque = (np.array(push.lift_angular, dtype=np.float64) +
                       np.array(push.damping_angular, dtype=np.float64)) / dt

    def step(self, dt, gravity=(0.0, -9.81, 0.0)):
        if not self.dynamic:
            self.x = self.x + self.v * dt
            return
        self.v = self.v + (np.array(gravity) + self.force / self.mass) * dt
        R = rotation_matrix(self.q)
        inv_world = R @ np.diag(1.0 / self.inertia) @ R.T
        self.w = self.w + inv_world @ self.torque * dt
        self.x = self.x + self.v * dt
        dq = quat_mul(np.array([*self.w, 0.0]), self.q) * (0.5 * dt)
        self.q = self.q + dq
        self.q = self.q / np.linalg.norm(self.q)
        # the floor: the lowest corner stays above y = 0
        low = min((R @ c)[1] for c in self.corners) + self.x[1]
        if low < 0.0:
            self.x[1] -= low
            if self.v[1] < 0.0:
                self.v[1] = 0.0
            self.v[[0, 2]] *= 0.9
            self.w *= 0.9
        self.force[:] = 0.0
        self.torque[:] = 0.0


def run(world, bodies, ticks, dt=np.float32(1.0 / 60.0)):
    """Steps water and bodies `ticks` times as FluidWorld::step_with_bodies and the rigid world's
    fixed step follow each other; returns the reports."""
    reports = []
    for _ in range(ticks):
        report, pushes = world.step_with_bodies(dt, [b.pose() for b in bodies])
        by = {p.body: p for p in pushes}
        for b in bodies:
            if b.handle in by:
                b.take(by[b.handle], float(dt))
            b.step(float(dt))
        reports.append(report)
    return reports
