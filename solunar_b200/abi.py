"""ctypes mirror of include/solunar_fluid.h: structs, status codes and settings helpers.

Pure definitions, no library loading, so that importing them never needs a GPU.
"""
from __future__ import annotations

import ctypes
import dataclasses
import enum

# ---- status codes (include/solunar_fluid.h; PhysicsError in src/error.rs:5-22) ----------
SLF_OK = 0
STATUS_NAMES = {
    1: "InvalidSettings",
    2: "NonFinite",
    3: "OutOfRange",
    4: "FluidFull",
    5: "DispatchIncomplete",
    6: "Unsupported",
    7: "Cuda",
    8: "Timeout",
    9: "InvalidArgument",
    10: "Snapshot",
    11: "InvalidShape",
}


class PhysicsError(Exception):
    """A failed call.  `.kind` is the PhysicsError variant name (src/error.rs:5-22)."""

    def __init__(self, code: int, message: str = ""):
        self.code = int(code)
        self.kind = STATUS_NAMES.get(self.code, f"Status{self.code}")
        super().__init__(f"{self.kind}" + (f": {message}" if message else ""))


class FluidSolver(enum.IntEnum):
    """FluidSolver (src/fluid/mod.rs:43-53)."""

    WCSPH = 0
    DFSPH = 1


class Positions(enum.IntEnum):
    ABSOLUTE = 0
    CELL_RELATIVE = 1


class Arithmetic(enum.IntEnum):
    EXACT = 0
    FAST = 1


class CSettings(ctypes.Structure):
    _fields_ = [
        ("solver", ctypes.c_int32),
        ("spacing", ctypes.c_float),
        ("rest_density", ctypes.c_float),
        ("support", ctypes.c_float),
        ("max_particles", ctypes.c_uint64),
        ("sound_speed", ctypes.c_float),
        ("viscosity", ctypes.c_float),
        ("gravity", ctypes.c_float * 3),
        ("courant", ctypes.c_float),
        ("max_substeps", ctypes.c_uint32),
        ("positions", ctypes.c_int32),
        ("arithmetic", ctypes.c_int32),
        ("warm_start", ctypes.c_int32),
        ("divergence_tolerance", ctypes.c_float),
        ("density_tolerance", ctypes.c_float),
        ("min_iterations", ctypes.c_uint32),
        ("max_iterations", ctypes.c_uint32),
        ("device", ctypes.c_int32),
    ]


class CReport(ctypes.Structure):
    _fields_ = [
        ("substeps", ctypes.c_uint32),
        ("capped", ctypes.c_int32),
        ("max_compression", ctypes.c_float),
        ("max_speed", ctypes.c_float),
        ("held_back", ctypes.c_uint32),
        ("iterations", ctypes.c_uint32),
        ("emitted", ctypes.c_uint32),
        ("drained", ctypes.c_uint32),
        ("lost", ctypes.c_uint32),
        ("sound_speed", ctypes.c_float),
    ]


@dataclasses.dataclass
class FluidSettings:
    """FluidSettings (src/fluid/mod.rs:55-95) plus this library's own fields."""

    solver: FluidSolver = FluidSolver.WCSPH
    spacing: float = 0.05
    rest_density: float = 1000.0
    support: float = 2.0
    max_particles: int = 1 << 22
    sound_speed: float = 20.0
    viscosity: float = 0.15
    gravity: tuple = (0.0, -9.81, 0.0)
    courant: float = 0.4
    max_substeps: int = 2000
    positions: Positions = Positions.ABSOLUTE
    arithmetic: Arithmetic = Arithmetic.EXACT
    warm_start: bool = False
    divergence_tolerance: float = 1e-3
    density_tolerance: float = 5e-4
    min_iterations: int = 2
    max_iterations: int = 100
    device: int = 0

    def radius(self) -> float:
        """FluidSettings::radius (mod.rs:120-122), in f32."""
        return float(ctypes.c_float(ctypes.c_float(self.spacing).value * ctypes.c_float(self.support).value).value)

    def to_c(self) -> CSettings:
        c = CSettings()
        c.solver = int(self.solver)
        c.spacing = self.spacing
        c.rest_density = self.rest_density
        c.support = self.support
        c.max_particles = int(self.max_particles)
        c.sound_speed = self.sound_speed
        c.viscosity = self.viscosity
        for i in range(3):
            c.gravity[i] = float(self.gravity[i])
        c.courant = self.courant
        c.max_substeps = int(self.max_substeps)
        c.positions = int(self.positions)
        c.arithmetic = int(self.arithmetic)
        c.warm_start = 1 if self.warm_start else 0
        c.divergence_tolerance = self.divergence_tolerance
        c.density_tolerance = self.density_tolerance
        c.min_iterations = int(self.min_iterations)
        c.max_iterations = int(self.max_iterations)
        c.device = int(self.device)
        return c

    @classmethod
    def from_c(cls, c: CSettings) -> "FluidSettings":
        return cls(
            solver=FluidSolver(c.solver),
            spacing=c.spacing,
            rest_density=c.rest_density,
            support=c.support,
            max_particles=c.max_particles,
            sound_speed=c.sound_speed,
            viscosity=c.viscosity,
            gravity=tuple(c.gravity),
            courant=c.courant,
            max_substeps=c.max_substeps,
            positions=Positions(c.positions),
            arithmetic=Arithmetic(c.arithmetic),
            warm_start=bool(c.warm_start),
            divergence_tolerance=c.divergence_tolerance,
            density_tolerance=c.density_tolerance,
            min_iterations=c.min_iterations,
            max_iterations=c.max_iterations,
            device=c.device,
        )


@dataclasses.dataclass
class FluidReport:
    """FluidReport (src/fluid/step.rs:27-49)."""

    substeps: int = 0
    capped: bool = False
    max_compression: float = 0.0
    max_speed: float = 0.0
    held_back: int = 0
    iterations: int = 0
    emitted: int = 0
    drained: int = 0
    lost: int = 0
    sound_speed: float = 0.0

    @classmethod
    def from_c(cls, r: CReport) -> "FluidReport":
        return cls(
            substeps=r.substeps,
            capped=bool(r.capped),
            max_compression=r.max_compression,
            max_speed=r.max_speed,
            held_back=r.held_back,
            iterations=r.iterations,
            emitted=r.emitted,
            drained=r.drained,
            lost=r.lost,
            sound_speed=r.sound_speed,
        )


class CProfileEntry(ctypes.Structure):
    _fields_ = [
        ("name", ctypes.c_char * 32),
        ("launches", ctypes.c_uint64),
        ("milliseconds", ctypes.c_double),
        ("algorithmic_bytes", ctypes.c_double),
    ]


class CParamGrads(ctypes.Structure):
    _fields_ = [
        ("viscosity", ctypes.c_double),
        ("sound_speed", ctypes.c_double),
        ("gravity", ctypes.c_double * 3),
    ]


class Shape(enum.IntEnum):
    """Shapes a coupled body may have (src/shape.rs Cuboid, Sphere, Capsule)."""
    CUBOID = 0   # dims: half extents
    SPHERE = 1   # dims: (radius,)
    CAPSULE = 2  # dims: (radius, half height)


def body_handle(index: int, generation: int = 0) -> int:
    """A BodyHandle's to_raw() pair as the library names bodies: index << 32 | generation."""
    return (int(index) << 32) | int(generation)


class CBodyPose(ctypes.Structure):
    _fields_ = [
        ("body", ctypes.c_uint64),
        ("position", ctypes.c_double * 3),
        ("rotation", ctypes.c_float * 4),
        ("linear_velocity", ctypes.c_float * 3),
        ("angular_velocity", ctypes.c_float * 3),
        ("dynamic", ctypes.c_int32),
    ]


class CBodyPush(ctypes.Structure):
    _fields_ = [
        ("body", ctypes.c_uint64),
        ("lift", ctypes.c_float * 3),
        ("lift_angular", ctypes.c_float * 3),
        ("damping", ctypes.c_float * 3),
        ("damping_angular", ctypes.c_float * 3),
        ("lifted", ctypes.c_int32),
    ]


@dataclasses.dataclass
class BodyPose:
    """Where a coupled body stands for a step and how it moves (src/substep.rs SubstepPose)."""
    body: int
    position: tuple
    rotation: tuple = (0.0, 0.0, 0.0, 1.0)  # x, y, z, w
    linear_velocity: tuple = (0.0, 0.0, 0.0)
    angular_velocity: tuple = (0.0, 0.0, 0.0)
    dynamic: bool = True

    def to_c(self) -> CBodyPose:
        c = CBodyPose()
        c.body = int(self.body)
        for a in range(3):
            c.position[a] = float(self.position[a])
            c.linear_velocity[a] = float(self.linear_velocity[a])
            c.angular_velocity[a] = float(self.angular_velocity[a])
        for a in range(4):
            c.rotation[a] = float(self.rotation[a])
        c.dynamic = 1 if self.dynamic else 0
        return c


@dataclasses.dataclass
class BodyPush:
    """What the water did to a coupled body over a step: impulses, to apply as force and
    torque (impulse / dt) to a dynamic body over the rigid step that follows."""
    body: int
    lift: tuple
    lift_angular: tuple
    damping: tuple
    damping_angular: tuple
    lifted: bool

    @classmethod
    def from_c(cls, c: CBodyPush) -> "BodyPush":
        return cls(int(c.body), tuple(c.lift), tuple(c.lift_angular), tuple(c.damping), tuple(c.damping_angular),
                   bool(c.lifted))


def step_with_bodies_call(fn, handle, dt, poses, check, capacity=64):
    """Runs a C step_with_bodies entry point (library or restatement) and `check`s its status:
    (report, pushes)."""
    arr = (CBodyPose * max(len(poses), 1))(*[p.to_c() for p in poses])
    out = (CBodyPush * capacity)()
    count = ctypes.c_uint64()
    r = CReport()
    check(fn(handle, ctypes.c_float(dt), arr, len(poses), ctypes.byref(r), out, capacity, ctypes.byref(count)))
    return FluidReport.from_c(r), [BodyPush.from_c(out[k]) for k in range(min(count.value, capacity))]


def vec3(v) -> "ctypes.Array[ctypes.c_float]":
    return (ctypes.c_float * 3)(float(v[0]), float(v[1]), float(v[2]))
