"""TEST INFRASTRUCTURE ONLY: ctypes wrapper of the CPU restatement (oracle/liboracle_fluid.so).

Used by tests/, __graft_entry__.smoke() and bench.py's CPU baseline as the checker; the
library never imports it.  `OracleWorld` has the method names of solunar_b200.FluidWorld so a
parity test can drive both the same way.  `precision=32` is the float restatement of the
reference (parity oracle), `precision=64` the double one (precision oracle).
`residual_sum=0` sums the DFSPH solver error as the reference does (sequential, working
precision, src/fluid/dfsph.rs:266-267); `residual_sum=1` takes a compensated sum in double, as
the CUDA library does.
"""
from __future__ import annotations

import ctypes
import os
import subprocess

import numpy as np

from solunar_b200.abi import (CBodyPose, CBodyPush, CReport, CSettings, FluidReport, FluidSettings, PhysicsError,
                               step_with_bodies_call, vec3)

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "liboracle_fluid.so")

_lib = None


def build() -> str:
    """Compiles the restatement with its Makefile (gcc, OpenMP)."""
    subprocess.run(["make", "-s", "-C", HERE], check=True)
    return LIB_PATH


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            build()
        L = ctypes.CDLL(LIB_PATH)
        vp = ctypes.c_void_p
        f3 = ctypes.POINTER(ctypes.c_float)
        u32p = ctypes.POINTER(ctypes.c_uint32)
        u64p = ctypes.POINTER(ctypes.c_uint64)
        dp = ctypes.POINTER(ctypes.c_double)
        sig = {
            "orc_create": [ctypes.POINTER(CSettings), ctypes.c_int32, ctypes.c_int32, ctypes.POINTER(vp)],
            "orc_set_threads": [vp, ctypes.c_int32],
            "orc_len": [vp, u64p],
            "orc_particle_mass": [vp, dp],
            "orc_kernel": [vp, dp, dp],
            "orc_add_particles": [vp, ctypes.c_uint64, f3, f3, u32p],
            "orc_fill_box": [vp, f3, f3, u64p],
            "orc_set_domain": [vp, f3, f3],
            "orc_add_box_container": [vp, f3, f3, u32p],
            "orc_add_wall": [vp, f3, f3, u32p],
            "orc_remove_boundary": [vp, ctypes.c_uint32, ctypes.POINTER(ctypes.c_int32)],
            "orc_add_emitter": [vp, f3, f3, f3, u32p],
            "orc_add_drain": [vp, f3, f3, u32p],
            "orc_remove_flow": [vp, ctypes.c_uint32, ctypes.POINTER(ctypes.c_int32)],
            "orc_run_flows": [vp, u32p, u32p],
            "orc_save_snapshot": [vp, ctypes.POINTER(ctypes.c_uint8), ctypes.c_uint64, u64p],
            "orc_load_snapshot": [ctypes.POINTER(ctypes.c_uint8), ctypes.c_uint64, ctypes.POINTER(CSettings),
                                  ctypes.c_int32, ctypes.c_int32, ctypes.POINTER(vp)],
            "orc_terrain_nodes": [vp, f3, f3, u64p],
            "orc_add_terrain": [vp, f3, f3, f3, ctypes.c_uint64, u32p],
            "orc_terrain_probe": [vp, ctypes.c_uint32, f3, dp, dp, dp, dp, ctypes.POINTER(ctypes.c_int32)],
            "orc_wall_count": [vp, u64p],
            "orc_read_wall_positions": [vp, dp, ctypes.c_uint64],
            "orc_step": [vp, ctypes.c_float, ctypes.POINTER(CReport)],
            "orc_couple": [vp, ctypes.c_uint64, ctypes.c_int32, f3],
            "orc_uncouple": [vp, ctypes.c_uint64, ctypes.POINTER(ctypes.c_int32)],
            "orc_coupled": [vp, u64p, u32p, u32p, ctypes.c_uint64, u64p],
            "orc_step_with_bodies": [vp, ctypes.c_float, ctypes.POINTER(CBodyPose), ctypes.c_uint64,
                                     ctypes.POINTER(CReport), ctypes.POINTER(CBodyPush), ctypes.c_uint64, u64p],
            "orc_update_neighbors": [vp],
            "orc_compute_densities": [vp],
            "orc_read_ids": [vp, u32p, ctypes.c_uint64],
            "orc_read_positions": [vp, dp, ctypes.c_uint64],
            "orc_read_velocities": [vp, dp, ctypes.c_uint64],
            "orc_read_densities": [vp, dp, ctypes.c_uint64],
            "orc_neighbor_lists": [vp, u32p, ctypes.c_uint64, u32p, ctypes.c_uint64, u64p],
            "orc_wall_neighbor_lists": [vp, u32p, ctypes.c_uint64, u32p, ctypes.c_uint64, u64p],
            "orc_state_hash": [vp, u64p],
            "orc_last_iterations": [vp, u32p],
            "orc_tangent_run": [ctypes.POINTER(CSettings), ctypes.c_int32, ctypes.c_int32, f3, f3, ctypes.c_uint64, f3,
                                f3, dp, dp, dp,
                                ctypes.c_uint32, ctypes.c_float, u32p, ctypes.c_uint64, dp, dp, dp, dp, u32p],
            "orc_kernel_eval_f32": [ctypes.c_float, ctypes.c_uint64, f3, f3, f3, f3],
            "orc_grid_ranges": [ctypes.POINTER(ctypes.c_int32), ctypes.c_uint64, ctypes.POINTER(ctypes.c_int32),
                                ctypes.c_uint64, ctypes.c_int32, u32p, ctypes.POINTER(ctypes.c_int32)],
        }
        for name, args in sig.items():
            fn = getattr(L, name)
            fn.argtypes = args
            fn.restype = ctypes.c_int32
        L.orc_tangent_hold.argtypes = [ctypes.c_uint32]
        L.orc_tangent_hold.restype = None
        L.orc_snapshot_message.argtypes = []
        L.orc_snapshot_message.restype = ctypes.c_char_p
        L.orc_destroy.argtypes = [vp]
        L.orc_destroy.restype = None
        _lib = L
    return _lib


def _check(code: int):
    if code != 0:
        raise PhysicsError(code)


def _ptr(a: np.ndarray, ctype):
    return a.ctypes.data_as(ctypes.POINTER(ctype))


# DFSPH quantities a tangent run can hold constant (their derivative dropped), for measuring what
# each path of the substep contributes (World::hold in oracle/fluid_oracle.hpp)
TANGENT_HOLD = {"fluid_gradients": 1, "wall_gradients": 2, "factors": 4, "densities": 8, "viscosity": 16,
                "stiffness": 32, "fluid_viscosity": 64, "wall_viscosity": 128}


def tangent_run(settings: FluidSettings, container, positions, velocities, dpositions, dvelocities,
                dparams=(0.0, 0.0, 0.0, 0.0, 0.0), steps: int = 1, dt: float = 1e-3, residual_sum: int = 1,
                forced_iterations=None, precision: int = 64, hold=()):
    """The restatement in forward-mode derivative numbers (oracle/dual.hpp): values of the FP64
    method (precision 64) or of the float restatement bit for bit (32, the FP32 program the CUDA
    library runs), derivatives in double; -32: the float restatement's values with every
    derivative operation rounded to float.  A world with one box container
    `container` = (low, high), the particles added in row order (ids 0..n-1), `steps` calls of
    step(dt).  Each input carries a tangent: dpositions, dvelocities (n x 3) and dparams (viscosity,
    sound speed, gravity x, y, z).  forced_iterations: the DFSPH solves' iteration counts
    (divergence, density of each substep in turn) to take instead of stopping on the tolerances,
    so that the run follows another run's discrete steps.  hold: names of TANGENT_HOLD whose
    derivative the run drops.  Returns (positions, velocities, their tangents, ids) of the final
    state, rows in id order."""
    p = np.ascontiguousarray(positions, dtype=np.float32).reshape(-1, 3)
    v = np.ascontiguousarray(velocities, dtype=np.float32).reshape(-1, 3)
    dp_ = np.ascontiguousarray(dpositions, dtype=np.float64).reshape(-1, 3)
    dv_ = np.ascontiguousarray(dvelocities, dtype=np.float64).reshape(-1, 3)
    dq = np.ascontiguousarray(dparams, dtype=np.float64).reshape(5)
    lo = np.ascontiguousarray(container[0], dtype=np.float32)
    hi = np.ascontiguousarray(container[1], dtype=np.float32)
    n = len(p)
    outs = [np.zeros((n, 3), dtype=np.float64) for _ in range(4)]
    ids = np.zeros(n, dtype=np.uint32)
    c = settings.to_c()
    f = ctypes.c_float
    d = ctypes.c_double
    forced = np.ascontiguousarray([] if forced_iterations is None else forced_iterations, dtype=np.uint32)
    mask = 0
    for name in hold:
        mask |= TANGENT_HOLD[name]
    lib().orc_tangent_hold(ctypes.c_uint32(mask))
    _check(lib().orc_tangent_run(ctypes.byref(c), precision, residual_sum, _ptr(lo, f), _ptr(hi, f), n, _ptr(p, f), _ptr(v, f),
                                 _ptr(dp_, d), _ptr(dv_, d), _ptr(dq, d), steps, dt, _ptr(forced, ctypes.c_uint32),
                                 len(forced), *(_ptr(o, d) for o in outs), _ptr(ids, ctypes.c_uint32)))
    order = np.argsort(ids)
    return tuple(o[order] for o in outs) + (ids[order],)


class OracleWorld:
    """FluidWorld (src/fluid/mod.rs:310-339) restated on the CPU."""

    def __init__(self, settings: FluidSettings | None = None, precision: int = 32, residual_sum: int = 0,
                 threads: int = 0):
        self._settings = settings or FluidSettings()
        self.precision = precision
        c = self._settings.to_c()
        h = ctypes.c_void_p()
        _check(lib().orc_create(ctypes.byref(c), precision, residual_sum, ctypes.byref(h)))
        self._h = h
        if threads:
            lib().orc_set_threads(self._h, threads)

    def __del__(self):
        h = getattr(self, "_h", None)
        if h is not None and _lib is not None:
            _lib.orc_destroy(h)
            self._h = None

    # -- snapshots (save.rs) --
    @classmethod
    def load_snapshot(cls, data: bytes, settings: FluidSettings | None = None, precision: int = 32,
                      residual_sum: int = 0) -> "OracleWorld":
        c = (settings or FluidSettings()).to_c()
        buf = (ctypes.c_uint8 * max(len(data), 1)).from_buffer_copy(bytes(data) or b"\0")
        h = ctypes.c_void_p()
        st = lib().orc_load_snapshot(buf, len(data), ctypes.byref(c), precision, residual_sum, ctypes.byref(h))
        if st != 0:
            raise PhysicsError(st, lib().orc_snapshot_message().decode())
        self = cls.__new__(cls)
        self._h = h
        self.precision = precision
        self._settings = settings or FluidSettings()
        return self

    def save_snapshot(self) -> bytes:
        size = ctypes.c_uint64()
        _check(lib().orc_save_snapshot(self._h, None, 0, ctypes.byref(size)))
        buf = (ctypes.c_uint8 * max(size.value, 1))()
        _check(lib().orc_save_snapshot(self._h, buf, size.value, ctypes.byref(size)))
        return bytes(buf[: size.value])

    # -- settings --
    def settings(self) -> FluidSettings:
        return self._settings

    def set_threads(self, threads: int):
        lib().orc_set_threads(self._h, threads)

    def particle_mass(self) -> float:
        v = ctypes.c_double()
        lib().orc_particle_mass(self._h, ctypes.byref(v))
        return v.value

    def kernel(self):
        r, s = ctypes.c_double(), ctypes.c_double()
        lib().orc_kernel(self._h, ctypes.byref(r), ctypes.byref(s))
        return r.value, s.value

    def len(self) -> int:
        v = ctypes.c_uint64()
        lib().orc_len(self._h, ctypes.byref(v))
        return v.value

    __len__ = len

    # -- particles and walls --
    def add_particle(self, position, velocity) -> int:
        return int(self.add_particles(np.asarray([position]), np.asarray([velocity]))[0])

    def add_particles(self, positions, velocities=None) -> np.ndarray:
        p = np.ascontiguousarray(positions, dtype=np.float32).reshape(-1, 3)
        v = np.zeros_like(p) if velocities is None else np.ascontiguousarray(velocities, dtype=np.float32).reshape(-1, 3)
        ids = np.zeros(len(p), dtype=np.uint32)
        _check(lib().orc_add_particles(self._h, len(p), _ptr(p, ctypes.c_float), _ptr(v, ctypes.c_float),
                                       _ptr(ids, ctypes.c_uint32)))
        return ids

    def fill_box(self, low, high) -> int:
        n = ctypes.c_uint64()
        _check(lib().orc_fill_box(self._h, vec3(low), vec3(high), ctypes.byref(n)))
        return n.value

    def set_domain(self, domain):
        if domain is None:
            _check(lib().orc_set_domain(self._h, None, None))
        else:
            _check(lib().orc_set_domain(self._h, vec3(domain[0]), vec3(domain[1])))

    def add_box_container(self, low, high) -> int:
        i = ctypes.c_uint32()
        _check(lib().orc_add_box_container(self._h, vec3(low), vec3(high), ctypes.byref(i)))
        return i.value

    def add_wall(self, low, high) -> int:
        i = ctypes.c_uint32()
        _check(lib().orc_add_wall(self._h, vec3(low), vec3(high), ctypes.byref(i)))
        return i.value

    def remove_boundary(self, boundary: int) -> bool:
        r = ctypes.c_int32()
        _check(lib().orc_remove_boundary(self._h, boundary, ctypes.byref(r)))
        return bool(r.value)

    # ---- terrain (terrain.rs) ----
    def terrain_nodes(self, low, high):
        n = (ctypes.c_uint64 * 3)()
        _check(lib().orc_terrain_nodes(self._h, vec3(low), vec3(high), n))
        return tuple(int(v) for v in n)

    def add_terrain(self, low, high, distances) -> int:
        d = np.ascontiguousarray(distances, dtype=np.float32).ravel()
        i = ctypes.c_uint32()
        _check(lib().orc_add_terrain(self._h, vec3(low), vec3(high), _ptr(d, ctypes.c_float), d.size, ctypes.byref(i)))
        return i.value

    def terrain_probe(self, region: int, point):
        """(distance, normal, ground density, ground gradient) at `point`, or None outside."""
        d, rho = ctypes.c_double(), ctypes.c_double()
        nrm, grad = (ctypes.c_double * 3)(), (ctypes.c_double * 3)()
        inside = ctypes.c_int32()
        _check(lib().orc_terrain_probe(self._h, region, vec3(point), ctypes.byref(d), nrm, ctypes.byref(rho), grad,
                                       ctypes.byref(inside)))
        if not inside.value:
            return None
        return d.value, np.array(nrm[:]), rho.value, np.array(grad[:])

    # ---- emitters and drains (flow.rs:86-139) ----
    def add_emitter(self, low, high, velocity) -> int:
        i = ctypes.c_uint32()
        _check(lib().orc_add_emitter(self._h, vec3(low), vec3(high), vec3(velocity), ctypes.byref(i)))
        return i.value

    def add_drain(self, low, high) -> int:
        i = ctypes.c_uint32()
        _check(lib().orc_add_drain(self._h, vec3(low), vec3(high), ctypes.byref(i)))
        return i.value

    def remove_flow(self, flow: int) -> bool:
        r = ctypes.c_int32()
        _check(lib().orc_remove_flow(self._h, flow, ctypes.byref(r)))
        return bool(r.value)

    def run_flows(self):
        e, d = ctypes.c_uint32(), ctypes.c_uint32()
        _check(lib().orc_run_flows(self._h, ctypes.byref(e), ctypes.byref(d)))
        return e.value, d.value

    def wall_positions(self) -> np.ndarray:
        n = ctypes.c_uint64()
        lib().orc_wall_count(self._h, ctypes.byref(n))
        out = np.zeros((n.value, 3), dtype=np.float64)
        _check(lib().orc_read_wall_positions(self._h, _ptr(out, ctypes.c_double), n.value))
        return out

    # -- stepping --
    def step(self, dt: float) -> FluidReport:
        r = CReport()
        _check(lib().orc_step(self._h, dt, ctypes.byref(r)))
        return FluidReport.from_c(r)

    def couple(self, body: int, shape, dims):
        """FluidWorld::couple (couple.rs:165-200)."""
        d = list(dims) + [0.0] * (3 - len(dims))
        _check(lib().orc_couple(self._h, body, int(shape), vec3(d)))

    def uncouple(self, body: int) -> bool:
        r = ctypes.c_int32()
        _check(lib().orc_uncouple(self._h, body, ctypes.byref(r)))
        return bool(r.value)

    def coupled(self):
        """[(body, points, probes)] in body order."""
        n = ctypes.c_uint64()
        _check(lib().orc_coupled(self._h, None, None, None, 0, ctypes.byref(n)))
        k = n.value
        b, p, q = (ctypes.c_uint64 * max(k, 1))(), (ctypes.c_uint32 * max(k, 1))(), (ctypes.c_uint32 * max(k, 1))()
        _check(lib().orc_coupled(self._h, b, p, q, k, ctypes.byref(n)))
        return [(int(b[i]), int(p[i]), int(q[i])) for i in range(k)]

    def step_with_bodies(self, dt: float, poses):
        """FluidWorld::step_with_bodies (couple.rs:219-248): (report, [BodyPush])."""
        return step_with_bodies_call(lib().orc_step_with_bodies, self._h, dt, list(poses), _check)

    def update_neighbors(self):
        _check(lib().orc_update_neighbors(self._h))

    def compute_densities(self):
        _check(lib().orc_compute_densities(self._h))

    def last_iterations(self):
        out = (ctypes.c_uint32 * 2)()
        lib().orc_last_iterations(self._h, out)
        return int(out[0]), int(out[1])

    # -- read-outs --
    def ids(self) -> np.ndarray:
        n = self.len()
        out = np.zeros(n, dtype=np.uint32)
        _check(lib().orc_read_ids(self._h, _ptr(out, ctypes.c_uint32), n))
        return out

    def _vecs(self, fn) -> np.ndarray:
        n = self.len()
        out = np.zeros((n, 3), dtype=np.float64)
        _check(fn(self._h, _ptr(out, ctypes.c_double), n))
        return out

    def positions(self) -> np.ndarray:
        return self._vecs(lib().orc_read_positions)

    def velocities(self) -> np.ndarray:
        return self._vecs(lib().orc_read_velocities)

    def densities(self) -> np.ndarray:
        n = self.len()
        out = np.zeros(n, dtype=np.float64)
        _check(lib().orc_read_densities(self._h, _ptr(out, ctypes.c_double), n))
        return out

    def _lists(self, fn):
        n = ctypes.c_uint64()
        _check(fn(self._h, None, 0, None, 0, ctypes.byref(n)))
        start = np.zeros(self.len() + 1, dtype=np.uint32)
        items = np.zeros(max(n.value, 1), dtype=np.uint32)
        _check(fn(self._h, _ptr(start, ctypes.c_uint32), len(start), _ptr(items, ctypes.c_uint32), n.value,
                  ctypes.byref(n)))
        return start, items[: n.value]

    def neighbor_lists(self):
        return self._lists(lib().orc_neighbor_lists)

    def wall_neighbor_lists(self):
        return self._lists(lib().orc_wall_neighbor_lists)

    def neighbors_of(self, index: int) -> np.ndarray:
        start, items = self.neighbor_lists()
        return items[start[index]:start[index + 1]]

    def state_hash(self) -> int:
        v = ctypes.c_uint64()
        lib().orc_state_hash(self._h, ctypes.byref(v))
        return v.value


def kernel_eval(radius: float, offsets) -> tuple:
    """Kernel::value, slope and gradient (src/fluid/mod.rs:140-164) in f32 at these offsets."""
    o = np.ascontiguousarray(offsets, dtype=np.float32).reshape(-1, 3)
    n = len(o)
    value = np.zeros(n, dtype=np.float32)
    slope = np.zeros(n, dtype=np.float32)
    grad = np.zeros((n, 3), dtype=np.float32)
    lib().orc_kernel_eval_f32(radius, n, _ptr(o, ctypes.c_float), _ptr(value, ctypes.c_float),
                              _ptr(slope, ctypes.c_float), _ptr(grad, ctypes.c_float))
    return value, slope, grad


def grid_ranges(sorted_keys, queries, force_search: bool):
    """Grid::build then Grid::range (src/fluid/mod.rs:180-247).  Returns (ranges, had_dense)."""
    k = np.ascontiguousarray(sorted_keys, dtype=np.int32).reshape(-1, 3)
    q = np.ascontiguousarray(queries, dtype=np.int32).reshape(-1, 3)
    out = np.zeros((len(q), 2), dtype=np.uint32)
    dense = ctypes.c_int32()
    lib().orc_grid_ranges(_ptr(k, ctypes.c_int32), len(k), _ptr(q, ctypes.c_int32), len(q),
                          1 if force_search else 0, _ptr(out, ctypes.c_uint32), ctypes.byref(dense))
    return out, bool(dense.value)
