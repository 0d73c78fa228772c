"""FluidWorld: solunar's particle-fluid API (src/fluid/mod.rs:310-739, step.rs, dfsph.rs,
boundary.rs) over the CUDA library's C ABI (include/solunar_fluid.h).

Method names, argument meaning and errors follow the Rust `FluidWorld`; errors raise
`PhysicsError` whose `.kind` names the PhysicsError variant.  The `&dyn JobDispatch` argument of
the Rust methods has no counterpart: the GPU runs every job.
"""
from __future__ import annotations

import ctypes
import os

import numpy as np

from .abi import (CBodyPose, CBodyPush, CParamGrads, CProfileEntry, CReport, CSettings, FluidReport, FluidSettings,
                  PhysicsError, step_with_bodies_call, vec3)

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_NAME = "libsolunar_fluid.so"

_lib = None


def library_path() -> str:
    return os.path.join(HERE, LIB_NAME)


def load_library():
    """Loads the in-tree CUDA library.  Raises if it was not built: there is no CPU path."""
    global _lib
    if _lib is not None:
        return _lib
    path = library_path()
    if not os.path.exists(path):
        raise RuntimeError(f"{path} is missing: build it with `python -m solunar_b200.build` "
                           "(the fluid step has no CPU fallback)")
    L = ctypes.CDLL(path)
    vp = ctypes.c_void_p
    fp = ctypes.POINTER(ctypes.c_float)
    u32p = ctypes.POINTER(ctypes.c_uint32)
    u64p = ctypes.POINTER(ctypes.c_uint64)
    i32p = ctypes.POINTER(ctypes.c_int32)
    sig = {
        "slf_settings_default": [ctypes.POINTER(CSettings)],
        "slf_create": [ctypes.POINTER(CSettings), ctypes.POINTER(vp)],
        "slf_get_settings": [vp, ctypes.POINTER(CSettings)],
        "slf_particle_mass": [vp, fp],
        "slf_kernel": [vp, fp, fp],
        "slf_len": [vp, u64p],
        "slf_add_particle": [vp, fp, fp, u32p],
        "slf_add_particles": [vp, ctypes.c_uint64, fp, fp, u32p],
        "slf_fill_box": [vp, fp, fp, u64p],
        "slf_set_domain": [vp, fp, fp],
        "slf_add_box_container": [vp, fp, fp, u32p],
        "slf_add_wall": [vp, fp, fp, u32p],
        "slf_remove_boundary": [vp, ctypes.c_uint32, i32p],
        "slf_add_emitter": [vp, fp, fp, fp, u32p],
        "slf_terrain_nodes": [vp, fp, fp, u64p],
        "slf_add_terrain": [vp, fp, fp, fp, ctypes.c_uint64, u32p],
        "slf_save_snapshot": [vp, ctypes.POINTER(ctypes.c_uint8), ctypes.c_uint64, u64p],
        "slf_load_snapshot": [ctypes.POINTER(ctypes.c_uint8), ctypes.c_uint64, ctypes.POINTER(CSettings),
                              ctypes.POINTER(vp)],
        "slf_add_drain": [vp, fp, fp, u32p],
        "slf_remove_flow": [vp, ctypes.c_uint32, i32p],
        "slf_couple": [vp, ctypes.c_uint64, ctypes.c_int32, fp],
        "slf_uncouple": [vp, ctypes.c_uint64, i32p],
        "slf_coupled": [vp, u64p, u32p, u32p, ctypes.c_uint64, u64p],
        "slf_step_with_bodies": [vp, ctypes.c_float, ctypes.POINTER(CBodyPose), ctypes.c_uint64,
                                 ctypes.POINTER(CReport), ctypes.POINTER(CBodyPush), ctypes.c_uint64, u64p],
        "slf_wall_count": [vp, u64p],
        "slf_read_wall_positions": [vp, fp, ctypes.c_uint64],
        "slf_step": [vp, ctypes.c_float, ctypes.POINTER(CReport)],
        "slf_update_neighbors": [vp],
        "slf_compute_densities": [vp],
        "slf_read_ids": [vp, u32p, ctypes.c_uint64],
        "slf_read_positions": [vp, fp, ctypes.c_uint64],
        "slf_read_velocities": [vp, fp, ctypes.c_uint64],
        "slf_read_state": [vp, fp, fp, ctypes.c_uint64],
        "slf_read_densities": [vp, fp, ctypes.c_uint64],
        "slf_neighbor_lists": [vp, u32p, ctypes.c_uint64, u32p, ctypes.c_uint64, u64p],
        "slf_wall_neighbor_lists": [vp, u32p, ctypes.c_uint64, u32p, ctypes.c_uint64, u64p],
        "slf_state_hash": [vp, u64p],
        "slf_last_iterations": [vp, u32p, u32p],
        "slf_debug_skip_job": [vp, ctypes.c_int64],
        "slf_debug_list_room": [vp, ctypes.c_uint32],
        "slf_write_state": [vp, fp, fp, ctypes.c_uint64],
        "slf_get_stream": [vp, ctypes.POINTER(vp)],
        "slf_profile_enable": [vp, ctypes.c_int32],
        "slf_solver_graphs": [vp, ctypes.c_int32],
        "slf_graph_substeps": [vp, ctypes.POINTER(ctypes.c_uint64)],
        "slf_profile_read": [vp, ctypes.POINTER(CProfileEntry), ctypes.c_uint32, u32p],
        "slf_profile_reset": [vp],
        "slf_kernel_launches": [u64p],
        "slf_sort_by_cell_noalloc": [vp, vp, ctypes.c_uint64, ctypes.c_float, vp, vp],
        "slf_tape_begin": [vp, ctypes.c_uint32],
        "slf_tape_end": [vp],
        "slf_step_backward": [vp, fp, fp, ctypes.c_uint64, fp, fp, ctypes.POINTER(CParamGrads)],
    }
    for name, args in sig.items():
        fn = getattr(L, name)
        fn.argtypes = args
        fn.restype = ctypes.c_int32
    L.slf_destroy.argtypes = [vp]
    L.slf_destroy.restype = None
    L.slf_last_error.argtypes = []
    L.slf_last_error.restype = ctypes.c_char_p
    _lib = L
    return L


def _check(code: int):
    if code != 0:
        msg = _lib.slf_last_error().decode(errors="replace") if _lib is not None else ""
        raise PhysicsError(code, msg)


def _ptr(a: np.ndarray, ctype):
    return a.ctypes.data_as(ctypes.POINTER(ctype))


def default_settings() -> FluidSettings:
    c = CSettings()
    _check(load_library().slf_settings_default(ctypes.byref(c)))
    return FluidSettings.from_c(c)


class FluidWorld:
    """FluidWorld (src/fluid/mod.rs:310-339) with its particles on the GPU."""

    def __init__(self, settings: FluidSettings | None = None):
        # FluidWorld::new (mod.rs:344-370)
        L = load_library()
        self._settings = settings or FluidSettings()
        c = self._settings.to_c()
        h = ctypes.c_void_p()
        _check(L.slf_create(ctypes.byref(c), ctypes.byref(h)))
        self._h = h

    new = classmethod(lambda cls, settings=None: cls(settings))

    # ---- snapshots (src/fluid/save.rs) ----
    @classmethod
    def load_snapshot(cls, data: bytes, settings: FluidSettings | None = None) -> "FluidWorld":
        """FluidWorld::load_snapshot (save.rs:79-181).  `settings` supplies only the library's
        own fields (arithmetic, positions, solver limits, device); the snapshot holds the rest."""
        L = load_library()
        buf = (ctypes.c_uint8 * max(len(data), 1)).from_buffer_copy(bytes(data) or b"\0")
        c = (settings or FluidSettings()).to_c()
        h = ctypes.c_void_p()
        _check(L.slf_load_snapshot(buf, len(data), ctypes.byref(c), ctypes.byref(h)))
        self = cls.__new__(cls)
        self._h = h
        self._settings = self.settings()
        return self

    def save_snapshot(self) -> bytes:
        """FluidWorld::save_snapshot (save.rs:18-73): SLFL version 3 bytes."""
        size = ctypes.c_uint64()
        _check(_lib.slf_save_snapshot(self._h, None, 0, ctypes.byref(size)))
        buf = (ctypes.c_uint8 * max(size.value, 1))()
        _check(_lib.slf_save_snapshot(self._h, buf, size.value, ctypes.byref(size)))
        return bytes(buf[: size.value])

    def close(self):
        h = getattr(self, "_h", None)
        if h is not None and _lib is not None:
            _lib.slf_destroy(h)
        self._h = None

    def __del__(self):
        self.close()

    @property
    def handle(self) -> ctypes.c_void_p:
        return self._h

    # ---- settings and sizes (mod.rs:372-390) ----
    def settings(self) -> FluidSettings:
        c = CSettings()
        _check(_lib.slf_get_settings(self._h, ctypes.byref(c)))
        return FluidSettings.from_c(c)

    def kernel(self):
        r, s = ctypes.c_float(), ctypes.c_float()
        _check(_lib.slf_kernel(self._h, ctypes.byref(r), ctypes.byref(s)))
        return r.value, s.value

    def particle_mass(self) -> float:
        m = ctypes.c_float()
        _check(_lib.slf_particle_mass(self._h, ctypes.byref(m)))
        return m.value

    def len(self) -> int:
        n = ctypes.c_uint64()
        _check(_lib.slf_len(self._h, ctypes.byref(n)))
        return n.value

    __len__ = len

    def is_empty(self) -> bool:
        return self.len() == 0

    # ---- particles (mod.rs:412-524) ----
    def add_particle(self, position, velocity) -> int:
        i = ctypes.c_uint32()
        _check(_lib.slf_add_particle(self._h, vec3(position), vec3(velocity), ctypes.byref(i)))
        return i.value

    def add_particles(self, positions, velocities=None) -> np.ndarray:
        p = np.ascontiguousarray(positions, dtype=np.float32).reshape(-1, 3)
        v = (np.zeros_like(p) if velocities is None
             else np.ascontiguousarray(velocities, dtype=np.float32).reshape(-1, 3))
        ids = np.zeros(len(p), dtype=np.uint32)
        _check(_lib.slf_add_particles(self._h, len(p), _ptr(p, ctypes.c_float), _ptr(v, ctypes.c_float),
                                      _ptr(ids, ctypes.c_uint32)))
        return ids

    def fill_box(self, low, high) -> int:
        n = ctypes.c_uint64()
        _check(_lib.slf_fill_box(self._h, vec3(low), vec3(high), ctypes.byref(n)))
        return n.value

    def set_domain(self, domain):
        if domain is None:
            _check(_lib.slf_set_domain(self._h, None, None))
        else:
            _check(_lib.slf_set_domain(self._h, vec3(domain[0]), vec3(domain[1])))

    # ---- walls (boundary.rs:41-120) ----
    def add_box_container(self, low, high) -> int:
        i = ctypes.c_uint32()
        _check(_lib.slf_add_box_container(self._h, vec3(low), vec3(high), ctypes.byref(i)))
        return i.value

    def add_wall(self, low, high) -> int:
        i = ctypes.c_uint32()
        _check(_lib.slf_add_wall(self._h, vec3(low), vec3(high), ctypes.byref(i)))
        return i.value

    def remove_boundary(self, boundary: int) -> bool:
        r = ctypes.c_int32()
        _check(_lib.slf_remove_boundary(self._h, boundary, ctypes.byref(r)))
        return bool(r.value)

    # ---- terrain (terrain.rs:262-302) ----
    def terrain_nodes(self, low, high):
        n = (ctypes.c_uint64 * 3)()
        _check(_lib.slf_terrain_nodes(self._h, vec3(low), vec3(high), n))
        return tuple(int(v) for v in n)

    def add_terrain(self, low, high, distances) -> int:
        """Ground under the signed distances sampled at the region's nodes (see terrain_nodes)."""
        d = np.ascontiguousarray(distances, dtype=np.float32).ravel()
        i = ctypes.c_uint32()
        _check(_lib.slf_add_terrain(self._h, vec3(low), vec3(high), _ptr(d, ctypes.c_float), d.size,
                                    ctypes.byref(i)))
        return i.value

    # ---- emitters and drains (flow.rs:86-139) ----
    def add_emitter(self, low, high, velocity) -> int:
        i = ctypes.c_uint32()
        _check(_lib.slf_add_emitter(self._h, vec3(low), vec3(high), vec3(velocity), ctypes.byref(i)))
        return i.value

    def add_drain(self, low, high) -> int:
        i = ctypes.c_uint32()
        _check(_lib.slf_add_drain(self._h, vec3(low), vec3(high), ctypes.byref(i)))
        return i.value

    def remove_flow(self, flow: int) -> bool:
        r = ctypes.c_int32()
        _check(_lib.slf_remove_flow(self._h, flow, ctypes.byref(r)))
        return bool(r.value)

    def couple(self, body: int, shape, dims):
        """FluidWorld::couple (couple.rs:165-200): body = index << 32 | generation, shape a
        `Shape`, dims its half extents, (radius,) or (radius, half height)."""
        d = list(dims) + [0.0] * (3 - len(dims))
        _check(_lib.slf_couple(self._h, body, int(shape), vec3(d)))

    def uncouple(self, body: int) -> bool:
        r = ctypes.c_int32()
        _check(_lib.slf_uncouple(self._h, body, ctypes.byref(r)))
        return bool(r.value)

    def coupled(self):
        """[(body, points, probes)] in body order."""
        n = ctypes.c_uint64()
        _check(_lib.slf_coupled(self._h, None, None, None, 0, ctypes.byref(n)))
        k = n.value
        b, p, q = (ctypes.c_uint64 * max(k, 1))(), (ctypes.c_uint32 * max(k, 1))(), (ctypes.c_uint32 * max(k, 1))()
        _check(_lib.slf_coupled(self._h, b, p, q, k, ctypes.byref(n)))
        return [(int(b[i]), int(p[i]), int(q[i])) for i in range(k)]

    def step_with_bodies(self, dt: float, poses):
        """FluidWorld::step_with_bodies (couple.rs:219-248) with the bodies where `poses` (a
        list of BodyPose) puts them: (report, [BodyPush])."""
        return step_with_bodies_call(_lib.slf_step_with_bodies, self._h, dt, list(poses), _check)

    def wall_positions(self) -> np.ndarray:
        n = ctypes.c_uint64()
        _check(_lib.slf_wall_count(self._h, ctypes.byref(n)))
        out = np.zeros((n.value, 3), dtype=np.float32)
        _check(_lib.slf_read_wall_positions(self._h, _ptr(out, ctypes.c_float), n.value))
        return out

    # ---- the step (step.rs:58-90) ----
    def step(self, dt: float) -> FluidReport:
        r = CReport()
        _check(_lib.slf_step(self._h, dt, ctypes.byref(r)))
        return FluidReport.from_c(r)

    def update_neighbors(self):
        _check(_lib.slf_update_neighbors(self._h))

    def compute_densities(self):
        _check(_lib.slf_compute_densities(self._h))

    def last_iterations(self):
        a, b = ctypes.c_uint32(), ctypes.c_uint32()
        _check(_lib.slf_last_iterations(self._h, ctypes.byref(a), ctypes.byref(b)))
        return a.value, b.value

    def debug_skip_job(self, job: int):
        _check(_lib.slf_debug_skip_job(self._h, job))

    def debug_list_room(self, room: int):
        """Test hook: shrinks the neighbour lists' room so the next substep outgrows it and runs again."""
        _check(_lib.slf_debug_list_room(self._h, room))

    # ---- read-outs (mod.rs:393-408, 612, 678) ----
    def ids(self) -> np.ndarray:
        n = self.len()
        out = np.zeros(n, dtype=np.uint32)
        _check(_lib.slf_read_ids(self._h, _ptr(out, ctypes.c_uint32), n))
        return out

    def _vecs(self, fn) -> np.ndarray:
        n = self.len()
        out = np.zeros((n, 3), dtype=np.float32)
        _check(fn(self._h, _ptr(out, ctypes.c_float), n))
        return out

    def positions(self) -> np.ndarray:
        return self._vecs(_lib.slf_read_positions)

    def velocities(self) -> np.ndarray:
        return self._vecs(_lib.slf_read_velocities)

    def densities(self) -> np.ndarray:
        n = self.len()
        out = np.zeros(n, dtype=np.float32)
        _check(_lib.slf_read_densities(self._h, _ptr(out, ctypes.c_float), n))
        return out

    def _lists(self, fn):
        total = ctypes.c_uint64()
        _check(fn(self._h, None, 0, None, 0, ctypes.byref(total)))
        start = np.zeros(self.len() + 1, dtype=np.uint32)
        items = np.zeros(max(total.value, 1), dtype=np.uint32)
        _check(fn(self._h, _ptr(start, ctypes.c_uint32), len(start), _ptr(items, ctypes.c_uint32), total.value,
                  ctypes.byref(total)))
        return start, items[: total.value]

    def neighbor_lists(self):
        """(start, items): every particle's neighbours, itself included (mod.rs:279-308)."""
        return self._lists(_lib.slf_neighbor_lists)

    def wall_neighbor_lists(self):
        return self._lists(_lib.slf_wall_neighbor_lists)

    def neighbors_of(self, index: int) -> np.ndarray:
        start, items = self.neighbor_lists()
        if index + 1 >= len(start):
            return items[:0]
        return items[start[index]:start[index + 1]]

    def state_hash(self) -> int:
        v = ctypes.c_uint64()
        _check(_lib.slf_state_hash(self._h, ctypes.byref(v)))
        return v.value

    # ---- the adjoint ----
    def tape_begin(self, checkpoint_every: int = 1):
        """Records the steps that follow for step_backward: keeps the state before every k-th
        substep as a checkpoint, or with k = 0 keeps every substep's state and solver record (no
        forward recomputation)."""
        _check(_lib.slf_tape_begin(self._h, checkpoint_every))

    def tape_end(self):
        _check(_lib.slf_tape_end(self._h))

    def step_backward(self, dpositions, dvelocities):
        """dL/d(positions, velocities at tape_begin, in their order then) and dL/d settings, from
        dL/d of the current positions and velocities (current order)."""
        n = self.len()
        dp = np.ascontiguousarray(dpositions, dtype=np.float32).reshape(n, 3)
        dv = np.ascontiguousarray(dvelocities, dtype=np.float32).reshape(n, 3)
        out_p = np.zeros((n, 3), dtype=np.float32)
        out_v = np.zeros((n, 3), dtype=np.float32)
        g = CParamGrads()
        _check(_lib.slf_step_backward(self._h, _ptr(dp, ctypes.c_float), _ptr(dv, ctypes.c_float), n,
                                      _ptr(out_p, ctypes.c_float), _ptr(out_v, ctypes.c_float), ctypes.byref(g)))
        params = {"viscosity": g.viscosity, "sound_speed": g.sound_speed, "gravity": tuple(g.gravity)}
        return out_p, out_v, params

    # ---- host-owned state, streams, profiling ----
    def write_state(self, positions, velocities):
        """Overwrites positions and velocities of the current particles (current order)."""
        p = np.ascontiguousarray(positions, dtype=np.float32).reshape(-1, 3)
        v = np.ascontiguousarray(velocities, dtype=np.float32).reshape(-1, 3)
        _check(_lib.slf_write_state(self._h, _ptr(p, ctypes.c_float), _ptr(v, ctypes.c_float), len(p)))

    def write_state_ptr(self, positions_ptr: int, velocities_ptr: int, n: int):
        """write_state from raw host pointers (pinned buffers)."""
        fp = ctypes.POINTER(ctypes.c_float)
        _check(_lib.slf_write_state(self._h, ctypes.cast(positions_ptr, fp), ctypes.cast(velocities_ptr, fp), n))

    def read_positions_ptr(self, ptr: int, n: int):
        _check(_lib.slf_read_positions(self._h, ctypes.cast(ptr, ctypes.POINTER(ctypes.c_float)), n))

    def read_velocities_ptr(self, ptr: int, n: int):
        _check(_lib.slf_read_velocities(self._h, ctypes.cast(ptr, ctypes.POINTER(ctypes.c_float)), n))

    def read_state_ptr(self, positions_ptr: int, velocities_ptr: int, n: int):
        """Positions and velocities into raw host pointers (pinned buffers), one wait."""
        fp = ctypes.POINTER(ctypes.c_float)
        _check(_lib.slf_read_state(self._h, ctypes.cast(positions_ptr, fp), ctypes.cast(velocities_ptr, fp), n))

    def stream(self) -> int:
        s = ctypes.c_void_p()
        _check(_lib.slf_get_stream(self._h, ctypes.byref(s)))
        return s.value or 0

    def profile(self, on: bool = True):
        """Times each kernel launch with CUDA events (solves then run launch by launch)."""
        _check(_lib.slf_profile_enable(self._h, 1 if on else 0))

    def solver_graphs(self, mode=2):
        """How steps launch: 2 (the default, also True) each substep as one CUDA graph,
        1 each solve as one graph whose loop the device ends, 0 (also False) solves as batches
        of launches with a host check between them; the results are identical."""
        mode = 2 if mode is True else 0 if mode is False else int(mode)
        _check(_lib.slf_solver_graphs(self._h, mode))

    def graph_substeps(self) -> int:
        """Substeps this world ran as one whole-substep graph launch."""
        out = ctypes.c_uint64(0)
        _check(_lib.slf_graph_substeps(self._h, ctypes.byref(out)))
        return out.value

    def profile_reset(self):
        _check(_lib.slf_profile_reset(self._h))

    def profile_read(self) -> dict:
        """{kernel: (launches, milliseconds, algorithmic bytes)} accumulated while profiling."""
        count = ctypes.c_uint32()
        _check(_lib.slf_profile_read(self._h, None, 0, ctypes.byref(count)))
        arr = (CProfileEntry * max(count.value, 1))()
        _check(_lib.slf_profile_read(self._h, arr, count.value, ctypes.byref(count)))
        return {arr[i].name.decode(): (arr[i].launches, arr[i].milliseconds, arr[i].algorithmic_bytes)
                for i in range(count.value)}


def kernel_launches() -> int:
    """Kernels launched through the library by this process so far."""
    v = ctypes.c_uint64()
    _check(load_library().slf_kernel_launches(ctypes.byref(v)))
    return v.value


def sort_by_cell_noalloc(positions_ptr: int, ids_ptr: int, n: int, radius: float, order_ptr: int,
                         stream: int = 0):
    """slf_sort_by_cell_noalloc on device pointers: order[k] = input index of the k-th particle
    in (cell, id) order.  For hosts that cannot allocate device memory: the library keeps this
    sort's scratch in a fixed device array and allocates nothing."""
    L = load_library()
    _check(L.slf_sort_by_cell_noalloc(ctypes.c_void_p(positions_ptr), ctypes.c_void_p(ids_ptr), n, radius,
                                      ctypes.c_void_p(order_ptr), ctypes.c_void_p(stream)))
