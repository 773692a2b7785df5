"""Python binding of the B200 WCSPH C ABI (include/vxl_sph.h) through ctypes.

This is the same thin binding a maintainer would add on the caller's side; the
reference's own caller is Rust (a `FluidStepper` impl over the C ABI: the crate under
rust-wl_b200/rust/vxl-phys-gpu-b200). `GpuFluidStepper` and `PhysGpuBackend` mirror the reference's trait
methods (crates/vxl-phys-core/src/interop.rs:293-316, crates/vxl-phys-gpu/src/lib.rs:20-29)
so tests read like the reference's own.

The library is built in-tree (rust-wl_b200/lib/libvxl_sph.so). There is no CPU
fallback: if the library is missing or no sm_100 device is present, calls raise.
"""
from __future__ import annotations

import ctypes as C
import os
from dataclasses import dataclass
from pathlib import Path

import numpy as np

PKG_DIR = Path(__file__).resolve().parent.parent
LIB_PATH = PKG_DIR / "lib" / "libvxl_sph.so"
ABI_VERSION = 1

OK, NULL_POINTER, VERSION_MISMATCH, SIZE_MISMATCH, NOT_READY, PANIC_CAUGHT = range(6)
INVALID_ARGUMENT, CUDA_ERROR, OUT_OF_MEMORY, DEVICE_FAULT_FLAG = range(6, 10)
STATUS_NAMES = {
    0: "Ok", 1: "NullPointer", 2: "VersionMismatch", 3: "SizeMismatch", 4: "NotReady",
    5: "PanicCaught", 6: "InvalidArgument", 7: "CudaError", 8: "OutOfMemory", 9: "DeviceFaultFlag",
}


class VxlError(RuntimeError):
    def __init__(self, status: int, msg: str):
        super().__init__(f"{STATUS_NAMES.get(status, status)}: {msg}")
        self.status = status


class BlockHeader(C.Structure):
    _fields_ = [("size", C.c_uint32), ("version", C.c_uint32)]


class Params(C.Structure):
    _fields_ = [
        ("hdr", BlockHeader),
        ("rest_density", C.c_float),
        ("smoothing_radius", C.c_float),
        ("xsph_viscosity", C.c_float),
        ("tensile_instability_suppression", C.c_uint32),
        ("sound_speed", C.c_float),
        ("gamma_tait", C.c_float),
        ("substeps", C.c_uint32),
        ("boundary_layers", C.c_uint32),
        ("gravity", C.c_float * 3),
        ("max_speed_frac", C.c_float),
        ("artificial_viscosity", C.c_float),
        ("particle_mass", C.c_float),
        ("max_bins", C.c_uint32),
    ]


class Desc(C.Structure):
    _fields_ = [
        ("hdr", BlockHeader),
        ("params", Params),
        ("n_fluid", C.c_uint64),
        ("n_boundary", C.c_uint64),
        ("pos_xyz", C.POINTER(C.c_float)),
        ("vel_xyz", C.POINTER(C.c_float)),
        ("pmass", C.POINTER(C.c_float)),
        ("device", C.c_int32),
    ]


class Span(C.Structure):
    _fields_ = [("body", C.c_uint32), ("origin", C.c_float * 3), ("start", C.c_uint32), ("end", C.c_uint32)]


class Reaction(C.Structure):
    _fields_ = [("body", C.c_uint32), ("force", C.c_float * 3), ("torque", C.c_float * 3)]


class GridInfo(C.Structure):
    _fields_ = [
        ("hdr", BlockHeader),
        ("min", C.c_float * 3),
        ("inv", C.c_float),
        ("bin", C.c_float),
        ("dims", C.c_uint32 * 3),
        ("total", C.c_uint64),
    ]


class Stats(C.Structure):
    _fields_ = [
        ("hdr", BlockHeader),
        ("n_fluid", C.c_uint64),
        ("n_boundary", C.c_uint64),
        ("cells", C.c_uint64),
        ("launches_last_tick", C.c_uint64),
        ("device_bytes", C.c_uint64),
        ("last_tick_ms", C.c_float),
    ]


class Tuning(C.Structure):
    _fields_ = [("hdr", BlockHeader), ("block", C.c_uint32), ("tile", C.c_uint32), ("waves", C.c_uint32),
                ("density", C.c_uint32), ("ms_per_substep", C.c_float)]


class RequestStatus(C.Structure):
    _fields_ = [("hdr", BlockHeader), ("state", C.c_uint32), ("ticks_done", C.c_uint32),
                ("ticks_total", C.c_uint32), ("pad", C.c_uint32), ("submit_s", C.c_double), ("admit_s", C.c_double),
                ("done_s", C.c_double), ("tick_p50_ms", C.c_double), ("tick_p99_ms", C.c_double)]


class ServeReport(C.Structure):
    _fields_ = [("hdr", BlockHeader), ("active", C.c_uint32), ("queued", C.c_uint32), ("admitted", C.c_uint32),
                ("retired", C.c_uint32), ("particles", C.c_uint64), ("device_bytes_in_use", C.c_uint64)]


class BodyPose(C.Structure):
    _fields_ = [("body", C.c_uint32), ("pos", C.c_float * 3), ("rot", C.c_float * 4), ("linvel", C.c_float * 3),
                ("angvel", C.c_float * 3)]


class RigidBody(C.Structure):
    _fields_ = [("pose", BodyPose), ("inv_mass", C.c_float), ("local_inv_inertia", C.c_float * 3),
                ("dynamic", C.c_uint32)]


class WallPlane(C.Structure):
    _fields_ = [("normal", C.c_float * 3), ("offset", C.c_float), ("axis", C.c_uint32), ("sign", C.c_float)]


class Provider(C.Structure):
    _fields_ = [("kind", C.c_uint32), ("first_plane", C.c_uint32), ("nplanes", C.c_uint32),
                ("has_bounds", C.c_uint32), ("bounds_min", C.c_float * 3), ("bounds_max", C.c_float * 3)]


PROVIDER_FACES, PROVIDER_CONVEX = 0, 1


@dataclass
class Faces:
    """Independent axis-aligned half-space faces (axis, plane, sign): solid where
    (p[axis] - plane) * sign < 0; bounds ((min xyz), (max xyz)) or None."""
    faces: list
    bounds: tuple | None = None


@dataclass
class Convex:
    """Convex solid {x : n . x <= d for every (n, d) in planes}; bounds or None."""
    planes: list
    bounds: tuple | None = None


def providers_arrays(providers):
    """(Provider array, n, WallPlane array, nplanes) for a list of Faces / Convex."""
    planes = []
    recs = []
    for pr in providers:
        first = len(planes)
        if isinstance(pr, Faces):
            for axis, plane, sign in pr.faces:
                planes.append(((0.0, 0.0, 0.0), plane, axis, sign))
            kind = PROVIDER_FACES
        else:
            for n, d in pr.planes:
                planes.append((tuple(n), d, 0, 1.0))
            kind = PROVIDER_CONVEX
        recs.append((kind, first, len(planes) - first, pr.bounds))
    parr = (Provider * max(len(recs), 1))()
    for q, (kind, first, cnt, b) in enumerate(recs):
        parr[q].kind, parr[q].first_plane, parr[q].nplanes = kind, first, cnt
        parr[q].has_bounds = 0 if b is None else 1
        if b is not None:
            for a in range(3):
                parr[q].bounds_min[a] = b[0][a]
                parr[q].bounds_max[a] = b[1][a]
    warr = (WallPlane * max(len(planes), 1))()
    for k, (n, d, axis, sign) in enumerate(planes):
        for a in range(3):
            warr[k].normal[a] = n[a]
        warr[k].offset, warr[k].axis, warr[k].sign = d, axis, sign
    return parr, len(recs), warr, len(planes)


def poses_array(bodies):
    """BodyPose array from objects with id, pos, rot, linvel, angvel (e.g. scenes.Body)."""
    arr = (BodyPose * max(len(bodies), 1))()
    for q, b in enumerate(bodies):
        arr[q].body = b.id
        for a in range(3):
            arr[q].pos[a] = b.pos[a]
            arr[q].linvel[a] = b.linvel[a]
            arr[q].angvel[a] = b.angvel[a]
        for a in range(4):
            arr[q].rot[a] = b.rot[a]
    return arr, len(bodies)


def header(struct_type) -> BlockHeader:
    return BlockHeader(C.sizeof(struct_type), ABI_VERSION)


# Every symbol include/vxl_sph.h declares, with its ctypes signature.
_FP = C.POINTER(C.c_float)
_U32P = C.POINTER(C.c_uint32)
_H = C.c_void_p
SIGNATURES = {
    "vxl_sph_abi_version": (C.c_uint32, []),
    "vxl_sph_last_error": (C.c_char_p, []),
    "vxl_sph_backend_name": (C.c_char_p, []),
    "vxl_sph_backend_available": (C.c_int, []),
    "vxl_sph_lattice_mass": (C.c_int, [C.POINTER(Params), C.c_float, _FP]),
    "vxl_sph_boundary_lattice": (C.c_int, [C.c_uint32, _FP, C.c_float, C.c_float, C.c_float, C.c_uint32, _FP,
                                           C.c_uint64, C.POINTER(C.c_uint64), _FP]),
    "vxl_sph_create": (C.c_int, [C.POINTER(Desc), C.POINTER(_H)]),
    "vxl_sph_destroy": (C.c_int, [_H]),
    "vxl_sph_upload_boundary": (C.c_int, [_H, C.c_uint64, _FP, _FP, C.c_uint64]),
    "vxl_sph_step_tick": (C.c_int, [_H, C.c_float, C.POINTER(Span), C.c_uint32, C.POINTER(Reaction)]),
    "vxl_sph_step_tick_async": (C.c_int, [_H, C.c_float, C.POINTER(Span), C.c_uint32]),
    "vxl_sph_sync": (C.c_int, [_H, C.POINTER(Reaction), C.c_uint32]),
    "vxl_sph_substep": (C.c_int, [_H, C.c_float]),
    "vxl_sph_bounds": (C.c_int, [_H, _FP, _FP]),
    "vxl_sph_read_state": (C.c_int, [_H, _FP, _FP]),
    "vxl_sph_write_state": (C.c_int, [_H, _FP, _FP]),
    "vxl_sph_set_record": (C.c_int, [_H, C.c_int]),
    "vxl_sph_read_fields": (C.c_int, [_H, _FP, _FP, _FP, _FP, _FP]),
    "vxl_sph_export_grid": (C.c_int, [_H, _U32P, _U32P, C.c_uint64, _U32P, C.POINTER(GridInfo)]),
    "vxl_sph_get_stats": (C.c_int, [_H, C.POINTER(Stats)]),
    "vxl_sph_set_stream": (C.c_int, [_H, C.c_void_p]),
    "vxl_sph_set_profile": (C.c_int, [_H, C.c_int]),
    "vxl_sph_serve_set_batch_cap": (C.c_int, [C.c_void_p, C.c_uint64]),
    "vxl_sph_set_wall_contacts": (C.c_int, [_H, C.c_uint32, C.c_uint32, _U32P, _U32P, C.c_uint32, _FP,
                                            C.c_uint32]),
    "vxl_sph_export_neighbors": (C.c_int, [_H, C.POINTER(C.c_uint64), C.c_uint64, _U32P, C.c_uint64,
                                           C.POINTER(C.c_uint64)]),
    "vxl_sph_profile_read": (C.c_int, [_H, C.c_uint32, C.POINTER(C.c_char_p), C.POINTER(C.c_double),
                                       C.POINTER(C.c_uint64)]),
    "vxl_sph_build_grid_static": (C.c_int, [C.c_void_p, C.c_uint32, C.c_float, C.c_uint32, C.c_void_p, C.c_void_p,
                                            C.c_uint64, C.POINTER(GridInfo), C.c_void_p]),
    "vxl_sph_create_batch": (C.c_int, [C.POINTER(Desc), C.c_uint32, C.c_int32, C.c_uint64, C.POINTER(_H)]),
    "vxl_sph_scene_count": (C.c_uint32, [_H]),
    "vxl_sph_read_state_scene": (C.c_int, [_H, C.c_uint32, _FP, _FP]),
    "vxl_sph_write_state_scene": (C.c_int, [_H, C.c_uint32, _FP, _FP]),
    "vxl_sph_upload_boundary_scene": (C.c_int, [_H, C.c_uint32, _FP, _FP, C.c_uint64]),
    "vxl_sph_set_spans_scene": (C.c_int, [_H, C.c_uint32, C.POINTER(Span), C.c_uint32]),
    "vxl_sph_export_grid_scene": (C.c_int, [_H, C.c_uint32, _U32P, _U32P, C.c_uint64, _U32P, C.POINTER(GridInfo)]),
    "vxl_sph_read_fields_scene": (C.c_int, [_H, C.c_uint32, _FP, _FP, _FP, _FP, _FP]),
    "vxl_sph_reactions_all": (C.c_int, [_H, C.POINTER(Reaction), C.c_uint32, C.POINTER(C.c_uint32)]),
    "vxl_sph_set_tuning": (C.c_int, [_H, C.POINTER(Tuning)]),
    "vxl_sph_get_tuning": (C.c_int, [_H, C.POINTER(Tuning)]),
    "vxl_sph_autotune": (C.c_int, [_H, C.c_float, C.c_uint32, C.POINTER(Tuning)]),
    "vxl_sph_request_state": (C.c_int, [_H]),
    "vxl_sph_take_state": (C.c_int, [_H, _FP, C.c_uint64]),
    "vxl_sph_set_rigid_bodies": (C.c_int, [_H, C.c_uint32, C.POINTER(RigidBody), C.c_uint32]),
    "vxl_sph_set_providers": (C.c_int, [_H, C.c_uint32, C.POINTER(Provider), C.c_uint32, C.POINTER(WallPlane),
                                        C.c_uint32]),
    "vxl_sph_step_coupled": (C.c_int, [_H, C.c_float, C.c_uint32, _FP, C.c_float, C.c_float, C.POINTER(Reaction),
                                       C.c_uint32]),
    "vxl_sph_read_rigid_bodies": (C.c_int, [_H, C.c_uint32, C.POINTER(RigidBody), C.c_uint32]),
    "vxl_sph_set_body_lattice": (C.c_int, [_H, C.c_uint32, _FP, C.POINTER(C.c_uint32), C.c_uint64, C.c_uint32]),
    "vxl_sph_set_body_poses": (C.c_int, [_H, C.c_uint32, C.POINTER(BodyPose), C.c_uint32]),
    "vxl_sph_serve_create": (C.c_int, [C.c_int32, C.c_uint64, C.c_uint32, C.POINTER(C.c_void_p)]),
    "vxl_sph_serve_destroy": (C.c_int, [C.c_void_p]),
    "vxl_sph_serve_submit": (C.c_int, [C.c_void_p, C.POINTER(Desc), C.c_uint32, C.POINTER(C.c_uint64)]),
    "vxl_sph_serve_step": (C.c_int, [C.c_void_p, C.c_float, C.POINTER(ServeReport)]),
    "vxl_sph_serve_poll": (C.c_int, [C.c_void_p, C.c_uint64, C.POINTER(RequestStatus)]),
    "vxl_sph_serve_read": (C.c_int, [C.c_void_p, C.c_uint64, _FP, _FP]),
    "vxl_sph_serve_tick_times": (C.c_int, [C.c_void_p, C.c_uint64, C.POINTER(C.c_double), C.c_uint32,
                                           C.POINTER(C.c_uint32)]),
}

_lib = None


def load(path: str | os.PathLike | None = None) -> C.CDLL:
    """Load the in-tree library (raises if it is missing: there is no fallback)."""
    global _lib
    if _lib is not None and path is None:
        return _lib
    p = Path(path) if path else LIB_PATH
    if not p.exists():
        raise FileNotFoundError(f"{p} not built (run rust-wl_b200/build.py)")
    lib = C.CDLL(str(p))
    for name, (res, args) in SIGNATURES.items():
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    if lib.vxl_sph_abi_version() != ABI_VERSION:
        raise VxlError(VERSION_MISMATCH, "library ABI version differs from the binding")
    if path is None:
        _lib = lib
    return lib


def _check(status: int) -> None:
    if status != OK:
        msg = load().vxl_sph_last_error()
        raise VxlError(status, msg.decode() if msg else "")


def _fptr(a: np.ndarray | None):
    if a is None:
        return None
    assert a.dtype == np.float32 and a.flags.c_contiguous
    return a.ctypes.data_as(_FP)


def _u32ptr(a: np.ndarray | None):
    if a is None:
        return None
    assert a.dtype == np.uint32 and a.flags.c_contiguous
    return a.ctypes.data_as(_U32P)


def make_params(*, rest_density=1000.0, smoothing_radius=0.1, xsph_viscosity=0.1, tensile_instability_suppression=True,
                sound_speed=10.0, gamma_tait=7.0, substeps=4, boundary_layers=2, gravity=(0.0, -9.81, 0.0),
                max_speed_frac=0.4, artificial_viscosity=1.0, particle_mass=0.0, max_bins=0) -> Params:
    """Params with the reference's FluidConfig defaults (crates/vxl-phys-fluid/src/config.rs:47-68)."""
    p = Params()
    p.hdr = header(Params)
    p.rest_density = rest_density
    p.smoothing_radius = smoothing_radius
    p.xsph_viscosity = xsph_viscosity
    p.tensile_instability_suppression = 1 if tensile_instability_suppression else 0
    p.sound_speed = sound_speed
    p.gamma_tait = gamma_tait
    p.substeps = substeps
    p.boundary_layers = boundary_layers
    for a in range(3):
        p.gravity[a] = gravity[a]
    p.max_speed_frac = max_speed_frac
    p.artificial_viscosity = artificial_viscosity
    p.particle_mass = particle_mass
    p.max_bins = max_bins
    return p


def lattice_mass(params: Params, spacing: float) -> float:
    out = C.c_float()
    _check(load().vxl_sph_lattice_mass(C.byref(params), spacing, C.byref(out)))
    return out.value


def boundary_lattice(shape: int, half=(0.0, 0.0, 0.0), radius: float = 0.0, spacing: float = 0.05, h: float = 0.1,
                     layers: int = 2) -> tuple[np.ndarray, float]:
    """Body-space Akinci lattice (N, 3) float32 and per-particle volume."""
    lib = load()
    hv = np.asarray(half, dtype=np.float32)
    n = C.c_uint64()
    vol = C.c_float()
    _check(lib.vxl_sph_boundary_lattice(shape, _fptr(hv), radius, spacing, h, layers, None, 0, C.byref(n), None))
    pts = np.zeros((n.value, 3), dtype=np.float32)
    _check(lib.vxl_sph_boundary_lattice(shape, _fptr(hv), radius, spacing, h, layers, _fptr(pts), n.value,
                                        C.byref(n), C.byref(vol)))
    return pts, vol.value


def spans_array(spans) -> tuple:
    arr = (Span * max(len(spans), 1))()
    for q, (body, origin, start, end) in enumerate(spans):
        arr[q].body = body
        for a in range(3):
            arr[q].origin[a] = origin[a]
        arr[q].start = start
        arr[q].end = end
    return arr, len(spans)


class Scene:
    """A resident scene on one GPU (handle of the C ABI)."""

    def __init__(self, params: Params, pos: np.ndarray, vel: np.ndarray, pmass: np.ndarray, n_fluid: int,
                 device: int = 0):
        lib = load()
        pos = np.ascontiguousarray(pos, dtype=np.float32).reshape(-1, 3)
        vel = np.ascontiguousarray(vel, dtype=np.float32).reshape(-1, 3)
        pmass = np.ascontiguousarray(pmass, dtype=np.float32).reshape(-1)
        n = pos.shape[0]
        if params.particle_mass == 0.0 and n_fluid > 0:
            params.particle_mass = float(pmass[0])
        d = Desc()
        d.hdr = header(Desc)
        d.params = params
        d.n_fluid = n_fluid
        d.n_boundary = n - n_fluid
        d.pos_xyz = _fptr(pos)
        d.vel_xyz = _fptr(vel)
        d.pmass = _fptr(pmass)
        d.device = device
        h = C.c_void_p()
        _check(lib.vxl_sph_create(C.byref(d), C.byref(h)))
        self._h = h
        self.lib = lib
        self.n_fluid = n_fluid
        self.n_total = n
        self.n_boundary = n - n_fluid
        self.params = params

    def close(self) -> None:
        if getattr(self, "_h", None):
            _check(self.lib.vxl_sph_destroy(self._h))
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def step_tick(self, dt_tick: float, spans=()) -> list[tuple[int, np.ndarray, np.ndarray]]:
        arr, ns = spans_array(spans)
        out = (Reaction * max(ns, 1))()
        _check(self.lib.vxl_sph_step_tick(self._h, dt_tick, arr, ns, out))
        return [(out[q].body, np.array(out[q].force[:], np.float32), np.array(out[q].torque[:], np.float32))
                for q in range(ns)]

    def step_tick_async(self, dt_tick: float, spans=()) -> None:
        arr, ns = spans_array(spans)
        self._async_spans = ns
        _check(self.lib.vxl_sph_step_tick_async(self._h, dt_tick, arr, ns))

    def sync(self):
        ns = getattr(self, "_async_spans", 0)
        out = (Reaction * max(ns, 1))()
        _check(self.lib.vxl_sph_sync(self._h, out, ns))
        return [(out[q].body, np.array(out[q].force[:], np.float32), np.array(out[q].torque[:], np.float32))
                for q in range(ns)]

    def substep(self, dt: float) -> None:
        _check(self.lib.vxl_sph_substep(self._h, dt))

    def upload_boundary(self, pos: np.ndarray, vel: np.ndarray) -> None:
        pos = np.ascontiguousarray(pos, dtype=np.float32).reshape(-1, 3)
        vel = np.ascontiguousarray(vel, dtype=np.float32).reshape(-1, 3)
        _check(self.lib.vxl_sph_upload_boundary(self._h, self.n_fluid, _fptr(pos), _fptr(vel), pos.shape[0]))

    def request_state(self) -> None:
        """Enqueue a copy of every position after the work already enqueued; returns at once."""
        _check(self.lib.vxl_sph_request_state(self._h))

    def take_state(self, out: np.ndarray | None = None) -> np.ndarray:
        """Wait for the requested copy; positions (N, 3) in reference order."""
        p = np.empty((self.n_total, 3), np.float32) if out is None else out
        _check(self.lib.vxl_sph_take_state(self._h, _fptr(p), p.shape[0]))
        return p

    def set_body_lattice(self, local_xyz: np.ndarray, body_index: np.ndarray, nbodies: int, scene: int = 0) -> None:
        """Body-frame lattice of the boundary segment (see scenes.body_lattice)."""
        lx = np.ascontiguousarray(local_xyz, dtype=np.float32).reshape(-1, 3)
        bi = np.ascontiguousarray(body_index, dtype=np.uint32).reshape(-1)
        _check(self.lib.vxl_sph_set_body_lattice(self._h, scene, _fptr(lx), _u32ptr(bi), lx.shape[0], nbodies))

    def set_body_poses(self, bodies, scene: int = 0) -> None:
        """Rebuild the boundary segment on the device from the bodies' poses."""
        arr, n = poses_array(bodies)
        _check(self.lib.vxl_sph_set_body_poses(self._h, scene, arr, n))

    def set_providers(self, providers, scene: int = 0) -> None:
        """Provider walls (a list of Faces / Convex, in the fluid's boundaries order)."""
        parr, n, warr, nw = providers_arrays(providers)
        _check(self.lib.vxl_sph_set_providers(self._h, scene, parr, n, warr, nw))

    def set_wall_contacts(self, side: int, ids, start, planes, scene: int = 0) -> None:
        """One side (0 mirror, 1 projection) of the scene's contact tables (vxl_sph_set_wall_contacts)."""
        ids = np.ascontiguousarray(ids, np.uint32)
        start = np.ascontiguousarray(start, np.uint32)
        planes = np.ascontiguousarray(planes, np.float32).reshape(-1, 6)
        n = ids.shape[0]
        _check(self.lib.vxl_sph_set_wall_contacts(self._h, scene, side, _u32ptr(ids) if n else None,
                                                  _u32ptr(start) if n else None, n,
                                                  _fptr(planes) if planes.shape[0] else None, planes.shape[0]))

    def set_spans(self, spans, scene: int = 0) -> None:
        """Spans for ticks that take none (vxl_sph_step_coupled)."""
        arr, n = spans_array(spans)
        _check(self.lib.vxl_sph_set_spans_scene(self._h, scene, arr, n))

    def set_rigid_bodies(self, bodies, inv_mass, local_inv_inertia, dynamic, scene: int = 0) -> None:
        """The lattice bodies as rigid bodies: poses from `bodies` (id, pos, rot, linvel,
        angvel), mass properties and dynamic flags per body."""
        arr = (RigidBody * max(len(bodies), 1))()
        poses, _ = poses_array(bodies)
        for q in range(len(bodies)):
            arr[q].pose = poses[q]
            arr[q].inv_mass = float(inv_mass[q])
            for a in range(3):
                arr[q].local_inv_inertia[a] = float(local_inv_inertia[q][a])
            arr[q].dynamic = 1 if dynamic[q] else 0
        _check(self.lib.vxl_sph_set_rigid_bodies(self._h, scene, arr, len(bodies)))
        self._rigid_n = getattr(self, "_rigid_n", {})
        self._rigid_n[scene] = len(bodies)

    def step_coupled(self, dt_tick: float, rigid_substeps: int = 2, gravity=(0.0, -9.81, 0.0),
                     max_linear: float = 100.0, max_angular: float = 50.0, nspans: int = 0):
        g = np.ascontiguousarray(gravity, dtype=np.float32)
        out = (Reaction * max(nspans, 1))()
        _check(self.lib.vxl_sph_step_coupled(self._h, dt_tick, rigid_substeps, _fptr(g), max_linear, max_angular,
                                             out, nspans))
        return [(out[q].body, np.array(out[q].force[:], np.float32), np.array(out[q].torque[:], np.float32))
                for q in range(nspans)]

    def read_rigid_bodies(self, scene: int = 0) -> np.ndarray:
        """(n, 13) float32: pos xyz, rot xyzw, linvel xyz, angvel xyz."""
        n = self._rigid_n[scene]
        arr = (RigidBody * max(n, 1))()
        _check(self.lib.vxl_sph_read_rigid_bodies(self._h, scene, arr, n))
        out = np.empty((n, 13), np.float32)
        for q in range(n):
            p = arr[q].pose
            out[q] = list(p.pos) + list(p.rot) + list(p.linvel) + list(p.angvel)
        return out

    def read_state(self, out=None) -> tuple[np.ndarray, np.ndarray]:
        """Positions and velocities in reference order; `out=(pos, vel)` reuses caller
        buffers (e.g. pinned host memory)."""
        if out is None:
            p = np.empty((self.n_total, 3), np.float32)
            v = np.empty((self.n_total, 3), np.float32)
        else:
            p, v = out
        _check(self.lib.vxl_sph_read_state(self._h, _fptr(p), _fptr(v)))
        return p, v

    def write_state(self, pos: np.ndarray | None, vel: np.ndarray | None) -> None:
        pp = None if pos is None else np.ascontiguousarray(pos, dtype=np.float32).reshape(-1, 3)
        vv = None if vel is None else np.ascontiguousarray(vel, dtype=np.float32).reshape(-1, 3)
        _check(self.lib.vxl_sph_write_state(self._h, _fptr(pp), _fptr(vv)))

    def set_record(self, on: bool) -> None:
        _check(self.lib.vxl_sph_set_record(self._h, 1 if on else 0))

    def read_fields(self, acc: bool = True):
        n = self.n_total
        dens = np.empty(n, np.float32)
        press = np.empty(n, np.float32)
        a = np.empty((n, 3), np.float32) if acc else None
        x = np.empty((n, 3), np.float32) if acc else None
        bf = np.empty((max(self.n_boundary, 0), 3), np.float32)
        _check(self.lib.vxl_sph_read_fields(self._h, _fptr(dens), _fptr(press), _fptr(a), _fptr(x),
                                            _fptr(bf) if self.n_boundary else None))
        return dens, press, a, x, bf

    def export_grid(self):
        info = GridInfo()
        info.hdr = header(GridInfo)
        _check(self.lib.vxl_sph_export_grid(self._h, None, None, 0, None, C.byref(info)))
        total = info.total
        items = np.empty(self.n_total, np.uint32)
        start = np.empty(total + 1, np.uint32)
        bins = np.empty(self.n_total, np.uint32)
        _check(self.lib.vxl_sph_export_grid(self._h, _u32ptr(items), _u32ptr(start), total + 1, _u32ptr(bins),
                                            C.byref(info)))
        return items, start, bins, info

    def export_neighbors(self):
        """The last substep's neighbour lists in reference index order, as CSR
        (offsets (n_total + 1,) uint64, entries uint32; vxl_sph_export_neighbors)."""
        n = self.n_fluid + self.n_boundary
        offs = np.empty(n + 1, np.uint64)
        tot = C.c_uint64()
        op = offs.ctypes.data_as(C.POINTER(C.c_uint64))
        _check(self.lib.vxl_sph_export_neighbors(self._h, op, n + 1, None, 0, C.byref(tot)))
        ent = np.empty(max(tot.value, 1), np.uint32)
        _check(self.lib.vxl_sph_export_neighbors(self._h, op, n + 1, _u32ptr(ent), tot.value, C.byref(tot)))
        return offs, ent[:tot.value]

    def bounds(self):
        lo = np.empty(3, np.float32)
        hi = np.empty(3, np.float32)
        _check(self.lib.vxl_sph_bounds(self._h, _fptr(lo), _fptr(hi)))
        return lo, hi

    def set_stream(self, stream_handle: int | None) -> None:
        """Enqueue on a caller-owned cudaStream_t (e.g. torch.cuda.Stream().cuda_stream)."""
        _check(self.lib.vxl_sph_set_stream(self._h, C.c_void_p(stream_handle or 0)))

    def set_profile(self, on: bool) -> None:
        _check(self.lib.vxl_sph_set_profile(self._h, 1 if on else 0))

    def profile(self) -> dict:
        """{kernel name: (total device ms, launches)} since profiling was switched on."""
        out = {}
        k = 0
        while True:
            name = C.c_char_p()
            ms = C.c_double()
            n = C.c_uint64()
            st = self.lib.vxl_sph_profile_read(self._h, k, C.byref(name), C.byref(ms), C.byref(n))
            if st == INVALID_ARGUMENT:
                break
            _check(st)
            out[name.value.decode()] = (ms.value, n.value)
            k += 1
        return out

    def stats(self) -> Stats:
        s = Stats()
        s.hdr = header(Stats)
        _check(self.lib.vxl_sph_get_stats(self._h, C.byref(s)))
        return s


def _desc_of(params: Params, pos, vel, pmass, n_fluid: int, device: int = 0, keep: list | None = None) -> Desc:
    pos = np.ascontiguousarray(pos, dtype=np.float32).reshape(-1, 3)
    vel = np.ascontiguousarray(vel, dtype=np.float32).reshape(-1, 3)
    pmass = np.ascontiguousarray(pmass, dtype=np.float32).reshape(-1)
    if params.particle_mass == 0.0 and n_fluid > 0:
        params.particle_mass = float(pmass[0])
    d = Desc()
    d.hdr = header(Desc)
    d.params = params
    d.n_fluid = n_fluid
    d.n_boundary = pos.shape[0] - n_fluid
    d.pos_xyz = _fptr(pos)
    d.vel_xyz = _fptr(vel)
    d.pmass = _fptr(pmass)
    d.device = device
    if keep is not None:
        keep.extend([pos, vel, pmass])
    return d


class Batch:
    """Many independent scenes in one handle (the batched form): stepped together, one
    launch per kernel per substep for all scenes."""

    def __init__(self, specs, device: int = 0, cell_capacity: int = 0):
        lib = load()
        keep: list = []
        arr = (Desc * len(specs))()
        for i, sp in enumerate(specs):
            arr[i] = _desc_of(sp.params, sp.pos, sp.vel, sp.pmass, sp.n_fluid, device, keep)
        h = C.c_void_p()
        _check(lib.vxl_sph_create_batch(arr, len(specs), device, cell_capacity, C.byref(h)))
        self._h = h
        self.lib = lib
        self.specs = list(specs)
        self.n_total = sum(sp.n_total for sp in specs)
        for q, sp in enumerate(specs):
            if sp.spans:
                a, n = spans_array(sp.spans)  # scene-local particle indices
                _check(lib.vxl_sph_set_spans_scene(h, q, a, n))

    def close(self):
        if getattr(self, "_h", None):
            _check(self.lib.vxl_sph_destroy(self._h))
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    @property
    def n_scenes(self) -> int:
        return int(self.lib.vxl_sph_scene_count(self._h))

    def step_tick(self, dt_tick: float):
        _check(self.lib.vxl_sph_step_tick(self._h, dt_tick, None, 0, None))
        return self.reactions()

    def step_tick_async(self, dt_tick: float):
        _check(self.lib.vxl_sph_step_tick_async(self._h, dt_tick, None, 0))

    def sync(self):
        _check(self.lib.vxl_sph_sync(self._h, None, 0))

    def reactions(self):
        n = C.c_uint32()
        _check(self.lib.vxl_sph_reactions_all(self._h, None, 0, C.byref(n)))
        out = (Reaction * max(n.value, 1))()
        _check(self.lib.vxl_sph_reactions_all(self._h, out, n.value, C.byref(n)))
        return [(out[q].body, np.array(out[q].force[:], np.float32), np.array(out[q].torque[:], np.float32))
                for q in range(n.value)]

    def substep(self, dt: float):
        _check(self.lib.vxl_sph_substep(self._h, dt))

    def read_state(self, scene: int):
        n = self.specs[scene].n_total
        p = np.empty((n, 3), np.float32)
        v = np.empty((n, 3), np.float32)
        _check(self.lib.vxl_sph_read_state_scene(self._h, scene, _fptr(p), _fptr(v)))
        return p, v

    def write_state(self, scene: int, pos, vel):
        pp = None if pos is None else np.ascontiguousarray(pos, dtype=np.float32).reshape(-1, 3)
        vv = None if vel is None else np.ascontiguousarray(vel, dtype=np.float32).reshape(-1, 3)
        _check(self.lib.vxl_sph_write_state_scene(self._h, scene, _fptr(pp), _fptr(vv)))

    def export_grid(self, scene: int):
        info = GridInfo()
        info.hdr = header(GridInfo)
        _check(self.lib.vxl_sph_export_grid_scene(self._h, scene, None, None, 0, None, C.byref(info)))
        n = self.specs[scene].n_total
        items = np.empty(n, np.uint32)
        start = np.empty(info.total + 1, np.uint32)
        bins = np.empty(n, np.uint32)
        _check(self.lib.vxl_sph_export_grid_scene(self._h, scene, _u32ptr(items), _u32ptr(start), info.total + 1,
                                                  _u32ptr(bins), C.byref(info)))
        return items, start, bins, info

    def set_tuning(self, block: int, tile: int, waves: int = 0, density: int | None = None):
        """Launch shape; density 0 (per-particle walk) or 1 (grouped segments), None keeps it."""
        t = Tuning()
        t.hdr = header(Tuning)
        if density is None:
            _check(self.lib.vxl_sph_get_tuning(self._h, C.byref(t)))
        t.block, t.tile, t.waves = block, tile, waves
        if density is not None:
            t.density = density
        _check(self.lib.vxl_sph_set_tuning(self._h, C.byref(t)))

    def tuning(self):
        t = Tuning()
        t.hdr = header(Tuning)
        _check(self.lib.vxl_sph_get_tuning(self._h, C.byref(t)))
        return t.block, t.tile, t.waves, t.density

    def autotune(self, dt_tick: float, trials: int = 3):
        t = Tuning()
        t.hdr = header(Tuning)
        _check(self.lib.vxl_sph_autotune(self._h, dt_tick, trials, C.byref(t)))
        return {"block": t.block, "tile": t.tile, "waves": t.waves, "density": ["walk", "grouped"][t.density],
                "ms_per_substep": t.ms_per_substep}

    def set_stream(self, stream_handle: int | None) -> None:
        _check(self.lib.vxl_sph_set_stream(self._h, C.c_void_p(stream_handle or 0)))

    def set_profile(self, on: bool) -> None:
        _check(self.lib.vxl_sph_set_profile(self._h, 1 if on else 0))

    profile = Scene.profile
    request_state = Scene.request_state
    take_state = Scene.take_state
    set_providers = Scene.set_providers
    set_body_lattice = Scene.set_body_lattice
    set_body_poses = Scene.set_body_poses
    set_spans = Scene.set_spans
    set_rigid_bodies = Scene.set_rigid_bodies
    step_coupled = Scene.step_coupled
    read_rigid_bodies = Scene.read_rigid_bodies

    def stats(self) -> Stats:
        s = Stats()
        s.hdr = header(Stats)
        _check(self.lib.vxl_sph_get_stats(self._h, C.byref(s)))
        return s


class Server:
    """The served form: a request loop with continuous batching under an HBM budget."""

    QUEUED, RUNNING, DONE, REJECTED = range(4)

    def __init__(self, budget_bytes: int, device: int = 0, max_scenes: int = 4096):
        lib = load()
        h = C.c_void_p()
        _check(lib.vxl_sph_serve_create(device, budget_bytes, max_scenes, C.byref(h)))
        self._h = h
        self.lib = lib
        self.n_total = {}

    def close(self):
        if getattr(self, "_h", None):
            _check(self.lib.vxl_sph_serve_destroy(self._h))
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def set_batch_cap(self, max_fluid_particles: int) -> None:
        """Stop admitting while the admitted scenes hold this many fluid particles (0: no cap)."""
        _check(self.lib.vxl_sph_serve_set_batch_cap(self._h, int(max_fluid_particles)))

    def submit(self, spec, ticks: int) -> int:
        keep: list = []
        d = _desc_of(spec.params, spec.pos, spec.vel, spec.pmass, spec.n_fluid, 0, keep)
        rid = C.c_uint64()
        _check(self.lib.vxl_sph_serve_submit(self._h, C.byref(d), ticks, C.byref(rid)))
        self.n_total[rid.value] = spec.n_total
        return rid.value

    def step(self, dt_tick: float) -> ServeReport:
        r = ServeReport()
        r.hdr = header(ServeReport)
        _check(self.lib.vxl_sph_serve_step(self._h, dt_tick, C.byref(r)))
        return r

    def poll(self, rid: int) -> RequestStatus:
        st = RequestStatus()
        st.hdr = header(RequestStatus)
        _check(self.lib.vxl_sph_serve_poll(self._h, rid, C.byref(st)))
        return st

    def read(self, rid: int):
        n = self.n_total[rid]
        p = np.empty((n, 3), np.float32)
        v = np.empty((n, 3), np.float32)
        _check(self.lib.vxl_sph_serve_read(self._h, rid, _fptr(p), _fptr(v)))
        return p, v

    def tick_times(self, rid: int) -> np.ndarray:
        """Wall time (ms) of each completed tick of a request."""
        n = C.c_uint32()
        _check(self.lib.vxl_sph_serve_tick_times(self._h, rid, None, 0, C.byref(n)))
        out = np.empty(n.value, np.float64)
        if n.value:
            _check(self.lib.vxl_sph_serve_tick_times(self._h, rid, out.ctypes.data_as(C.POINTER(C.c_double)),
                                                     n.value, C.byref(n)))
        return out


class PhysGpuBackend:
    """Mirror of `PhysGpuBackend` (crates/vxl-phys-gpu/src/lib.rs:20-29)."""

    def name(self) -> str:
        return load().vxl_sph_backend_name().decode()

    def available(self) -> bool:
        return bool(load().vxl_sph_backend_available())

    def submit(self, tag: str) -> bool:
        # The reference's fluid path never calls submit (for it the trait is a marker); the
        # fluid entry points are the stepper's.
        return False


class GpuFluidStepper:
    """Mirror of `FluidStepper` as implemented by GpuFluidStepper
    (crates/vxl-phys-gpu/src/pipeline/stepper.rs:69-147) over the C ABI.

    Built once from the full particle set; each `step` re-uploads the boundary segment
    (length mismatches raise, stepper.rs:84-96), advances one tick on the device and
    keeps the tick-averaged reactions.
    """

    def __init__(self, params: Params, n_fluid: int, pos, vel, pmass, device: int = 0, boundaries=()):
        self.scene = Scene(params, pos, vel, pmass, n_fluid, device)
        self.n_fluid = n_fluid
        self.nb = self.scene.n_boundary
        self.boundaries = list(boundaries)  # provider ids of the fluid's walls (stepper.rs:27)
        self._reactions: list = []

    def step(self, dt_tick: float, n_fluid: int, pos, vel, pmass, spans) -> None:
        pos = np.asarray(pos, np.float32).reshape(-1, 3)
        vel = np.asarray(vel, np.float32).reshape(-1, 3)
        if n_fluid != self.n_fluid:
            raise VxlError(SIZE_MISMATCH, f"fluid prefix {n_fluid} != {self.n_fluid}")
        if pos.shape[0] != n_fluid + self.nb:
            raise VxlError(SIZE_MISMATCH, f"particle count {pos.shape[0]} != {n_fluid}+{self.nb}")
        if len(pmass) != pos.shape[0]:
            raise VxlError(SIZE_MISMATCH, "pmass length differs from the particle count")
        if self.nb:
            self.scene.upload_boundary(pos[n_fluid:], vel[n_fluid:])
        self._reactions = self.scene.step_tick(dt_tick, spans)

    def reactions(self):
        return self._reactions

    def bounds(self):
        try:
            return self.scene.bounds()
        except VxlError:
            return None

    def gather_walls(self, h: float, providers) -> None:
        """The reference's gather_walls (stepper.rs:118-137): with provider ids registered,
        read the fluid positions from the device, gather the mirror and projection contact
        tables on the host and upload them for the next tick's substeps."""
        if not self.boundaries:
            return None
        from . import walls
        pos, _ = self.scene.read_state()
        ps = pos[:self.n_fluid]
        for side in (walls.MIRROR, walls.PROJECT):
            ids, start, planes = walls.gather_contacts(self.boundaries, h, ps, providers, side)
            self.scene.set_wall_contacts(side, ids, start, planes)
        return None


# launch shape and autotuner on the plain handle too (same C entry points as the batch's)
Scene.set_tuning = Batch.set_tuning
Scene.tuning = Batch.tuning
Scene.autotune = Batch.autotune
