"""ctypes binding of the WCSPH oracle — TEST INFRASTRUCTURE ONLY.

Used by tests/, __graft_entry__.smoke() and bench.py's cpu_baseline leg as the
checker; the library under rust-wl_b200/ never imports it. The oracle is a C++
restatement of the reference's Rust CPU path (wcsph_oracle.hpp), pinned against the
reference's published CPU grid-table hashes (tests/golden/grid_hashes.json).
"""
from __future__ import annotations

import ctypes as C
import subprocess
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
LIB_PATH = HERE / "liboracle_wcsph.so"


class Cfg(C.Structure):
    _fields_ = [
        ("rest_density", C.c_float),
        ("smoothing_radius", C.c_float),
        ("xsph_viscosity", C.c_float),
        ("tensile_instability_suppression", C.c_uint32),
        ("sound_speed", C.c_float),
        ("gamma_tait", C.c_float),
        ("substeps", C.c_uint32),
        ("threads", C.c_uint32),
        ("boundary_layers", C.c_uint32),
        ("gravity", C.c_float * 3),
        ("max_speed_frac", C.c_float),
        ("artificial_viscosity", C.c_float),
        ("max_bins", C.c_uint64),
    ]


class OBody(C.Structure):
    _fields_ = [
        ("id", C.c_uint32), ("shape", C.c_uint32), ("half", C.c_float * 3), ("radius", C.c_float),
        ("pos", C.c_float * 3), ("rot", C.c_float * 4), ("linvel", C.c_float * 3), ("angvel", C.c_float * 3),
    ]


class OSpan(C.Structure):
    _fields_ = [("body", C.c_uint32), ("origin", C.c_float * 3), ("start", C.c_uint32), ("end", C.c_uint32)]


class OWallPlane(C.Structure):
    _fields_ = [("normal", C.c_float * 3), ("d", C.c_float), ("axis", C.c_uint32), ("sign", C.c_float)]


class OProvider(C.Structure):
    _fields_ = [("kind", C.c_uint32), ("first", C.c_uint32), ("count", C.c_uint32), ("has_bounds", C.c_uint32),
                ("bmin", C.c_float * 3), ("bmax", C.c_float * 3)]


class OReaction(C.Structure):
    _fields_ = [("body", C.c_uint32), ("force", C.c_float * 3), ("torque", C.c_float * 3)]


def build() -> Path:
    """Compile the oracle library if it is missing or older than its sources."""
    srcs = [HERE / "oracle_capi.cpp", HERE / "wcsph_oracle.hpp", HERE / "Makefile"]
    if not LIB_PATH.exists() or any(s.stat().st_mtime > LIB_PATH.stat().st_mtime for s in srcs):
        subprocess.run(["make", "-s", "-C", str(HERE)], check=True)
    return LIB_PATH


_lib = None
_FP = C.POINTER(C.c_float)
_DP = C.POINTER(C.c_double)
_U32P = C.POINTER(C.c_uint32)


def load() -> C.CDLL:
    global _lib
    if _lib is not None:
        return _lib
    lib = C.CDLL(str(build()))
    sig = {
        "orc_create": (C.c_void_p, [C.POINTER(Cfg), _FP, C.POINTER(C.c_uint64), C.c_float, C.c_int]),
        "orc_destroy": (None, [C.c_void_p]),
        "orc_n_total": (C.c_uint64, [C.c_void_p]),
        "orc_n_fluid": (C.c_uint64, [C.c_void_p]),
        "orc_mass": (C.c_double, [C.c_void_p]),
        "orc_set_threads": (None, [C.c_void_p, C.c_uint32]),
        "orc_set_mass": (None, [C.c_void_p, C.c_double]),
        "orc_lattice_mass": (C.c_float, [C.POINTER(Cfg), C.c_float]),
        "orc_set_state": (C.c_int, [C.c_void_p, _FP, _FP, C.c_uint64]),
        "orc_set_bodies": (C.c_uint64, [C.c_void_p, C.POINTER(OBody), C.c_uint32]),
        "orc_set_boundary_raw": (C.c_int, [C.c_void_p, C.c_uint64, _FP, _FP, _FP, C.POINTER(OSpan), C.c_uint32]),
        "orc_step": (None, [C.c_void_p, C.c_float]),
        "orc_substep": (None, [C.c_void_p, C.c_float]),
        "orc_run_ticks": (C.c_double, [C.c_void_p, C.c_float, C.c_uint32]),
        "orc_read": (None, [C.c_void_p] + [_DP] * 8),
        "orc_read_f32": (None, [C.c_void_p] + [_FP] * 8),
        "orc_grid": (C.c_uint64, [C.c_void_p, _U32P, C.c_uint64, _U32P, _FP, _FP, _U32P]),
        "orc_reactions": (C.c_uint32, [C.c_void_p, C.POINTER(OReaction), C.c_uint32]),
        "orc_neighbors": (C.c_uint64, [C.c_void_p, C.POINTER(C.c_uint64), _U32P, C.c_uint64]),
        "orc_aggregate_with": (None, [C.c_void_p, _FP, C.c_int]),
        "orc_scale_reactions": (None, [C.c_void_p, C.c_float]),
        "orc_spans": (C.c_uint32, [C.c_void_p, C.POINTER(OSpan), C.c_uint32]),
        "orc_grid_box": (None, [_FP, _FP, C.c_float, C.c_uint64, _FP, _FP, _U32P]),
        "orc_rebuild_grid": (C.c_uint64, [_FP, C.c_uint64, C.c_float, C.c_uint64, _U32P, C.c_uint64, _U32P, _U32P]),
        "orc_lattice": (C.c_uint64, [C.c_uint32, _FP, C.c_float, C.c_float, C.c_float, C.c_uint32, _FP, C.c_uint64,
                                     _FP, C.POINTER(C.c_uint64)]),
        "orc_boundary_self_sum": (C.c_float, [_FP, C.c_uint64, C.c_float]),
        "orc_grid_probe_hash": (C.c_uint64, [C.c_uint64, C.c_uint64, C.c_uint32]),
        "orc_consts": (None, [C.c_void_p, _DP]),
        "orc_set_providers": (None, [C.c_void_p, C.POINTER(OProvider), C.c_uint32, C.POINTER(OWallPlane)]),
        "orc_set_wall_contacts": (None, [C.c_void_p, C.c_uint32, _U32P, _U32P, C.c_uint32, _FP]),
        "orc_rigid_step": (None, [_FP, C.c_uint32, _FP, _FP, C.c_float, C.c_uint32, C.c_float, C.c_float]),
        "orc_box_mass_props": (None, [_FP, C.c_float, _FP, _FP]),
    }
    for name, (res, args) in sig.items():
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    _lib = lib
    return lib


def _f(a):
    return None if a is None else a.ctypes.data_as(_FP)


def cfg_from_params(p, threads: int = 1) -> Cfg:
    """Oracle FluidConfig from the library's Params struct (same fields)."""
    c = Cfg()
    c.rest_density = p.rest_density
    c.smoothing_radius = p.smoothing_radius
    c.xsph_viscosity = p.xsph_viscosity
    c.tensile_instability_suppression = p.tensile_instability_suppression
    c.sound_speed = p.sound_speed
    c.gamma_tait = p.gamma_tait
    c.substeps = p.substeps
    c.threads = threads
    c.boundary_layers = p.boundary_layers
    for a in range(3):
        c.gravity[a] = p.gravity[a]
    c.max_speed_frac = p.max_speed_frac
    c.artificial_viscosity = p.artificial_viscosity
    c.max_bins = p.max_bins
    return c


def default_cfg(**over) -> Cfg:
    """The reference's FluidConfig::default() (crates/vxl-phys-fluid/src/config.rs:47-68)."""
    c = Cfg()
    vals = dict(rest_density=1000.0, smoothing_radius=0.1, xsph_viscosity=0.1, tensile_instability_suppression=1,
                sound_speed=10.0, gamma_tait=7.0, substeps=4, threads=1, boundary_layers=2, max_speed_frac=0.4,
                artificial_viscosity=1.0, max_bins=0)
    grav = over.pop("gravity", (0.0, -9.81, 0.0))
    vals.update(over)
    for k, v in vals.items():
        setattr(c, k, v)
    for a in range(3):
        c.gravity[a] = grav[a]
    return c


class OracleSystem:
    """FluidSystem restated (f32, or the FP64 twin with fp64=True)."""

    def __init__(self, cfg: Cfg, origin=(0.0, 0.0, 0.0), dims=(1, 1, 1), spacing=0.05, fp64: bool = False):
        lib = load()
        o = np.asarray(origin, np.float32)
        d = (C.c_uint64 * 3)(*dims)
        self._h = lib.orc_create(C.byref(cfg), _f(o), d, spacing, 1 if fp64 else 0)
        self.lib = lib
        self.fp64 = fp64

    @classmethod
    def from_scene(cls, spec, threads: int = 1, fp64: bool = False) -> "OracleSystem":
        """Oracle over exactly a SceneSpec's arrays (fluid prefix + boundary suffix)."""
        cfg = cfg_from_params(spec.params, threads)
        dims = (spec.n_fluid, 1, 1)
        o = cls(cfg, (0.0, 0.0, 0.0), dims, spec.spacing, fp64)
        if fp64:
            # identical state: the twin uses the f32 system's mass value
            o.lib.orc_set_mass(o._h, float(np.float32(spec.params.particle_mass)))
        elif np.float32(o.mass) != np.float32(spec.params.particle_mass):
            raise AssertionError("oracle lattice mass differs from the scene's calibrated mass")
        pos = np.ascontiguousarray(spec.pos[:spec.n_fluid], np.float32)
        vel = np.ascontiguousarray(spec.vel[:spec.n_fluid], np.float32)
        o.set_state(pos, vel)
        if spec.n_boundary:
            o.set_boundary_raw(spec.pos[spec.n_fluid:], spec.vel[spec.n_fluid:], spec.pmass[spec.n_fluid:],
                               spec.spans)
        return o

    def close(self):
        if getattr(self, "_h", None):
            self.lib.orc_destroy(self._h)
            self._h = None

    def __del__(self):
        self.close()

    @property
    def n_total(self) -> int:
        return int(self.lib.orc_n_total(self._h))

    @property
    def n_fluid(self) -> int:
        return int(self.lib.orc_n_fluid(self._h))

    @property
    def mass(self) -> float:
        return float(self.lib.orc_mass(self._h))

    def set_threads(self, t: int):
        self.lib.orc_set_threads(self._h, t)

    def set_state(self, pos, vel):
        pos = None if pos is None else np.ascontiguousarray(pos, np.float32)
        vel = None if vel is None else np.ascontiguousarray(vel, np.float32)
        n = pos.shape[0] if pos is not None else vel.shape[0]
        rc = self.lib.orc_set_state(self._h, _f(pos), _f(vel), n)
        assert rc == 0, "state length differs"

    def set_bodies(self, bodies) -> int:
        arr = (OBody * max(len(bodies), 1))()
        for q, b in enumerate(bodies):
            arr[q].id = b.id
            arr[q].shape = 0
            for a in range(3):
                arr[q].half[a] = b.half[a]
                arr[q].pos[a] = b.pos[a]
                arr[q].linvel[a] = b.linvel[a]
                arr[q].angvel[a] = b.angvel[a]
            for a in range(4):
                arr[q].rot[a] = b.rot[a]
        return int(self.lib.orc_set_bodies(self._h, arr, len(bodies)))

    def consts(self) -> dict:
        """h, h2, k6, ks, w0, skin (as float32 values) and the particle mass."""
        out = np.zeros(6)
        self.lib.orc_consts(self._h, out.ctypes.data_as(_DP))
        d = dict(zip(("h", "h2", "k6", "ks", "w0", "skin"), (np.float32(x) for x in out)))
        d["mass"] = np.float32(self.lib.orc_mass(self._h))
        return d

    def set_providers(self, providers) -> None:
        """Provider walls: objects with `faces` [(axis, plane, sign)] (axis-aligned faces)
        or `planes` [((nx, ny, nz), d)] (convex half-space set), and `bounds` or None."""
        planes, recs = [], []
        for pr in providers:
            first = len(planes)
            if hasattr(pr, "faces"):
                planes += [((0.0, 0.0, 0.0), pl, ax, sg) for ax, pl, sg in pr.faces]
                kind = 0
            else:
                planes += [(tuple(n), d, 0, 1.0) for n, d in pr.planes]
                kind = 1
            recs.append((kind, first, len(planes) - first, pr.bounds))
        parr = (OProvider * max(len(recs), 1))()
        for q, (kind, first, cnt, b) in enumerate(recs):
            parr[q].kind, parr[q].first, parr[q].count = kind, first, cnt
            parr[q].has_bounds = 0 if b is None else 1
            if b is not None:
                for a in range(3):
                    parr[q].bmin[a] = b[0][a]
                    parr[q].bmax[a] = b[1][a]
        warr = (OWallPlane * max(len(planes), 1))()
        for k, (n, d, ax, sg) in enumerate(planes):
            for a in range(3):
                warr[k].normal[a] = n[a]
            warr[k].d, warr[k].axis, warr[k].sign = d, ax, sg
        self.lib.orc_set_providers(self._h, parr, len(recs), warr)

    def set_wall_contacts(self, side: int, ids, start, planes) -> None:
        """Contact table of one side (0 mirror, 1 projection): ids (E,) ascending fluid
        indices, start (E + 1,), planes (P, 6) point + outward normal; E = 0 removes it."""
        ids = np.ascontiguousarray(ids, np.uint32)
        start = np.ascontiguousarray(start, np.uint32)
        planes = np.ascontiguousarray(planes, np.float32).reshape(-1, 6)
        self.lib.orc_set_wall_contacts(self._h, side, ids.ctypes.data_as(_U32P), start.ctypes.data_as(_U32P),
                                       ids.shape[0], _f(planes))

    def set_boundary_raw(self, pos, vel, pmass, spans):
        pos = np.ascontiguousarray(pos, np.float32)
        vel = np.ascontiguousarray(vel, np.float32)
        pm = np.ascontiguousarray(pmass, np.float32)
        arr = (OSpan * max(len(spans), 1))()
        for q, (b, o, s, e) in enumerate(spans):
            arr[q].body = b
            for a in range(3):
                arr[q].origin[a] = o[a]
            arr[q].start = s
            arr[q].end = e
        self.lib.orc_set_boundary_raw(self._h, pos.shape[0], _f(pos), _f(vel), _f(pm), arr, len(spans))

    def step(self, dt_tick: float):
        self.lib.orc_step(self._h, dt_tick)

    def substep(self, dt: float):
        self.lib.orc_substep(self._h, dt)

    def run_ticks(self, dt_tick: float, ticks: int) -> float:
        return float(self.lib.orc_run_ticks(self._h, dt_tick, ticks))

    def read(self) -> dict:
        """All per-particle arrays as float64 (exact for the f32 system)."""
        n = self.n_total
        out = {k: np.empty((n, 3)) for k in ("pos", "vel", "acc", "xsph", "bforce")}
        out.update({k: np.empty(n) for k in ("dens", "press", "pmass")})
        p = lambda a: a.ctypes.data_as(_DP)
        self.lib.orc_read(self._h, p(out["pos"]), p(out["vel"]), p(out["dens"]), p(out["press"]), p(out["acc"]),
                          p(out["xsph"]), p(out["bforce"]), p(out["pmass"]))
        return out

    def read_f32(self) -> dict:
        n = self.n_total
        out = {k: np.empty((n, 3), np.float32) for k in ("pos", "vel", "acc", "xsph", "bforce")}
        out.update({k: np.empty(n, np.float32) for k in ("dens", "press", "pmass")})
        self.lib.orc_read_f32(self._h, _f(out["pos"]), _f(out["vel"]), _f(out["dens"]), _f(out["press"]),
                              _f(out["acc"]), _f(out["xsph"]), _f(out["bforce"]), _f(out["pmass"]))
        return out

    def grid(self):
        mn = np.empty(3, np.float32)
        ib = np.empty(2, np.float32)
        dims = np.empty(3, np.uint32)
        total = int(self.lib.orc_grid(self._h, None, 0, None, _f(mn), _f(ib), dims.ctypes.data_as(_U32P)))
        start = np.empty(total + 1, np.uint32)
        items = np.empty(self.n_total, np.uint32)
        self.lib.orc_grid(self._h, start.ctypes.data_as(_U32P), total + 1, items.ctypes.data_as(_U32P), None, None,
                          None)
        return {"start": start, "items": items, "min": mn, "inv": ib[0], "bin": ib[1], "dims": dims, "total": total}

    def neighbors(self):
        """The next substep's neighbour lists (walk order; fluid neighbours only for boundary
        particles) from the current positions, as CSR (offsets (n + 1,) uint64, entries uint32)."""
        n = self.n_total
        offs = np.empty(n + 1, np.uint64)
        total = int(self.lib.orc_neighbors(self._h, offs.ctypes.data_as(C.POINTER(C.c_uint64)), None, 0))
        ent = np.empty(max(total, 1), np.uint32)
        self.lib.orc_neighbors(self._h, offs.ctypes.data_as(C.POINTER(C.c_uint64)), ent.ctypes.data_as(_U32P), total)
        return offs, ent[:total]

    def reactions(self):
        arr = (OReaction * 4096)()
        n = int(self.lib.orc_reactions(self._h, arr, 4096))
        return [(arr[q].body, np.array(arr[q].force[:], np.float32), np.array(arr[q].torque[:], np.float32))
                for q in range(min(n, 4096))]

    def spans(self):
        arr = (OSpan * 4096)()
        n = int(self.lib.orc_spans(self._h, arr, 4096))
        return [(arr[q].body, tuple(arr[q].origin[:]), arr[q].start, arr[q].end) for q in range(min(n, 4096))]

    def aggregate_with(self, bforce_suffix, clear: bool):
        bf = np.ascontiguousarray(bforce_suffix, np.float32)
        self.lib.orc_aggregate_with(self._h, _f(bf), 1 if clear else 0)

    def scale_reactions(self, inv: float):
        self.lib.orc_scale_reactions(self._h, inv)


def grid_box(lo, hi, h, max_bins=0):
    lo = np.asarray(lo, np.float32)
    hi = np.asarray(hi, np.float32)
    mn = np.empty(3, np.float32)
    b = np.empty(1, np.float32)
    dims = np.empty(3, np.uint32)
    load().orc_grid_box(_f(lo), _f(hi), h, max_bins or (1 << 21), _f(mn), _f(b), dims.ctypes.data_as(_U32P))
    return mn, float(b[0]), dims


def rebuild_grid(pos, h, max_bins=0):
    pos = np.ascontiguousarray(pos, np.float32)
    dims = np.empty(3, np.uint32)
    lib = load()
    total = int(lib.orc_rebuild_grid(_f(pos), pos.shape[0], h, max_bins or (1 << 21), None, 0, None,
                                     dims.ctypes.data_as(_U32P)))
    start = np.empty(total + 1, np.uint32)
    items = np.empty(pos.shape[0], np.uint32)
    lib.orc_rebuild_grid(_f(pos), pos.shape[0], h, max_bins or (1 << 21), start.ctypes.data_as(_U32P), total + 1,
                         items.ctypes.data_as(_U32P), dims.ctypes.data_as(_U32P))
    return start, items, dims


def lattice(shape, half=(0, 0, 0), radius=0.0, s=0.05, h=0.1, layers=2):
    lib = load()
    hv = np.asarray(half, np.float32)
    vol = np.empty(1, np.float32)
    n0 = C.c_uint64()
    n = int(lib.orc_lattice(shape, _f(hv), radius, s, h, layers, None, 0, _f(vol), C.byref(n0)))
    pts = np.empty((n, 3), np.float32)
    lib.orc_lattice(shape, _f(hv), radius, s, h, layers, _f(pts), n, _f(vol), C.byref(n0))
    return pts, float(vol[0]), int(n0.value)


def boundary_self_sum(pts, h):
    pts = np.ascontiguousarray(pts, np.float32)
    return float(load().orc_boundary_self_sum(_f(pts), pts.shape[0], h))


def grid_probe_hash(n: int, max_bins: int = 0, threads: int = 8) -> int:
    return int(load().orc_grid_probe_hash(n, max_bins, threads))


def table_hash(start, items, np_count: int) -> int:
    """FNV-1a over start, items and per-particle bins recovered from the table
    (crates/vxl-phys-gpu/examples/gpu_grid_probe.rs:37-67)."""
    start = np.asarray(start, np.uint64)
    items = np.asarray(items, np.uint64)
    total = start.shape[0] - 1
    bins = np.full(np_count, 0xFFFFFFFF, np.uint64)
    counts = np.diff(start).astype(np.int64)
    bins_of_slot = np.repeat(np.arange(total, dtype=np.uint64), counts)
    bins[items.astype(np.int64)] = bins_of_slot
    h = 0xcbf29ce484222325
    prime = 0x00000100000001b3
    mask = (1 << 64) - 1
    for seq in (start, [0xFFFFFFFF], items, [0xFFFFFFFF], bins):
        for v in seq:
            h = ((h ^ int(v)) * prime) & mask
    return h


def rigid_step(states: np.ndarray, reactions: np.ndarray, gravity, dt: float, substeps: int, max_linear: float,
               max_angular: float) -> None:
    """Rigid substeps of the coupling loop (no contacts) on (n, 18) float32 states in place:
    pos, rot xyzw, linvel, angvel, inv_mass, local inverse inertia, dynamic; reactions (n, 6)."""
    lib = load()
    st = np.ascontiguousarray(states, np.float32)
    rx = np.ascontiguousarray(reactions, np.float32)
    g = np.ascontiguousarray(gravity, np.float32)
    lib.orc_rigid_step(_f(st), st.shape[0], _f(rx), _f(g), float(dt), int(substeps), float(max_linear),
                       float(max_angular))
    states[...] = st


def box_mass_props(half, density: float):
    lib = load()
    h = np.ascontiguousarray(half, np.float32)
    im = C.c_float()
    ii = np.zeros(3, np.float32)
    lib.orc_box_mass_props(_f(h), float(density), C.byref(im), _f(ii))
    return np.float32(im.value), ii


def lattice_mass(params, spacing: float) -> float:
    """FluidSystem::new's mass calibration (crates/vxl-phys-fluid/src/fluid_access.rs:27-42)
    for a library Params struct."""
    return float(load().orc_lattice_mass(C.byref(cfg_from_params(params)), spacing))


def scene_lattice_source():
    """(mass_fn, lattice_fn) for vxl_sph.scenes.use_lattice_source: the oracle's own
    restatement of the lattice-mass calibration and of boundary::lattice, so a CPU-only
    caller builds the same scenes without loading the CUDA library."""
    def lat(shape, half, radius, spacing, h, layers):
        pts, vol, _ = lattice(shape, half, radius, spacing, h, layers)
        return pts, vol
    return lattice_mass, lat
