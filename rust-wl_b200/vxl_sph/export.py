"""State export for rendering: VXLD v3 dumps of a fluid run.

The reference's fluid demos write VXLD v3 (crates/vxl-phys/examples/dam_break.rs:80-125),
read by its renderer: header "VXLD", u32 version 3, u32 ticks, u32 ticks per frame, f32 tick
dt, the voxel volume (3 x u32 dims, 3 x f32 origin, f32 step), u32 splat count, u32 mesh
count, u32 fluid system count; then per frame u32 tick, f32 tick milliseconds, u32 rigid
body count, the voxel occupancy bits (x-major, one bit per cell) and per fluid system a u32
particle count followed by its xyz triples; all little-endian. This library has no voxel
terrain, so the volume written is one empty cell, no splats, no meshes, no rigid bodies;
the fluid section carries the fluid particles (the prefix of each scene's state).

Frames come from the deferred readback (vxl_sph_request_state / vxl_sph_take_state): the
copy of tick t's positions is requested right behind that tick and taken while tick t + 1
runs, so writing the file overlaps the simulation.
"""
from __future__ import annotations

import struct
import time

import numpy as np

VXLD_VERSION = 3


def write_header(f, ticks: int, ticks_per_frame: int, dt_tick: float, n_systems: int) -> None:
    f.write(b"VXLD")
    f.write(struct.pack("<IIIf", VXLD_VERSION, ticks, ticks_per_frame, dt_tick))
    f.write(struct.pack("<III", 1, 1, 1))           # voxel dims: one cell
    f.write(struct.pack("<fff", 0.0, 0.0, 0.0))     # voxel origin
    f.write(struct.pack("<f", 1.0))                 # voxel step
    f.write(struct.pack("<III", 0, 0, n_systems))   # splats, meshes, fluid systems


def write_frame(f, tick: int, ms: float, systems) -> None:
    """systems: iterable of (N, 3) float32 position arrays (one per fluid system)."""
    f.write(struct.pack("<IfI", tick, ms, 0))
    f.write(b"\x00")                                # occupancy bits of the one empty cell
    for p in systems:
        p = np.ascontiguousarray(p, dtype="<f4").reshape(-1, 3)
        f.write(struct.pack("<I", p.shape[0]))
        f.write(p.tobytes())


def dump_run(scene, path: str, ticks: int, dt_tick: float, spans=(), ticks_per_frame: int = 2) -> dict:
    """Step a plain handle `ticks` ticks and write every `ticks_per_frame`-th tick's fluid
    positions to a VXLD v3 file, the readback of each frame overlapping the next tick."""
    nf = scene.n_fluid
    buf = np.empty((scene.n_total, 3), np.float32)
    pending = None  # (tick, ms) of a requested frame not yet written
    with open(path, "wb") as f:
        write_header(f, ticks, ticks_per_frame, dt_tick, 1)
        for t in range(1, ticks + 1):
            t0 = time.perf_counter()
            scene.step_tick_async(dt_tick, spans)
            if pending is not None:  # the previous frame's copy is ahead of this tick
                scene.take_state(buf)
                write_frame(f, pending[0], pending[1], [buf[:nf]])
                pending = None
            scene.sync()
            ms = 1e3 * (time.perf_counter() - t0)
            if t % ticks_per_frame == 0:
                scene.request_state()
                pending = (t, ms)
        if pending is not None:
            scene.take_state(buf)
            write_frame(f, pending[0], pending[1], [buf[:nf]])
    return {"path": path, "ticks": ticks, "frames": ticks // ticks_per_frame, "particles": nf}


def read_vxld(path: str) -> dict:
    """Parse a VXLD v3 file written by dump_run (the same layout the reference writes)."""
    with open(path, "rb") as f:
        data = f.read()
    assert data[:4] == b"VXLD"
    off = 4
    version, ticks, tpf, dt = struct.unpack_from("<IIIf", data, off)
    off += 16
    dims = struct.unpack_from("<III", data, off)
    off += 12 + 12 + 4
    splats, meshes, nsys = struct.unpack_from("<III", data, off)
    off += 12
    nbits = (dims[0] * dims[1] * dims[2] + 7) // 8
    frames = []
    while off < len(data):
        tick, ms, nbodies = struct.unpack_from("<IfI", data, off)
        off += 12
        assert nbodies == 0
        off += nbits
        systems = []
        for _ in range(nsys):
            (n,) = struct.unpack_from("<I", data, off)
            off += 4
            systems.append(np.frombuffer(data, "<f4", 3 * n, off).reshape(n, 3).copy())
            off += 12 * n
        frames.append({"tick": tick, "ms": ms, "systems": systems})
    return {"version": version, "ticks": ticks, "ticks_per_frame": tpf, "dt": dt, "frames": frames}
