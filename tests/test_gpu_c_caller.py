"""The library driven from C (tests/c/stepper_loop.c), the way a Rust shim or a C++ engine
calls it: the FluidStepper::step pattern over several ticks gives the same state and
reactions, bit for bit, as the same calls made through the Python binding."""
import ctypes as C
import struct
import subprocess
from pathlib import Path

import numpy as np
import pytest

pytestmark = pytest.mark.gpu
ROOT = Path(__file__).resolve().parent.parent


def test_c_caller_equals_python_binding(vxl, tmp_path):
    from vxl_sph import scenes
    spec = scenes.small_dam(n=(10, 12, 9), spacing=0.05, tank=(0.8, 0.7, 0.6))
    nf, nb = spec.n_fluid, spec.n_boundary
    dt = float(np.float32(1.0) / np.float32(60.0))
    ticks = 5
    spans, nspans = vxl.spans_array(spec.spans)
    inp = tmp_path / "in.bin"
    with open(inp, "wb") as f:
        f.write(struct.pack("<4Q", nf, nb, nspans, ticks))
        f.write(struct.pack("<f", dt))
        params = spec.params
        params.particle_mass = float(spec.pmass[0])
        f.write(bytes(params))
        for a in (spec.pos, spec.vel):
            f.write(np.ascontiguousarray(a, np.float32).tobytes())
        f.write(np.ascontiguousarray(spec.pmass, np.float32).tobytes())
        f.write(bytes(spans)[:nspans * C.sizeof(vxl.Span)])
    lib_dir = ROOT / "rust-wl_b200" / "lib"
    exe = tmp_path / "stepper_loop"
    subprocess.run(["gcc", "-std=c99", "-O2", "-I", str(ROOT / "include"), str(ROOT / "tests" / "c" / "stepper_loop.c"),
                    "-L", str(lib_dir), "-lvxl_sph", f"-Wl,-rpath,{lib_dir}", "-o", str(exe)], check=True)
    out = tmp_path / "out.bin"
    r = subprocess.run([str(exe), str(inp), str(out)], capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stderr
    raw = out.read_bytes()
    n = nf + nb
    cpos = np.frombuffer(raw[:12 * n], np.float32).reshape(n, 3)
    cvel = np.frombuffer(raw[12 * n:24 * n], np.float32).reshape(n, 3)
    creact = (vxl.Reaction * max(nspans, 1)).from_buffer_copy(raw[24 * n:].ljust(C.sizeof(vxl.Reaction) * max(nspans, 1), b"\0"))

    g = vxl.Scene(spec.params, spec.pos, spec.vel, spec.pmass, nf)
    bpos, bvel = spec.pos[nf:], spec.vel[nf:]
    for _ in range(ticks):
        g.upload_boundary(bpos, bvel)
        rg = g.step_tick(dt, spec.spans)
    p, v = g.read_state()
    g.close()
    assert cpos.tobytes() == np.ascontiguousarray(p, np.float32).tobytes()
    assert cvel.tobytes() == np.ascontiguousarray(v, np.float32).tobytes()
    for q, (bid, fg, tg) in enumerate(rg):
        assert creact[q].body == bid
        assert np.array(creact[q].force[:], np.float32).tobytes() == fg.tobytes()
        assert np.array(creact[q].torque[:], np.float32).tobytes() == tg.tobytes()
