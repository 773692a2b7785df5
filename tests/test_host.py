"""Host-side checks that need no GPU: the C ABI library loads and exports every symbol
include/vxl_sph.h declares, its struct layouts match the header, its host set-up math
(lattice mass, Akinci lattice) equals the oracle bit for bit, the scene builders give
the oracle's set_boundary_particles result, and argument errors come back as the
reference's FfiError codes (crates/vxl-phys-ffi/src/lib.rs:26-33) rather than crashes.
"""
import ctypes as C
import re
import subprocess
from pathlib import Path

import numpy as np
import pytest

ROOT = Path(__file__).resolve().parent.parent
HEADER = ROOT / "include" / "vxl_sph.h"


def declared_functions():
    text = HEADER.read_text()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(vxl_sph_[a-z_0-9]+)\s*\(", text)))


def test_library_exports_every_declared_symbol(vxl):
    lib = vxl.load()
    names = declared_functions()
    assert len(names) >= 20
    missing = [n for n in names if not hasattr(lib, n)]
    assert not missing, missing
    # and the binding covers every one of them
    assert set(names) == set(vxl.SIGNATURES), set(names) ^ set(vxl.SIGNATURES)


def test_abi_version(vxl):
    assert vxl.load().vxl_sph_abi_version() == vxl.ABI_VERSION == 1


def test_struct_sizes_match_header(vxl, tmp_path):
    src = tmp_path / "sizes.c"
    src.write_text(
        '#include <stdio.h>\n#include "vxl_sph.h"\nint main(void){printf("%zu %zu %zu %zu %zu %zu %zu\\n",'
        "sizeof(vxl_sph_params),sizeof(vxl_sph_desc),sizeof(vxl_sph_span),sizeof(vxl_sph_reaction),"
        "sizeof(vxl_sph_grid_info),sizeof(vxl_sph_stats),sizeof(vxl_block_header));"
        'printf("%zu %zu %zu %zu\\n",sizeof(vxl_sph_tuning),sizeof(vxl_sph_request_status),sizeof(vxl_sph_serve_report),sizeof(vxl_sph_body_pose));'
        'printf("%zu %zu %zu\\n",sizeof(vxl_sph_rigid_body),sizeof(vxl_sph_wall_plane),sizeof(vxl_sph_provider));'
        "return 0;}\n")
    exe = tmp_path / "sizes"
    subprocess.run(["gcc", "-std=c99", "-I", str(ROOT / "include"), str(src), "-o", str(exe)], check=True)
    got = [int(x) for x in subprocess.run([str(exe)], capture_output=True, text=True, check=True).stdout.split()]
    want = [C.sizeof(t) for t in (vxl.Params, vxl.Desc, vxl.Span, vxl.Reaction, vxl.GridInfo, vxl.Stats,
                                  vxl.BlockHeader, vxl.Tuning, vxl.RequestStatus, vxl.ServeReport, vxl.BodyPose, vxl.RigidBody, vxl.WallPlane,
                                  vxl.Provider)]
    assert got == want


@pytest.mark.parametrize("half,density", [((0.2, 0.15, 0.1), 500.0), ((0.05, 0.05, 0.05), 1000.0),
                                          ((0.3, 0.02, 0.17), -1.0), ((0.125, 0.25, 0.5), 740.0)])
def test_box_mass_props_bit_identical(vxl, oracle_mod, half, density):
    from vxl_sph.scenes import box_mass_props
    im, ii = box_mass_props(half, density)
    im_o, ii_o = oracle_mod.box_mass_props(half, density)
    assert np.float32(im).tobytes() == np.float32(im_o).tobytes()
    assert np.asarray(ii, np.float32).tobytes() == ii_o.tobytes()


@pytest.mark.parametrize("h,s", [(0.1, 0.05), (0.04, 0.02), (0.02, 0.01), (0.01, 0.005), (0.1, 0.03)])
def test_lattice_mass_bit_identical(vxl, oracle_mod, h, s):
    p = vxl.make_params(smoothing_radius=h)
    c = oracle_mod.default_cfg(smoothing_radius=h)
    m_lib = vxl.lattice_mass(p, s)
    m_orc = float(oracle_mod.load().orc_lattice_mass(C.byref(c), s))
    assert np.float32(m_lib).tobytes() == np.float32(m_orc).tobytes()


@pytest.mark.parametrize("shape,half,radius,s,h,layers", [
    (0, (0.06, 0.06, 0.06), 0.0, 0.05, 0.1, 2),
    (0, (0.3, 0.05, 0.3), 0.0, 0.05, 0.1, 2),
    (0, (0.02, 0.32, 0.36), 0.0, 0.02, 0.04, 1),
    (0, (0.07, 0.11, 0.13), 0.0, 0.01, 0.02, 3),
    (1, (0, 0, 0), 0.2, 0.05, 0.1, 2),
    (1, (0, 0, 0), 0.13, 0.02, 0.04, 1),
])
def test_boundary_lattice_bit_identical(vxl, oracle_mod, shape, half, radius, s, h, layers):
    pts_l, vol_l = vxl.boundary_lattice(shape, half, radius, s, h, layers)
    pts_o, vol_o, _ = oracle_mod.lattice(shape, half, radius, s, h, layers)
    assert pts_l.shape == pts_o.shape
    assert pts_l.tobytes() == pts_o.tobytes()
    assert np.float32(vol_l) == np.float32(vol_o)


def test_scene_bodies_equal_oracle_set_boundary_particles(vxl, oracle_mod):
    from vxl_sph import scenes
    spec = scenes.small_dam()
    c = oracle_mod.cfg_from_params(spec.params)
    o = oracle_mod.OracleSystem(c, (0, 0, 0), (spec.n_fluid, 1, 1), spec.spacing)
    bodies = scenes.tank_bodies(spec.meta["tank"], 2.0 * spec.spacing)
    nb = o.set_bodies(bodies)
    assert nb == spec.n_boundary
    r = o.read_f32()
    nf = spec.n_fluid
    assert r["pos"][nf:].tobytes() == spec.pos[nf:].tobytes()
    assert r["vel"][nf:].tobytes() == spec.vel[nf:].tobytes()
    assert r["pmass"][nf:].tobytes() == spec.pmass[nf:].tobytes()
    assert [(b, s, e) for b, _, s, e in o.spans()] == [(b, s, e) for b, _, s, e in spec.spans]
    assert np.float32(o.mass) == np.float32(spec.params.particle_mass)


def test_scene_moving_body_velocity_matches_oracle(vxl, oracle_mod):
    from vxl_sph import scenes
    b = scenes.Body(3, (0.05, 0.07, 0.04), (0.2, 0.3, 0.1), rot=(0.0, 0.38268343, 0.0, 0.9238795),
                    linvel=(0.5, -0.2, 0.1), angvel=(0.3, 1.2, -0.7))
    params = scenes.baseline_params(0.01)
    pos, vel, pm, spans = scenes.body_particles([b], 0.01, params.smoothing_radius, 1, 1000.0)
    c = oracle_mod.cfg_from_params(params)
    o = oracle_mod.OracleSystem(c, (0, 0, 0), (1, 1, 1), 0.01)
    o.set_bodies([b])
    r = o.read_f32()
    assert r["pos"][1:].tobytes() == pos.tobytes()
    assert r["vel"][1:].tobytes() == vel.tobytes()


def _desc(vxl, n=8):
    p = vxl.make_params(particle_mass=1.0)
    pos = np.zeros((n, 3), np.float32)
    d = vxl.Desc()
    d.hdr = vxl.header(vxl.Desc)
    d.params = p
    d.n_fluid = n
    d.n_boundary = 0
    d.pos_xyz = pos.ctypes.data_as(C.POINTER(C.c_float))
    d.vel_xyz = pos.ctypes.data_as(C.POINTER(C.c_float))
    d.pmass = None
    return d, pos


def test_create_argument_errors(vxl):
    lib = vxl.load()
    h = C.c_void_p()
    assert lib.vxl_sph_create(None, C.byref(h)) == vxl.NULL_POINTER
    d, keep = _desc(vxl)
    d.hdr.version = 2
    assert lib.vxl_sph_create(C.byref(d), C.byref(h)) == vxl.VERSION_MISMATCH
    d, keep = _desc(vxl)
    d.hdr.size = 8
    assert lib.vxl_sph_create(C.byref(d), C.byref(h)) == vxl.SIZE_MISMATCH
    d, keep = _desc(vxl)
    d.params.particle_mass = 0.0
    assert lib.vxl_sph_create(C.byref(d), C.byref(h)) == vxl.INVALID_ARGUMENT
    d, keep = _desc(vxl)
    d.params.max_bins = (1 << 21) + 1
    assert lib.vxl_sph_create(C.byref(d), C.byref(h)) == vxl.INVALID_ARGUMENT
    assert b"max_bins" in lib.vxl_sph_last_error()


def test_null_handle_errors(vxl):
    lib = vxl.load()
    assert lib.vxl_sph_destroy(None) == vxl.NULL_POINTER
    assert lib.vxl_sph_step_tick(None, 1 / 60, None, 0, None) == vxl.NULL_POINTER
    assert lib.vxl_sph_read_state(None, None, None) == vxl.NULL_POINTER
    assert lib.vxl_sph_upload_boundary(None, 0, None, None, 0) == vxl.NULL_POINTER


def test_no_cpu_fallback_without_gpu(vxl):
    """Without a usable sm_100 device the library refuses to run (no CPU path)."""
    import torch
    if torch.cuda.is_available():
        pytest.skip("a GPU is present")
    assert vxl.PhysGpuBackend().available() is False
    assert vxl.PhysGpuBackend().name() == "b200-cuda-wcsph"
    d, keep = _desc(vxl)
    h = C.c_void_p()
    st = vxl.load().vxl_sph_create(C.byref(d), C.byref(h))
    assert st == vxl.CUDA_ERROR and not h.value


def test_scene_sizes(vxl):
    from vxl_sph import scenes
    s0 = scenes.dam0()
    assert s0.n_fluid == 16384 and s0.n_boundary > 0
    assert s0.params.substeps == 10 and abs(s0.params.smoothing_radius - 0.04) < 1e-9
    assert all(s0.pmass[:s0.n_fluid] == np.float32(s0.params.particle_mass))
    # jitter is within +-1% of the spacing and seeded
    lat = scenes.fluid_block((0, 0, 0), (16, 32, 32), 0.02)
    dj = np.abs(s0.pos[:s0.n_fluid] - lat)
    assert dj.max() <= 0.01 * 0.02 * 1.0001 and dj.max() > 0
    assert scenes.dam0().pos.tobytes() == s0.pos.tobytes()


def test_body_lattice_matches_body_particles(vxl):
    """scenes.body_lattice + the pose transform restate body_particles exactly (the inputs
    of the device-side rebuild describe the same boundary segment)."""
    from vxl_sph import scenes
    bodies = [scenes.Body(3, (0.05, 0.07, 0.04), (0.2, 0.3, 0.1), rot=(0.0, 0.38268343, 0.0, 0.9238795),
                          linvel=(0.5, -0.2, 0.1), angvel=(0.3, 1.2, -0.7)),
              scenes.Body(7, (0.03, 0.03, 0.06), (-0.1, 0.2, 0.05), rot=(0.1, 0.2, 0.3, 0.9273618))]
    pos, vel, _, _ = scenes.body_particles(bodies, 0.01, 0.02, 1, 1000.0)
    local, idx = scenes.body_lattice(bodies, 0.01, 0.02, 1)
    assert local.shape == pos.shape and idx.shape == (pos.shape[0],)
    F = np.float32
    for q, b in enumerate(bodies):
        sel = idx == q
        bp = np.asarray(b.pos, F)
        wp = (bp + scenes.rotate(b.rot, local[sel])).astype(F)
        assert wp.tobytes() == pos[sel].tobytes()
        r = (wp - bp).astype(F)
        wv = (np.asarray(b.linvel, F) + scenes._cross(np.broadcast_to(np.asarray(b.angvel, F), r.shape), r)).astype(F)
        assert wv.tobytes() == vel[sel].tobytes()


def test_vxld_round_trip(tmp_path):
    """VXLD v3 writer/reader round trip (the layout of the reference's demo dumps)."""
    from vxl_sph import export
    rng = np.random.Generator(np.random.PCG64(1))
    frames = [rng.standard_normal((17, 3)).astype(np.float32) for _ in range(3)]
    path = tmp_path / "run.bin"
    with open(path, "wb") as f:
        export.write_header(f, 6, 2, 1.0 / 60.0, 1)
        for k, p in enumerate(frames):
            export.write_frame(f, 2 * (k + 1), 1.5, [p])
    r = export.read_vxld(str(path))
    assert r["version"] == 3 and r["ticks"] == 6 and r["ticks_per_frame"] == 2
    assert [fr["tick"] for fr in r["frames"]] == [2, 4, 6]
    for fr, p in zip(r["frames"], frames):
        assert fr["systems"][0].tobytes() == p.tobytes()
    # header size: magic + 4 words + voxel block (28 B) + 3 counts
    assert path.stat().st_size == 4 + 16 + 28 + 12 + 3 * (12 + 1 + 4 + 17 * 12)


def test_provider_arrays_packing(vxl):
    """Faces and Convex providers pack into the C ABI's provider and plane arrays in order,
    each provider's planes as one run of the plane array."""
    from vxl_sph import scenes
    prs = [scenes.tank_provider(0.3), scenes.box_obstacle((0.0, 0.1, 0.0), (0.05, 0.1, 0.05)), vxl.Faces([(2, 1.5, -1.0)])]
    parr, n, warr, nw = vxl.providers_arrays(prs)
    assert n == 3 and nw == 5 + 6 + 1
    assert [(parr[q].kind, parr[q].first_plane, parr[q].nplanes, parr[q].has_bounds) for q in range(n)] == \
        [(vxl.PROVIDER_FACES, 0, 5, 1), (vxl.PROVIDER_CONVEX, 5, 6, 1), (vxl.PROVIDER_FACES, 11, 1, 0)]
    assert (warr[1].axis, np.float32(warr[1].offset), warr[1].sign) == (0, np.float32(-0.3), 1.0)
    assert (warr[2].axis, np.float32(warr[2].offset), warr[2].sign) == (0, np.float32(0.3), -1.0)
    # box obstacle: +x face at c + h, -x face at -(c - h)
    assert list(warr[5].normal) == [1.0, 0.0, 0.0] and np.isclose(warr[5].offset, 0.05)
    assert list(warr[6].normal) == [-1.0, 0.0, 0.0] and np.isclose(warr[6].offset, 0.05)
    assert (warr[11].axis, warr[11].offset, warr[11].sign) == (2, 1.5, -1.0)


def _rigid_substep_restated(b, react, g, dt, maxl, maxa):
    """One rigid substep of the coupling loop, float32, written from the reference's formulas:
    gravity field force m g with m = 1 / inv_mass (crates/vxl-phys-field/src/lib.rs:22-31), the
    fluid reaction added, Integrator::integrate_velocities with gravity zero and whole-vector
    clamps, integrate_positions with Quat::integrate_angular (crates/vxl-phys-integrate/src/
    lib.rs:18-60, crates/vxl-phys-core/src/math.rs:216-252, body.rs:172-176)."""
    f = np.float32
    pos, q, v, w = [list(map(f, b[a:c])) for a, c in ((0, 3), (3, 7), (7, 10), (10, 13))]
    inv_m, ii = f(b[13]), list(map(f, b[14:17]))
    mass = f(f(1.0) / inv_m)
    force = [f(f(0.0) + f(g[a]) * mass) for a in range(3)]
    force = [f(force[a] + f(react[a])) for a in range(3)]
    torque = [f(f(0.0) + f(react[3 + a])) for a in range(3)]
    v = [f(v[a] + f(f(0.0) + f(force[a] * inv_m)) * f(dt)) for a in range(3)]
    x, y, z, qw = q
    xx, yy, zz, xy, xz, yz, wx, wy, wz = (f(x * x), f(y * y), f(z * z), f(x * y), f(x * z), f(y * z), f(qw * x),
                                          f(qw * y), f(qw * z))
    m = [[f(1.0) - f(2.0) * f(yy + zz), f(2.0) * f(xy - wz), f(2.0) * f(xz + wy)],
         [f(2.0) * f(xy + wz), f(1.0) - f(2.0) * f(xx + zz), f(2.0) * f(yz - wx)],
         [f(2.0) * f(xz - wy), f(2.0) * f(yz + wx), f(1.0) - f(2.0) * f(xx + yy)]]
    lt = [f(f(f(m[0][c] * torque[0]) + f(m[1][c] * torque[1])) + f(m[2][c] * torque[2])) for c in range(3)]
    lt = [f(lt[c] * ii[c]) for c in range(3)]
    aa = [f(f(f(m[r][0] * lt[0]) + f(m[r][1] * lt[1])) + f(m[r][2] * lt[2])) for r in range(3)]
    w = [f(w[a] + f(aa[a] * f(dt))) for a in range(3)]
    sp = np.sqrt(f(f(f(v[0] * v[0]) + f(v[1] * v[1])) + f(v[2] * v[2])), dtype=f)
    if sp > f(maxl):
        s = f(f(maxl) / sp)
        v = [f(c * s) for c in v]
    ws = np.sqrt(f(f(f(w[0] * w[0]) + f(w[1] * w[1])) + f(w[2] * w[2])), dtype=f)
    if ws > f(maxa):
        s = f(f(maxa) / ws)
        w = [f(c * s) for c in w]
    pos = [f(pos[a] + f(v[a] * f(dt))) for a in range(3)]
    # dq = (w, 0) * q, Hamilton product
    dqw = f(f(f(f(f(0.0) * qw) - f(w[0] * x)) - f(w[1] * y)) - f(w[2] * z))
    dqx = f(f(f(f(f(0.0) * x) + f(w[0] * qw)) + f(w[1] * z)) - f(w[2] * y))
    dqy = f(f(f(f(f(0.0) * y) - f(w[0] * z)) + f(w[1] * qw)) + f(w[2] * x))
    dqz = f(f(f(f(f(0.0) * z) + f(w[0] * y)) - f(w[1] * x)) + f(w[2] * qw))
    hd = f(f(0.5) * f(dt))
    nq = [f(x + f(dqx * hd)), f(y + f(dqy * hd)), f(z + f(dqz * hd)), f(qw + f(dqw * hd))]
    len2 = f(f(f(f(nq[0] * nq[0]) + f(nq[1] * nq[1])) + f(nq[2] * nq[2])) + f(nq[3] * nq[3]))
    inv = f(f(1.0) / np.sqrt(len2, dtype=f))
    nq = [f(c * inv) for c in nq]
    return pos + nq + v + w


@pytest.mark.parametrize("case", range(4))
def test_oracle_rigid_substep_equals_direct_restatement(oracle_mod, case):
    """The oracle's rigid substep (what the device coupling loop is checked against) equals a
    float32 restatement of the reference's integrator formulas, bit for bit, including the
    speed clamps."""
    rng = np.random.default_rng(100 + case)
    q = rng.normal(size=4).astype(np.float32)
    q /= np.linalg.norm(q)
    st = np.zeros((1, 18), np.float32)
    st[0, 0:3] = rng.uniform(-1, 1, 3)
    st[0, 3:7] = q
    st[0, 7:10] = rng.uniform(-2, 2, 3) * (60.0 if case == 3 else 1.0)
    st[0, 10:13] = rng.uniform(-3, 3, 3) * (30.0 if case == 3 else 1.0)
    st[0, 13] = np.float32(1.0) / np.float32(rng.uniform(0.5, 5.0))
    st[0, 14:17] = rng.uniform(1.0, 40.0, 3)
    st[0, 17] = 1.0
    react = rng.uniform(-20, 20, (1, 6)).astype(np.float32)
    g = (0.0, -9.81, 0.0)
    dt = float(np.float32(np.float32(1.0) / np.float32(60.0)) / np.float32(2.0))
    want = _rigid_substep_restated(st[0].copy(), react[0], g, dt, 100.0, 50.0)
    oracle_mod.rigid_step(st, react, g, dt, 1, 100.0, 50.0)
    assert st[0, :13].tobytes() == np.array(want, np.float32).tobytes(), (st[0, :13], want)
