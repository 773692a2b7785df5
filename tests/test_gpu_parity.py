"""CUDA path against the oracle, through the C ABI, on a B200.

The kernels keep the reference's summation order and f32 rounding (no FMA
contraction, IEEE div/sqrt), so the bar is bit-exactness for everything the reference
computes per particle: cell keys, the sort permutation and cell table
(crates/vxl-phys-fluid/src/grid.rs:29-76), density, pressure, acceleration, XSPH,
the per-boundary-particle reaction, and the integrated positions and velocities, over
many substeps. Per-body reactions are summed in index order, like the reference's
sequential loop (fluid_boundary.rs:10-28), for every span (bodies and tank walls), and are
compared bitwise.

The reference's own golden values enter twice: the published CPU grid-table hashes
are recomputed from tables the GPU built (test_published_hash_through_gpu), and the
oracle that the rest compares against is pinned to the same hashes.
"""
import json
from pathlib import Path

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

GOLDEN = json.loads((Path(__file__).parent / "golden" / "grid_hashes.json").read_text())
DENS_RTOL = 1e-5       # per-step tolerance of the f32 fluid step, used where bitwise is not claimed
F32 = np.float32


def f32_dt(sub):
    return float(F32(F32(1.0) / F32(60.0)) / F32(sub))


def pair(vxl, oracle_mod, spec, threads=8, fp64=False):
    g = vxl.Scene(spec.params, spec.pos, spec.vel, spec.pmass, spec.n_fluid)
    o = oracle_mod.OracleSystem.from_scene(spec, threads=threads, fp64=fp64)
    return g, o


def assert_bits(a, b, what):
    a = np.ascontiguousarray(a, np.float32)
    b = np.ascontiguousarray(b, np.float32)
    assert a.shape == b.shape, what
    if a.tobytes() != b.tobytes():
        bad = np.nonzero((a != b) & ~(np.isnan(a) & np.isnan(b)))
        first = tuple(x[0] for x in bad) if bad[0].size else None
        diff = np.nanmax(np.abs(a.astype(np.float64) - b.astype(np.float64)))
        raise AssertionError(f"{what}: {bad[0].size} entries differ (first {first}), max |diff| {diff:.3e}")


def compare_grid(g, o, label=""):
    items, start, bins, info = g.export_grid()
    og = o.grid()
    assert list(info.dims) == list(og["dims"]), label
    assert F32(info.inv) == F32(og["inv"]) and F32(info.bin) == F32(og["bin"]), label
    assert np.array_equal(np.array(info.min[:], F32), og["min"]), label
    assert np.array_equal(start, og["start"]), f"{label}: start differs"
    assert np.array_equal(items, og["items"]), f"{label}: items (permutation) differs"
    total = int(info.total)
    ob = np.repeat(np.arange(total, dtype=np.uint32), np.diff(og["start"].astype(np.int64)))
    ref_bins = np.empty_like(bins)
    ref_bins[og["items"]] = ob
    assert np.array_equal(bins, ref_bins), f"{label}: per-particle cell keys differ"
    return items, start, bins, info


def compare_state(g, o, label=""):
    gp, gv = g.read_state()
    r = o.read_f32()
    assert_bits(gp, r["pos"], f"{label} pos")
    assert_bits(gv, r["vel"], f"{label} vel")


def test_backend_available(vxl):
    b = vxl.PhysGpuBackend()
    assert b.available() and b.name() == "b200-cuda-wcsph"


@pytest.mark.parametrize("density", [0, 1])
def test_single_substep_bit_exact(vxl, oracle_mod, density):
    """One substep from identical state: table, rho, p, a, xsph, bforce, pos, vel (with each
    density kernel)."""
    from vxl_sph import scenes
    spec = scenes.small_dam(n=(10, 12, 9), spacing=0.05, tank=(0.8, 0.7, 0.6))
    g, o = pair(vxl, oracle_mod, spec)
    g.set_tuning(256, 256, 0, density)
    g.set_record(True)
    dt = f32_dt(spec.params.substeps)
    g.substep(dt)
    o.substep(dt)
    compare_grid(g, o, "substep grid")
    dens, press, acc, xsph, bf = g.read_fields()
    r = o.read_f32()
    nf = spec.n_fluid
    assert_bits(dens, r["dens"], "density")
    assert_bits(press, r["press"], "pressure")
    assert_bits(acc[:nf], r["acc"][:nf], "acceleration")
    assert_bits(xsph[:nf], r["xsph"][:nf], "xsph")
    assert_bits(bf, r["bforce"][nf:], "boundary reaction per particle")
    compare_state(g, o, "after substep")


def test_fp64_error_equal_for_gpu_and_oracle(vxl, oracle_mod):
    """Error of both f32 paths against the FP64 twin from identical state (they are
    bitwise equal, so their errors are too); both within the per-step tolerance."""
    from vxl_sph import scenes
    spec = scenes.small_dam(n=(10, 10, 10), spacing=0.05, tank=(0.8, 0.7, 0.6))
    g = vxl.Scene(spec.params, spec.pos, spec.vel, spec.pmass, spec.n_fluid)
    o64 = oracle_mod.OracleSystem.from_scene(spec, threads=8, fp64=True)
    g.set_record(True)
    dt = f32_dt(spec.params.substeps)
    g.substep(dt)
    o64.substep(dt)
    dens, press, acc, xsph, _ = g.read_fields()
    r = o64.read()
    nf = spec.n_fluid
    rel_rho = np.max(np.abs(dens - r["dens"]) / r["dens"])
    amax = np.abs(r["acc"][:nf]).max()
    rel_acc = np.max(np.abs(acc[:nf] - r["acc"][:nf])) / amax
    assert rel_rho < DENS_RTOL and rel_acc < DENS_RTOL, (rel_rho, rel_acc)


@pytest.mark.parametrize("ticks", [6])
def test_multi_tick_bit_exact_with_reactions(vxl, oracle_mod, ticks):
    """Whole ticks (4 substeps each) with Akinci tank walls: positions and velocities
    stay bitwise equal to the oracle tick after tick; per-body reactions are bitwise equal,
    the tank walls' spans above 8,192 particles (summed by a block each) included."""
    from vxl_sph import scenes
    spec = scenes.small_dam(n=(10, 12, 9), spacing=0.05, tank=(0.8, 0.7, 0.6))
    g, o = pair(vxl, oracle_mod, spec)
    dt_tick = float(F32(1.0) / F32(60.0))
    for t in range(ticks):
        rg = g.step_tick(dt_tick, spec.spans)
        o.step(dt_tick)
        compare_state(g, o, f"tick {t}")
        ro = o.reactions()
        assert [x[0] for x in rg] == [x[0] for x in ro]
        for (bid, fg, tg), (_, fo, to), (_, _, s0, s1) in zip(rg, ro, spec.spans):
            assert fg.tobytes() == fo.tobytes() and tg.tobytes() == to.tobytes(), (t, bid, s1 - s0, fg, fo, tg, to)
    compare_grid(g, o, "final grid")


@pytest.mark.parametrize("case", GOLDEN["cases"], ids=lambda c: f"n{c['n']}_bins{c['max_bins']}")
def test_published_hash_through_gpu(vxl, oracle_mod, case):
    """The reference's grid-probe scene run on the GPU: 5 + 1 ticks of the default
    config, then the FNV hash of the table of the last substep equals the published
    CPU hash (crates/vxl-phys-gpu/examples/gpu_grid_probe.rs:181-226) — for every published
    case, up to the 9,938,375-particle lattice, whose 2^20 cell budget doubles the bins (the
    half-culled density walk at full size)."""
    n = case["n"]
    s = F32(0.05)
    nf = F32(n)
    origin = (-nf * s * F32(0.5), F32(0.5), -nf * s * F32(0.5))
    from vxl_sph import scenes
    pos = scenes.fluid_block(origin, (n, n, n), 0.05)
    p = vxl.make_params(max_bins=case["max_bins"])
    p.particle_mass = vxl.lattice_mass(p, 0.05)
    g = vxl.Scene(p, pos, np.zeros_like(pos), np.full(pos.shape[0], F32(p.particle_mass)), pos.shape[0])
    dt_tick = float(F32(1.0) / F32(60.0))
    for _ in range(6):
        g.step_tick(dt_tick)
    items, start, bins, info = g.export_grid()
    h = oracle_mod.table_hash(start, items, pos.shape[0])
    assert h == int(case["hash"], 16), f"{h:#018x} != {case['hash']}"


def test_run_to_run_bitwise(vxl):
    from vxl_sph import scenes
    spec = scenes.dam0()

    def run():
        g = vxl.Scene(spec.params, spec.pos, spec.vel, spec.pmass, spec.n_fluid)
        react = []
        for _ in range(15):
            react.append(g.step_tick(float(F32(1) / F32(60)), spec.spans))
        p, v = g.read_state()
        g.close()
        return p.tobytes() + v.tobytes() + b"".join(np.concatenate([f, t]).tobytes() for r in react for _, f, t in r)

    assert run() == run()


def test_dam0_ticks_bit_exact(vxl, oracle_mod):
    """The 16,384-particle dam break (1-layer Akinci tank, 10 substeps) for 3 ticks."""
    from vxl_sph import scenes
    spec = scenes.dam0()
    g, o = pair(vxl, oracle_mod, spec)
    dt_tick = float(F32(1) / F32(60))
    for t in range(3):
        g.step_tick(dt_tick, spec.spans)
        o.step(dt_tick)
    compare_state(g, o, "dam0")
    compare_grid(g, o, "dam0")


def test_dam1_full_size_one_tick_bit_exact(vxl, oracle_mod):
    """1,000,000 fluid particles at full size: one tick (10 substeps) bitwise equal, the
    tank walls' per-body reactions (spans of 42,816-83,216 particles, a block each) too."""
    from vxl_sph import scenes
    spec = scenes.dam1()
    assert max(e - s for _, _, s, e in spec.spans) > 8192
    g, o = pair(vxl, oracle_mod, spec, threads=16)
    dt_tick = float(F32(1) / F32(60))
    rg = g.step_tick(dt_tick, spec.spans)
    o.step(dt_tick)
    compare_state(g, o, "dam1")
    compare_grid(g, o, "dam1")
    ro = o.reactions()
    assert [x[0] for x in rg] == [x[0] for x in ro]
    for (bid, fg, tg), (_, fo, to) in zip(rg, ro):
        assert fg.tobytes() == fo.tobytes() and tg.tobytes() == to.tobytes(), (bid, fg, fo, tg, to)


# ---------------------------------------------------------------- edge cases

def _custom(vxl, pos, vel=None, h=0.1, spacing=0.05, max_bins=0, boundary=None, **over):
    """Scene from explicit fluid (and optional boundary) arrays."""
    from vxl_sph import scenes
    p = vxl.make_params(smoothing_radius=h, max_bins=max_bins, **over)
    p.particle_mass = vxl.lattice_mass(p, spacing)
    pos = np.asarray(pos, F32).reshape(-1, 3)
    vel = np.zeros_like(pos) if vel is None else np.asarray(vel, F32).reshape(-1, 3)
    nf = pos.shape[0]
    pm = np.full(nf, F32(p.particle_mass), F32)
    spans = []
    if boundary is not None:
        bpos, bvel, bm, bsp = boundary
        pos = np.concatenate([pos, bpos]).astype(F32)
        vel = np.concatenate([vel, bvel]).astype(F32)
        pm = np.concatenate([pm, bm]).astype(F32)
        spans = [(b, o_, s + nf, e + nf) for b, o_, s, e in bsp]
    return scenes.SceneSpec("custom", p, pos, vel, pm, nf, spans, spacing, 1)


def _run_both(vxl, oracle_mod, spec, substeps=1):
    """The oracle and the GPU with each density kernel (per-particle walk, grouped segments)
    from identical state, `substeps` substeps, everything bit for bit."""
    o = oracle_mod.OracleSystem.from_scene(spec, threads=8)
    dt = f32_dt(4)
    for _ in range(substeps):
        o.substep(dt)
    r = o.read_f32()
    nf = spec.n_fluid
    for density in (0, 1):
        g = vxl.Scene(spec.params, spec.pos, spec.vel, spec.pmass, spec.n_fluid)
        g.set_tuning(256, 256, 0, density)
        g.set_record(True)
        for _ in range(substeps):
            g.substep(dt)
        compare_grid(g, o, f"density kernel {density}")
        dens, press, acc, xsph, bf = g.read_fields()
        assert_bits(dens, r["dens"], f"density (kernel {density})")
        assert_bits(acc[:nf], r["acc"][:nf], f"acc (kernel {density})")
        assert_bits(xsph[:nf], r["xsph"][:nf], f"xsph (kernel {density})")
        if spec.n_boundary:
            assert_bits(bf, r["bforce"][nf:], f"bforce (kernel {density})")
        compare_state(g, o, f"density kernel {density}")
    return g, o


def test_single_particle(vxl, oracle_mod):
    _run_both(vxl, oracle_mod, _custom(vxl, [[0.1, 0.2, 0.3]]), substeps=5)


def test_one_crowded_cell_canon_paths(vxl, oracle_mod):
    """Cells of > 32, > 512 and > 1024 particles take the shared-memory sort paths (keys and
    source slots staged; keys only) and the global one."""
    rng = np.random.default_rng(7)
    for n in (200, 800, 1500):
        pos = rng.uniform(0.0, 0.08, (n, 3)).astype(F32)
        _run_both(vxl, oracle_mod, _custom(vxl, pos, h=0.1), substeps=2)


def test_bin_budget_doubling(vxl, oracle_mod):
    """A small max_bins forces the reference's cell doubling (core/grid.rs:44-47)."""
    from vxl_sph import scenes
    pos = scenes.jitter(scenes.fluid_block((0, 0, 0), (12, 10, 8), 0.05), 0.05, 11)
    spec = _custom(vxl, pos, max_bins=64)
    g, o = _run_both(vxl, oracle_mod, spec, substeps=3)
    _, _, _, info = g.export_grid()
    assert info.bin > 0.1 and info.total <= 64


def test_far_apart_particles(vxl, oracle_mod):
    """Huge extent: per-axis dims clamp at 2^14 and the budget doubles many times."""
    pos = np.array([[-40.0, 0.0, -40.0], [40.0, 30.0, 40.0], [0.0, 1.0, 0.0], [0.01, 1.0, 0.0]], F32)
    _run_both(vxl, oracle_mod, _custom(vxl, pos), substeps=3)


def test_clamped_edge_cell_with_doubled_bins(vxl, oracle_mod):
    """A 1 km long scene at h = 0.01: the budget quadruples the bin to 0.04 and the x axis
    still hits the 16,384-cell cap, so every particle beyond x = 655.32 is clamped into the
    last x cell. Two clusters there (x = 900 and x = 1000) find their neighbours in that
    cell — the half-cell culling must not treat its upper face as a wall."""
    from vxl_sph import scenes
    s = 0.005
    blocks = [scenes.fluid_block(o, (4, 4, 4), s) for o in ((0.0, 0.0, 0.0), (900.0, 0.1, 0.1),
                                                          (999.98, 0.28, 0.28))]
    spec = _custom(vxl, np.concatenate(blocks), h=2 * s, spacing=s)
    lo, hi = spec.pos.min(0), spec.pos.max(0)
    _, bin_, dims = oracle_mod.grid_box(lo, hi, 2 * s)
    assert dims[0] == 16384 and bin_ >= 4 * s * 0.999, (bin_, dims)
    g, o = _run_both(vxl, oracle_mod, spec, substeps=2)
    dens, _, _, _, _ = g.read_fields()
    h = 2 * s
    self_only = spec.params.particle_mass * 315.0 / (64.0 * np.pi * h ** 3)  # mass * W(0)
    assert np.all(dens[64:] > 1.5 * self_only), "the clamped clusters found their neighbours"


def test_boundary_with_many_fluid_neighbours(vxl, oracle_mod):
    """h = 4 s gives boundary particles > 64 fluid neighbours (the gather's slow path)."""
    from vxl_sph import scenes
    s = 0.025
    fluid = scenes.fluid_block((0.0, 0.0, 0.0), (10, 8, 10), s)
    b = scenes.body_particles([scenes.Body(0, (0.2, 0.05, 0.2), (0.125, -0.05, 0.125))], s, 4 * s, 1, 1000.0)
    spec = _custom(vxl, fluid, h=4 * s, spacing=s, boundary=b)
    _run_both(vxl, oracle_mod, spec, substeps=2)


def test_boundary_only_scene_is_not_driven(vxl):
    """n_fluid == 0: the reference's substep returns immediately (fluid_step.rs:93-95)."""
    from vxl_sph import scenes
    b = scenes.body_particles([scenes.Body(0, (0.1, 0.1, 0.1), (0, 0, 0))], 0.05, 0.1, 1, 1000.0)
    p = vxl.make_params(particle_mass=1.0)
    g = vxl.Scene(p, b[0], b[1], b[2], 0)
    g.step_tick(1 / 60)
    pp, _ = g.read_state()
    assert pp.tobytes() == b[0].tobytes()


def test_upload_boundary_length_mismatch_is_an_error(vxl):
    from vxl_sph import scenes
    spec = scenes.small_dam()
    g = vxl.Scene(spec.params, spec.pos, spec.vel, spec.pmass, spec.n_fluid)
    with pytest.raises(vxl.VxlError) as e:
        g.upload_boundary(spec.pos[spec.n_fluid + 1:], spec.vel[spec.n_fluid + 1:])
    assert e.value.status == vxl.SIZE_MISMATCH


def test_stepper_mirror_moving_body(vxl, oracle_mod):
    """GpuFluidStepper mirror: each tick the facade re-uploads a moving body's boundary
    segment; the GPU tracks the oracle driven the same way, bit for bit."""
    from vxl_sph import scenes
    spec = scenes.small_dam(n=(8, 10, 8), spacing=0.05, tank=(0.8, 0.7, 0.6))
    box = scenes.Body(9, (0.06, 0.06, 0.06), (0.4, 0.45, 0.3), linvel=(0.0, -0.3, 0.0))
    bodies = scenes.tank_bodies(spec.meta["tank"], 0.1)
    cache = {}

    def boundary_at(t):
        b = scenes.Body(box.id, box.half, (0.4, 0.45 - 0.005 * t, 0.3), linvel=box.linvel)
        return scenes.body_particles(bodies + [b], 0.05, spec.params.smoothing_radius, 1, 1000.0, cache)

    bpos, bvel, bm, bsp = boundary_at(0)
    nf = spec.n_fluid
    pos = np.concatenate([spec.pos[:nf], bpos])
    vel = np.concatenate([spec.vel[:nf], bvel])
    pm = np.concatenate([spec.pmass[:nf], bm])
    spans = [(b, o_, s + nf, e + nf) for b, o_, s, e in bsp]
    st = vxl.GpuFluidStepper(spec.params, nf, pos, vel, pm)
    full = scenes.SceneSpec("m", spec.params, pos, vel, pm, nf, spans, 0.05, 1)
    o = oracle_mod.OracleSystem.from_scene(full, threads=8)
    dt_tick = float(F32(1) / F32(60))
    for t in range(4):
        bpos, bvel, bm, bsp = boundary_at(t)
        pos[nf:] = bpos
        vel[nf:] = bvel
        st.step(dt_tick, nf, pos, vel, pm, spans)
        o.set_boundary_raw(bpos, bvel, bm, spans)
        o.step(dt_tick)
    compare_state(st.scene, o, "stepper")
    lo, hi = st.bounds()
    fp = o.read_f32()["pos"][:nf]
    assert np.array_equal(lo, fp.min(0)) and np.array_equal(hi, fp.max(0))
    with pytest.raises(vxl.VxlError):
        st.step(dt_tick, nf, pos[:-1], vel[:-1], pm[:-1], spans)


def test_write_read_state_roundtrip(vxl):
    from vxl_sph import scenes
    spec = scenes.small_dam()
    g = vxl.Scene(spec.params, spec.pos, spec.vel, spec.pmass, spec.n_fluid)
    g.step_tick(1 / 60, spec.spans)
    rng = np.random.default_rng(3)
    p = (spec.pos + rng.normal(0, 1e-3, spec.pos.shape)).astype(F32)
    v = rng.normal(0, 0.1, spec.pos.shape).astype(F32)
    g.write_state(p, v)
    p2, v2 = g.read_state()
    assert p2.tobytes() == p.tobytes() and v2.tobytes() == v.tobytes()


def test_dam1_table_properties_and_determinism(vxl):
    """Size-independent properties at the full 1M workload after several ticks."""
    from vxl_sph import scenes
    spec = scenes.dam1()
    g = vxl.Scene(spec.params, spec.pos, spec.vel, spec.pmass, spec.n_fluid)
    for _ in range(3):
        g.step_tick(1 / 60, spec.spans)
    items, start, bins, info = g.export_grid()
    nt = spec.n_total
    assert start[0] == 0 and start[-1] == nt and np.all(np.diff(start.astype(np.int64)) >= 0)
    assert np.array_equal(np.sort(items), np.arange(nt, dtype=np.uint32))
    cell_of_slot = np.repeat(np.arange(info.total, dtype=np.uint32), np.diff(start.astype(np.int64)))
    assert np.array_equal(bins[items], cell_of_slot)
    same = cell_of_slot[1:] == cell_of_slot[:-1]
    assert np.all(items[1:][same] > items[:-1][same]), "cell contents must ascend by particle index"
    p, v = g.read_state()
    assert np.isfinite(p).all() and np.isfinite(v).all()


def test_doubled_bins_many_per_cell(vxl, oracle_mod):
    """A cell budget that forces bins of 4h with ~500 particles per cell: the density pass
    culls half-cells out of reach and must still accept the same neighbours in the same
    order (table, fields and state bit for bit over six substeps)."""
    from vxl_sph import scenes
    s = 0.01
    fluid = scenes.fluid_block((0.0, 0.0, 0.0), (20, 16, 18), s)
    b = scenes.body_particles([scenes.Body(0, (0.12, 0.01, 0.11), (0.1, -0.01, 0.09))], s, 2 * s, 1, 1000.0)
    spec = _custom(vxl, fluid, h=2 * s, spacing=s, boundary=b, max_bins=64)
    _run_both(vxl, oracle_mod, spec, substeps=6)


def test_device_body_rebuild_equals_host_upload(vxl, oracle_mod):
    """Moving and rotating bodies: rebuilding the boundary segment on the device from the
    poses (vxl_sph_set_body_poses) gives, tick after tick, exactly the state and reactions
    of uploading the host-built segment (vxl_sph_upload_boundary) and of the oracle's
    set_boundary_particles."""
    from vxl_sph import scenes
    s = 0.02
    h = 2 * s
    tank = (0.6, 0.5, 0.4)
    walls = scenes.tank_bodies(tank, 2 * s)
    paddle = scenes.Body(9, (0.02, 0.12, 0.08), (0.42, 0.16, 0.2), rot=(0.0, 0.0, 0.0, 1.0),
                         linvel=(-0.3, 0.0, 0.05), angvel=(0.0, 1.5, 0.4))
    bodies = walls + [paddle]
    params = scenes.baseline_params(s, substeps=4)
    fluid = scenes.jitter(scenes.fluid_block((0.0, 0.0, 0.0), (10, 12, 10), s), s, 17)
    spec = scenes.assemble("paddle", params, fluid, bodies, s, 4)
    a = vxl.Scene(spec.params, spec.pos, spec.vel, spec.pmass, spec.n_fluid)
    b = vxl.Scene(spec.params, spec.pos, spec.vel, spec.pmass, spec.n_fluid)
    o = oracle_mod.OracleSystem.from_scene(spec, threads=4)
    local, idx = scenes.body_lattice(bodies, s, h, params.boundary_layers)
    b.set_body_lattice(local, idx, len(bodies))
    dt = float(np.float32(1.0) / np.float32(60.0))
    for t in range(4):
        # advance the paddle's pose on the host (the caller's rigid integrator)
        p = np.asarray(paddle.pos, F32) + np.asarray(paddle.linvel, F32) * F32(dt)
        ang = F32(0.05 * (t + 1))
        q = (0.0, float(np.sin(ang)), 0.0, float(np.cos(ang)))
        paddle = scenes.Body(9, paddle.half, tuple(float(x) for x in p), rot=q, linvel=paddle.linvel,
                             angvel=paddle.angvel)
        bodies = walls + [paddle]
        bpos, bvel, _, bsp = scenes.body_particles(bodies, s, h, params.boundary_layers, params.rest_density)
        spans = [(bb, org, st + spec.n_fluid, en + spec.n_fluid) for bb, org, st, en in bsp]
        a.upload_boundary(bpos, bvel)
        b.set_body_poses(bodies)
        o.set_bodies(bodies)
        ra = a.step_tick(dt, spans)
        rb = b.step_tick(dt, spans)
        o.step(dt)
        for (b1, f1, t1), (b2, f2, t2) in zip(ra, rb):
            assert b1 == b2 and f1.tobytes() == f2.tobytes() and t1.tobytes() == t2.tobytes()
        pa, va = a.read_state()
        pb, vb = b.read_state()
        assert_bits(pb, pa, f"tick {t} pos (device rebuild vs upload)")
        assert_bits(vb, va, f"tick {t} vel (device rebuild vs upload)")
        r = o.read_f32()
        assert_bits(pb, r["pos"], f"tick {t} pos vs oracle")
    o.close()


def _body_states(bodies, dynamic, density):
    from vxl_sph import scenes
    st = np.zeros((len(bodies), 18), F32)
    for q, b in enumerate(bodies):
        st[q, 0:3] = b.pos
        st[q, 3:7] = b.rot
        st[q, 7:10] = b.linvel
        st[q, 10:13] = b.angvel
        if dynamic[q]:
            im, ii = scenes.box_mass_props(b.half, density)
            st[q, 13] = im
            st[q, 14:17] = ii
            st[q, 17] = 1.0
    return st


def _floating_scene(seed=23, dims=(10, 12, 10), shift=(0.0, 0.0, 0.0)):
    """Tank walls (static) and two boxes (dynamic) floating in the fluid's top layers."""
    from vxl_sph import scenes
    s = 0.02
    tank = (0.6, 0.5, 0.4)
    walls = scenes.tank_bodies(tank, 2 * s)
    a = float(np.sin(F32(0.2)))
    c = float(np.cos(F32(0.2)))
    top = F32(dims[1]) * F32(s)
    sx, sy, sz = shift
    boxes = [scenes.Body(20, (0.05, 0.03, 0.04), (0.1 + sx, float(top) - 0.005, 0.1 + sz), rot=(0.0, a, 0.0, c),
                         angvel=(0.3, 0.0, -0.2)),
             scenes.Body(21, (0.03, 0.03, 0.03), (0.16 + sx, float(top) - 0.015 + sy, 0.06 + sz),
                         linvel=(0.0, -0.2, 0.1))]
    bodies = walls + boxes
    dynamic = [False] * len(walls) + [True] * len(boxes)
    params = scenes.baseline_params(s, substeps=4)
    fluid = scenes.jitter(scenes.fluid_block((0.0, 0.0, 0.0), dims, s), s, seed)
    spec = scenes.assemble("floating", params, fluid, bodies, s, 4)
    local, idx = scenes.body_lattice(bodies, s, 2 * s, params.boundary_layers)
    return spec, bodies, dynamic, local, idx


def _couple(g, spec, bodies, dynamic, local, idx, scene=0):
    st = _body_states(bodies, dynamic, 400.0)
    g.set_body_lattice(local, idx, len(bodies), scene=scene)
    g.set_rigid_bodies(bodies, st[:, 13], st[:, 14:17], dynamic, scene=scene)
    g.set_spans(spec.spans, scene=scene)
    return st


GRAVITY = np.array([0.0, -9.81, 0.0], F32)


@pytest.mark.parametrize("rigid_substeps", [2, 3])
def test_coupled_loop_on_device_equals_oracle_loop(vxl, oracle_mod, rigid_substeps):
    """Floating boxes driven by the fluid: vxl_sph_step_coupled (rigid substeps from the
    previous tick's reactions, boundary rebuilt from the new poses, one fluid tick — all on
    the device) gives, tick after tick, bitwise the bodies, the fluid state and the
    reactions of the same loop run on the host around the oracle (rigid substeps, then
    set_boundary_particles, then step)."""
    from vxl_sph import scenes
    spec, bodies, dynamic, local, idx = _floating_scene()
    boxes = [b for b, d in zip(bodies, dynamic) if d]
    g = vxl.Scene(spec.params, spec.pos, spec.vel, spec.pmass, spec.n_fluid)
    o = oracle_mod.OracleSystem.from_scene(spec, threads=4)
    st = _couple(g, spec, bodies, dynamic, local, idx)
    nspans = len(spec.spans)
    dt = float(F32(1.0) / F32(60.0))
    react = np.zeros((len(bodies), 6), F32)
    row = {b.id: q for q, b in enumerate(bodies)}
    felt = set()
    for t in range(5):
        oracle_mod.rigid_step(st, react, GRAVITY, float(F32(dt) / F32(rigid_substeps)), rigid_substeps, 100.0, 50.0)
        posed = [scenes.Body(b.id, b.half, tuple(float(x) for x in st[q, 0:3]), rot=tuple(float(x) for x in st[q, 3:7]),
                             linvel=tuple(float(x) for x in st[q, 7:10]), angvel=tuple(float(x) for x in st[q, 10:13]))
                 for q, b in enumerate(bodies)]
        o.set_bodies(posed)
        o.step(dt)
        ro = o.reactions()
        rg = g.step_coupled(dt, rigid_substeps, GRAVITY, 100.0, 50.0, nspans)
        dev = g.read_rigid_bodies()
        assert_bits(dev, st[:, :13], f"tick {t} rigid bodies")
        assert [x[0] for x in rg] == [x[0] for x in ro]
        react[:] = 0
        for (bid, fg, tg), (_, fo, to) in zip(rg, ro):
            if dynamic[row[bid]]:
                assert fg.tobytes() == fo.tobytes() and tg.tobytes() == to.tobytes(), (t, bid, fg, fo, tg, to)
                if np.any(fo != 0):
                    felt.add(bid)
            react[row[bid], 0:3] = fo
            react[row[bid], 3:6] = to
        r = o.read_f32()
        p, v = g.read_state()
        assert_bits(p, r["pos"], f"tick {t} pos")
        assert_bits(v, r["vel"], f"tick {t} vel")
    # the fluid pushed every box at some tick, and the boxes moved
    assert felt == {b.id for b in boxes}, felt
    assert np.all(np.abs(st[[row[b.id] for b in boxes], 0:3] - np.array([b.pos for b in boxes], F32)) > 0)
    o.close()
    g.close()


def test_coupled_loop_batched_equals_scenes_alone(vxl):
    """One vxl_sph_step_coupled over a batch of two floating scenes (different sizes) and one
    scene without rigid bodies equals each scene stepped alone (coupled or plain), bitwise:
    bodies, fluid state and reactions."""
    from vxl_sph import scenes
    a = _floating_scene(seed=5, dims=(10, 12, 10))
    b = _floating_scene(seed=9, dims=(14, 10, 9), shift=(0.2, 0.0, 0.1))
    plain = scenes.small_dam(n=(8, 9, 8), spacing=0.05, tank=(0.8, 0.7, 0.6), seed=3)
    bat = vxl.Batch([a[0], b[0], plain])
    alone = [vxl.Scene(x.params, x.pos, x.vel, x.pmass, x.n_fluid) for x in (a[0], b[0], plain)]
    for q, (x, sc) in enumerate(zip((a, b), alone)):
        _couple(bat, *x, scene=q)
        _couple(sc, *x)
    dt = float(F32(1.0) / F32(60.0))
    for t in range(4):
        bat.step_coupled(dt, 2, GRAVITY)
        rb = bat.reactions()
        ra = []
        for q in range(2):
            ra += alone[q].step_coupled(dt, 2, GRAVITY, nspans=len((a, b)[q][0].spans))
        ra += alone[2].step_tick(dt, plain.spans)
        assert len(ra) == len(rb)
        for (b1, f1, t1), (b2, f2, t2) in zip(ra, rb):
            assert b1 == b2 and f1.tobytes() == f2.tobytes() and t1.tobytes() == t2.tobytes(), (t, b1)
        for q in range(3):
            p1, v1 = bat.read_state(q)
            p2, v2 = alone[q].read_state()
            assert_bits(p1, p2, f"tick {t} scene {q} pos")
            assert_bits(v1, v2, f"tick {t} scene {q} vel")
        for q in range(2):
            assert_bits(bat.read_rigid_bodies(q), alone[q].read_rigid_bodies(), f"tick {t} scene {q} bodies")
    bat.close()
    for sc in alone:
        sc.close()


def test_deferred_readback_and_vxld_dump(vxl, oracle_mod, tmp_path):
    """vxl_sph_request_state / vxl_sph_take_state return the state that vxl_sph_read_state
    returns, and a VXLD dump's frames are the oracle's fluid positions at those ticks."""
    from vxl_sph import export, scenes
    spec = scenes.small_dam(n=(8, 10, 8), spacing=0.05, tank=(0.8, 0.7, 0.6), seed=4)
    g = vxl.Scene(spec.params, spec.pos, spec.vel, spec.pmass, spec.n_fluid)
    dt = float(F32(1.0) / F32(60.0))
    g.step_tick(dt, spec.spans)
    g.request_state()
    p1 = g.take_state()
    p2, _ = g.read_state()
    assert_bits(p1, p2, "take_state vs read_state")
    g.close()
    g = vxl.Scene(spec.params, spec.pos, spec.vel, spec.pmass, spec.n_fluid)
    path = str(tmp_path / "dam.bin")
    info = export.dump_run(g, path, ticks=6, dt_tick=dt, spans=spec.spans)
    assert info["frames"] == 3
    r = export.read_vxld(path)
    o = oracle_mod.OracleSystem.from_scene(spec, threads=4)
    for t in range(1, 7):
        o.step(dt)
        if t % 2 == 0:
            fr = r["frames"][t // 2 - 1]
            assert fr["tick"] == t
            assert_bits(fr["systems"][0], o.read_f32()["pos"][:spec.n_fluid], f"frame at tick {t}")
    o.close()


def test_canon_window_at_its_limit(vxl, oracle_mod):
    """Sixteen particles per cell (two interleaved lattices at spacing h/2): 32 consecutive
    cells hold exactly 512 entries, the limit of the sort's window path, and cells at the
    block's edges fall back to the per-cell path; the table, fields and state stay bit-exact."""
    from vxl_sph import scenes
    s = 0.025
    a = scenes.fluid_block((0.0, 0.0, 0.0), (12, 10, 32), s)
    b = (a + F32(0.3 * s)).astype(F32)
    fluid = np.concatenate([a, b]).astype(F32)
    spec = _custom(vxl, fluid, h=2 * s, spacing=s)
    _run_both(vxl, oracle_mod, spec, substeps=2)
