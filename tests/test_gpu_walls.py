"""Provider walls on the device against the oracle, through the C ABI (B200).

Mirror ghosts in the density, projection after integration and the coincident-particle
separation, with the fluid crate's FloorY / Tank providers and a convex box obstacle: the
state stays bitwise equal to the oracle (which passes the reference's own provider tests,
test_oracle_walls.py) tick after tick.
"""
import numpy as np
import pytest

from test_gpu_parity import _custom, assert_bits, compare_grid, pair

pytestmark = pytest.mark.gpu
F32 = np.float32


def _run(vxl, oracle_mod, spec, providers, ticks, check_every=1):
    g, o = pair(vxl, oracle_mod, spec, threads=4)
    g.set_providers(providers)
    o.set_providers(providers)
    dt = float(F32(1.0) / F32(60.0))
    for t in range(ticks):
        g.step_tick(dt, spec.spans)
        o.step(dt)
        if (t + 1) % check_every == 0 or t + 1 == ticks:
            p, v = g.read_state()
            r = o.read_f32()
            assert_bits(p, r["pos"], f"tick {t} pos")
            assert_bits(v, r["vel"], f"tick {t} vel")
    return g, o


def _block(vxl, origin, dims, xsph=0.05):
    from vxl_sph import scenes
    pos = scenes.fluid_block(origin, dims, 0.05)
    return _custom(vxl, pos, h=0.1, spacing=0.05, xsph_viscosity=xsph)


def test_block_falls_onto_floor_provider(vxl, oracle_mod):
    """A 5^3 block dropped from y = 0.3 onto FloorY: impact, projection and mirror ghosts."""
    from vxl_sph import scenes
    spec = _block(vxl, (-0.1, 0.3, -0.1), (5, 5, 5))
    g, o = _run(vxl, oracle_mod, spec, [scenes.floor_provider()], ticks=40)
    y = g.read_state()[0][:, 1]
    assert y.min() > -0.01 and y.min() < 0.1, y.min()  # it landed and did not sink
    g.set_record(True)
    dt = float(F32(F32(1.0) / F32(60.0)) / F32(spec.params.substeps))
    g.substep(dt)
    o.substep(dt)
    compare_grid(g, o, "grid after landing")
    dens = g.read_fields()[0]
    assert_bits(dens, o.read_f32()["dens"], "density with mirror ghosts")
    o.close()
    g.close()


def test_column_in_tank_provider(vxl, oracle_mod):
    """The 7^3 column of the reference's hydrostatic test in the Tank provider (five faces)."""
    from vxl_sph import scenes
    spec = _block(vxl, (-0.15, 0.05, -0.15), (7, 7, 7))
    g, o = _run(vxl, oracle_mod, spec, [scenes.tank_provider()], ticks=30, check_every=5)
    o.close()
    g.close()


def test_block_lands_on_convex_obstacle(vxl, oracle_mod):
    """A block falling onto a convex box obstacle standing on FloorY: the decisive-plane
    contacts of the half-space set, and two providers per particle."""
    from vxl_sph import scenes
    spec = _block(vxl, (-0.15, 0.35, -0.1), (7, 4, 5))
    walls = [scenes.floor_provider(), scenes.box_obstacle((0.0, 0.1, 0.0), (0.06, 0.1, 0.06))]
    g, o = _run(vxl, oracle_mod, spec, walls, ticks=40, check_every=4)
    o.close()
    g.close()


def test_coincident_pushed_particles_are_separated(vxl, oracle_mod):
    """Two isolated particles 1e-4 apart inside the floor: both are projected to the same
    height, then the later one is moved 0.2 h - r along its normal (separate_coincident)."""
    from vxl_sph import scenes
    pos = np.array([[0.0, -0.001, 0.0], [0.0001, -0.001, 0.0], [0.5, 0.5, 0.5]], F32)
    spec = _custom(vxl, pos, h=0.1, spacing=0.05)
    g, o = pair(vxl, oracle_mod, spec, threads=1)
    g.set_providers([scenes.floor_provider()])
    o.set_providers([scenes.floor_provider()])
    dt = float(F32(F32(1.0) / F32(60.0)) / F32(4))
    g.substep(dt)
    o.substep(dt)
    p, v = g.read_state()
    r = o.read_f32()
    assert_bits(p, r["pos"], "pos")
    assert_bits(v, r["vel"], "vel")
    assert p[1, 1] - p[0, 1] > 0.019, p[:2]  # the separation ran
    for _ in range(7):
        g.substep(dt)
        o.substep(dt)
    assert_bits(g.read_state()[0], o.read_f32()["pos"], "pos after 8 substeps")
    o.close()
    g.close()


def test_batch_with_and_without_providers_equals_alone(vxl):
    """A batch of a scene with provider walls and one without equals each stepped alone."""
    from vxl_sph import scenes
    a = _block(vxl, (-0.1, 0.2, -0.1), (5, 6, 5))
    b = scenes.small_dam(n=(8, 9, 8), spacing=0.05, tank=(0.8, 0.7, 0.6), seed=3)
    bat = vxl.Batch([a, b])
    bat.set_providers([scenes.tank_provider()], scene=0)
    ga = vxl.Scene(a.params, a.pos, a.vel, a.pmass, a.n_fluid)
    ga.set_providers([scenes.tank_provider()])
    gb = vxl.Scene(b.params, b.pos, b.vel, b.pmass, b.n_fluid)
    dt = float(F32(1.0) / F32(60.0))
    for t in range(6):
        bat.step_tick(dt)
        ga.step_tick(dt)
        gb.step_tick(dt, b.spans)
        for q, sc in ((0, ga), (1, gb)):
            p1, v1 = bat.read_state(q)
            p2, v2 = sc.read_state()
            assert_bits(p1, p2, f"tick {t} scene {q} pos")
            assert_bits(v1, v2, f"tick {t} scene {q} vel")
    # removing the providers returns the scene to the plain path
    bat.set_providers([], scene=0)
    ga.set_providers([])
    bat.step_tick(dt)
    ga.step_tick(dt)
    assert_bits(bat.read_state(0)[0], ga.read_state()[0], "after removing the providers")
    for x in (bat, ga, gb):
        x.close()


def test_set_providers_rejects_bad_input(vxl):
    from vxl_sph import scenes
    spec = _block(vxl, (0.0, 0.2, 0.0), (3, 3, 3))
    g = vxl.Scene(spec.params, spec.pos, spec.vel, spec.pmass, spec.n_fluid)
    bad = [vxl.Faces([(3, 0.0, 1.0)]), vxl.Faces([(1, 0.0, 2.0)]), vxl.Faces([(1, float("nan"), 1.0)]),
           vxl.Convex([((float("inf"), 0.0, 0.0), 0.0)])]
    for pr in bad:
        with pytest.raises(vxl.VxlError) as e:
            g.set_providers([pr])
        assert e.value.status == vxl.INVALID_ARGUMENT
    with pytest.raises(vxl.VxlError):
        g.set_providers([scenes.floor_provider()], scene=3)
    g.set_providers([scenes.floor_provider()])  # still usable
    g.step_tick(float(F32(1.0) / F32(60.0)))
    g.close()


def test_coupled_loop_with_provider_floor(vxl, oracle_mod):
    """The device coupling loop (floating boxes) on a handle that also has a provider floor:
    bodies and fluid stay bitwise equal to the oracle loop with the same provider."""
    from test_gpu_parity import GRAVITY, _couple, _floating_scene
    from vxl_sph import scenes
    spec, bodies, dynamic, local, idx = _floating_scene()
    floor = [vxl.Faces([(1, 0.01, 1.0)], ((-50.0, -1.0, -50.0), (50.0, 0.01, 50.0)))]
    g = vxl.Scene(spec.params, spec.pos, spec.vel, spec.pmass, spec.n_fluid)
    o = oracle_mod.OracleSystem.from_scene(spec, threads=4)
    g.set_providers(floor)
    o.set_providers(floor)
    st = _couple(g, spec, bodies, dynamic, local, idx)
    dt = float(F32(1.0) / F32(60.0))
    react = np.zeros((len(bodies), 6), F32)
    row = {b.id: q for q, b in enumerate(bodies)}
    for t in range(4):
        oracle_mod.rigid_step(st, react, GRAVITY, float(F32(dt) / F32(2)), 2, 100.0, 50.0)
        posed = [scenes.Body(b.id, b.half, tuple(float(x) for x in st[q, 0:3]), rot=tuple(float(x) for x in st[q, 3:7]),
                             linvel=tuple(float(x) for x in st[q, 7:10]), angvel=tuple(float(x) for x in st[q, 10:13]))
                 for q, b in enumerate(bodies)]
        o.set_bodies(posed)
        o.step(dt)
        g.step_coupled(dt, 2, GRAVITY, 100.0, 50.0, 0)
        assert_bits(g.read_rigid_bodies(), st[:, :13], f"tick {t} bodies")
        for bid, fo, to in o.reactions():
            react[row[bid], 0:3] = fo
            react[row[bid], 3:6] = to
        p, v = g.read_state()
        r = o.read_f32()
        assert_bits(p, r["pos"], f"tick {t} pos")
        assert_bits(v, r["vel"], f"tick {t} vel")
    o.close()
    g.close()


def test_provider_walls_at_doubled_bins(vxl, oracle_mod):
    """Provider walls with a cell budget that doubles the bins (the half-culled density walk
    with mirror ghosts, and the x-half thread order): bitwise with the oracle."""
    from vxl_sph import scenes
    pos = scenes.jitter(scenes.fluid_block((-0.3, 0.05, -0.2), (12, 10, 8), 0.05), 0.05, 5)
    spec = _custom(vxl, pos, h=0.1, spacing=0.05, max_bins=64, xsph_viscosity=0.05)
    walls = [scenes.floor_provider(), scenes.box_obstacle((0.0, 0.08, 0.0), (0.08, 0.08, 0.08))]
    g, o = _run(vxl, oracle_mod, spec, walls, ticks=12, check_every=3)
    _, _, _, info = g.export_grid()
    assert info.bin >= 0.2 * 0.999, info.bin  # bins of at least 2h
    o.close()
    g.close()


def test_batch_mixing_doubled_and_h_bins(vxl):
    """One batch holding a scene whose bins doubled and one at h-sized bins equals each
    scene stepped alone, bitwise."""
    from vxl_sph import scenes
    pos = scenes.jitter(scenes.fluid_block((0.0, 0.0, 0.0), (12, 10, 8), 0.05), 0.05, 11)
    a = _custom(vxl, pos, h=0.1, spacing=0.05, max_bins=64)
    b = scenes.small_dam(n=(8, 9, 8), spacing=0.05, tank=(0.8, 0.7, 0.6), seed=3)
    bat = vxl.Batch([a, b])
    alone = [vxl.Scene(x.params, x.pos, x.vel, x.pmass, x.n_fluid) for x in (a, b)]
    dt = float(F32(1.0) / F32(60.0))
    for t in range(5):
        bat.step_tick(dt)
        alone[0].step_tick(dt)
        alone[1].step_tick(dt, b.spans)
        for q in range(2):
            p1, v1 = bat.read_state(q)
            p2, v2 = alone[q].read_state()
            assert_bits(p1, p2, f"tick {t} scene {q} pos")
            assert_bits(v1, v2, f"tick {t} scene {q} vel")
    assert bat.export_grid(0)[3].bin > 0.1 and bat.export_grid(1)[3].bin <= 0.1 + 1e-6
    for x in [bat] + alone:
        x.close()
