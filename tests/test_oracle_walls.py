"""The oracle's provider walls against the reference's own tests of them (CPU).

The oracle restates the provider tier of the fluid step (mirror ghosts in the density,
boundary_pass and separate_coincident after integration) with the fluid crate's FloorY and
Tank test providers. These tests are the reference's provider tests run on the oracle, with
their thresholds (crates/vxl-phys-fluid/src/tests.rs:155-223 and :273-289); the GPU path is
compared with the oracle bit for bit in test_gpu_walls.py.
"""
import numpy as np

F32 = np.float32


def _system(oracle_mod, origin, dims, providers, **cfg):
    c = oracle_mod.default_cfg(**cfg)
    o = oracle_mod.OracleSystem(c, origin=origin, dims=dims, spacing=0.05)
    o.set_providers(providers)
    return o


def test_particles_rest_on_floor_provider_without_penetration(oracle_mod):
    """tests.rs:273-289: a 5^3 block dropped from y = 1.2 onto FloorY for 300 ticks neither
    sinks below -0.01 nor bounces above 0.6."""
    from vxl_sph import scenes
    o = _system(oracle_mod, (-0.1, 1.2, -0.1), (5, 5, 5), [scenes.floor_provider()], xsph_viscosity=0.05)
    dt = float(F32(1.0) / F32(60.0))
    for _ in range(300):
        o.step(dt)
    y = o.read_f32()["pos"][:, 1]
    assert np.all(y > -0.01), y.min()
    assert np.all(y < 0.6), y.max()
    o.close()


def test_hydrostatic_pressure_increases_with_depth_in_tank_provider(oracle_mod):
    """tests.rs:155-223: a 7^3 column settles in the Tank provider for 240 ticks; column height
    0.20-0.32 m, pressure rising with depth in thirds, the middle third within 0.4-1.1 of
    rho0 g H / 2, the bottom below twice its hydrostatic reference, the top under a third of
    the middle, speeds below 3 m/s."""
    from vxl_sph import scenes
    o = _system(oracle_mod, (-0.15, 0.05, -0.15), (7, 7, 7), [scenes.tank_provider()], xsph_viscosity=0.05)
    dt = float(F32(1.0) / F32(60.0))
    for _ in range(240):
        o.step(dt)
    r = o.read_f32()
    y = r["pos"][:, 1]
    height = float(y.max() - y.min())
    assert 0.20 < height < 0.32, height
    t = (y - y.min()) / height
    pr = r["press"]
    lo, mid, hi = pr[t < 1 / 3].mean(), pr[(t >= 1 / 3) & (t < 2 / 3)].mean(), pr[t >= 2 / 3].mean()
    assert lo > mid > hi, (lo, mid, hi)
    mid_ref = 1000.0 * 9.81 * 0.5 * height
    assert 0.4 * mid_ref < mid < 1.1 * mid_ref, (mid, mid_ref)
    assert lo < 2.0 * 1000.0 * 9.81 * height * 5.0 / 6.0, lo
    assert hi * 3.0 < mid, (hi, mid)
    assert np.all((r["vel"] ** 2).sum(1) < 9.0)
    o.close()


def test_walls_change_the_density_only_near_them(oracle_mod):
    """Mirror ghosts: a block standing on FloorY (layers at y = 0.025, 0.075, ...; h = 0.1)
    gains density only in its bottom layer, whose neighbours' mirror images lie within h;
    every other layer's density is the same bit for bit as without providers."""
    from vxl_sph import scenes
    a = _system(oracle_mod, (-0.1, 0.0, -0.1), (5, 5, 5), [scenes.floor_provider()])
    b = _system(oracle_mod, (-0.1, 0.0, -0.1), (5, 5, 5), [])
    y0 = a.read()["pos"][:, 1].copy()
    dt = float(F32(1.0) / F32(240.0))
    a.substep(dt)
    b.substep(dt)
    da, db = a.read_f32()["dens"], b.read_f32()["dens"]
    bottom = y0 < 0.05
    assert np.all(da[bottom] > db[bottom])
    assert da[~bottom].tobytes() == db[~bottom].tobytes()
    a.close()
    b.close()


def test_projection_and_separation_against_a_direct_restatement(oracle_mod):
    """Two isolated particles 1e-4 apart inside FloorY, one substep: no pressure (the Tait
    pressure clamps at 0), no viscosity or XSPH (equal velocities), so each integrates
    gravity, is projected out of the floor (boundary_pass, fluid_boundary.rs:45-101) and the
    later one is separated from the earlier (separate_coincident, :103-128). The oracle's
    result equals this float32 restatement of those three steps bit for bit."""
    from vxl_sph import scenes
    f = F32
    c = oracle_mod.default_cfg()
    o = oracle_mod.OracleSystem(c, origin=(0.0, 0.0, 0.0), dims=(2, 1, 1), spacing=0.05)
    p0 = np.array([[0.0, -0.001, 0.0], [0.0001, -0.001, 0.0]], F32)
    o.set_state(p0, np.zeros_like(p0))
    o.set_providers([scenes.floor_provider()])
    dt = f(f(f(1.0) / f(60.0)) / f(4.0))
    o.substep(float(dt))
    got = o.read_f32()
    h, eps, g = f(0.1), f(c.xsph_viscosity), f(-9.81)
    skin = f(0.15) * h
    vmax = f(0.4) * h / dt
    pos, vel = [], []
    for p in p0:
        # v = vel + acc dt + xsph eps with acc = gravity, vel = xsph = 0 (fluid_step.rs:112-123)
        v = np.array([f(f(0.0) + f(0.0) * dt) + f(0.0) * eps, f(f(0.0) + g * dt) + f(0.0) * eps,
                      f(f(0.0) + f(0.0) * dt) + f(0.0) * eps], F32)
        assert f(f(v[0] * v[0] + v[1] * v[1]) + v[2] * v[2]) <= vmax * vmax
        q = np.array([p[a] + v[a] * dt for a in range(3)], F32)
        # FloorY contact at (x, 0, z), normal +y; sdf = (q - point) . n
        sdf = f(f(f(q[0] - q[0]) * f(0.0) + f(q[1] - f(0.0)) * f(1.0)) + f(q[2] - q[2]) * f(0.0))
        pen = -sdf
        assert pen > 0
        m = min(f(pen + skin), h)
        q = np.array([q[0] + f(0.0) * m, q[1] + f(1.0) * m, q[2] + f(0.0) * m], F32)
        vn = f(f(v[0] * f(0.0) + v[1] * f(1.0)) + v[2] * f(0.0))
        if vn < 0:
            v = np.array([v[0] - f(0.0) * vn, v[1] - f(1.0) * vn, v[2] - f(0.0) * vn], F32)
        pos.append(q)
        vel.append(v)
    # the later particle moves along its normal sum (0, 1, 0) until r_min from the earlier one
    r_min = f(0.2) * h
    inv = f(1.0) / np.sqrt(f(f(f(0.0) + f(1.0)) + f(0.0)), dtype=F32)
    d = np.array([pos[1][a] - pos[0][a] for a in range(3)], F32)
    r2 = f(f(d[0] * d[0] + d[1] * d[1]) + d[2] * d[2])
    assert r2 < r_min * r_min
    r = np.sqrt(r2, dtype=F32)
    step = f(r_min - r)
    pos[1] = np.array([pos[1][a] + f(n * inv) * step for a, n in enumerate((f(0.0), f(1.0), f(0.0)))], F32)
    assert got["pos"].astype(F32).tobytes() == np.array(pos, F32).tobytes(), (got["pos"], pos)
    assert got["vel"].astype(F32).tobytes() == np.array(vel, F32).tobytes(), (got["vel"], vel)
    o.close()


def test_mirror_ghost_density_against_a_direct_restatement(oracle_mod):
    """One fluid particle 0.03 above FloorY with one neighbour: its density is
    mass (w0 + W(r) + W(|pi - g|)) with g the neighbour mirrored in the floor plane collected
    by wall_planes_in (fluid_density.rs:25-47, 76-118), each term in the reference's order;
    the neighbour, 0.04 up, gets its own ghost of the first. Bit for bit."""
    from vxl_sph import scenes
    f = F32
    c = oracle_mod.default_cfg()
    o = oracle_mod.OracleSystem(c, origin=(0.0, 0.0, 0.0), dims=(2, 1, 1), spacing=0.05)
    p0 = np.array([[0.0, 0.03, 0.0], [0.02, 0.04, 0.01]], F32)
    o.set_state(p0, np.zeros_like(p0))
    o.set_providers([scenes.floor_provider()])
    k = o.consts()
    o.substep(float(f(f(1.0) / f(240.0))))
    got = o.read_f32()["dens"]
    h, h2, k6, w0, mass = k["h"], k["h2"], k["k6"], k["w0"], k["mass"]

    def W(r2):
        t = f(h2 - r2)
        return f(f(f(k6 * t) * t) * t)

    want, ghosts = [], 0
    for i, j in ((0, 1), (1, 0)):
        pi, pj = p0[i], p0[j]
        d = np.array([pi[a] - pj[a] for a in range(3)], F32)
        r2 = f(f(d[0] * d[0] + d[1] * d[1]) + d[2] * d[2])
        total = f(w0 + W(r2))
        # the plane: contact (pi.x, 0, pi.z), normal +y; sdf = pi.y in (0, h)
        q = np.array([pi[a] - d[a] for a in range(3)], F32)  # pj as pi - d
        dn = f(f(f(q[0] - pi[0]) * f(0.0) + f(q[1] - f(0.0)) * f(1.0)) + f(q[2] - pi[2]) * f(0.0))
        gpt = np.array([q[0] - f(0.0) * f(f(2.0) * dn), q[1] - f(1.0) * f(f(2.0) * dn), q[2] - f(0.0) * f(f(2.0) * dn)], F32)
        e = np.array([pi[a] - gpt[a] for a in range(3)], F32)
        rg2 = f(f(e[0] * e[0] + e[1] * e[1]) + e[2] * e[2])
        if rg2 <= h2:
            total = f(total + W(rg2))
            ghosts += 1
        want.append(f(f(mass * total) + f(0.0)))
    assert ghosts == 2
    assert np.asarray(got, F32)[:2].tobytes() == np.array(want, F32).tobytes(), (got, want)
    o.close()


def test_convex_provider_decisive_plane_ghost_against_a_direct_restatement(oracle_mod):
    """Two particles 0.02 and 0.03 off the +x face of a convex box obstacle (HalfSpaceSet): the plane of
    largest n.p - d decides (plane_set.rs:60-76), its contact point p - n (n.p - d) and
    normal give the mirror plane; the particle's density with one neighbour is
    mass (w0 + W(r) + W(|pi - g|)) in the reference's order, bit for bit."""
    from vxl_sph import scenes
    f = F32
    c = oracle_mod.default_cfg()
    o = oracle_mod.OracleSystem(c, origin=(0.0, 0.0, 0.0), dims=(2, 1, 1), spacing=0.05)
    p0 = np.array([[0.07, 0.1, 0.0], [0.08, 0.11, 0.01]], F32)  # the box spans x in [-0.05, 0.05]
    o.set_state(p0, np.zeros_like(p0))
    box = scenes.box_obstacle((0.0, 0.1, 0.0), (0.05, 0.1, 0.05))
    o.set_providers([box])
    k = o.consts()
    o.substep(float(f(f(1.0) / f(240.0))))
    got = o.read_f32()["dens"]
    h, h2, k6, w0, mass = k["h"], k["h2"], k["k6"], k["w0"], k["mass"]

    def W(r2):
        t = f(h2 - r2)
        return f(f(f(k6 * t) * t) * t)

    def dot(a, b):
        return f(f(f(a[0] * b[0]) + f(a[1] * b[1])) + f(a[2] * b[2]))

    planes = [(np.array(n, F32), f(d)) for n, d in box.planes]
    want, ghosts = [], 0
    for i, j in ((0, 1), (1, 0)):
        pi, pj = p0[i], p0[j]
        ss = [f(dot(n, pi) - d) for n, d in planes]
        kb = int(np.argmax(ss))  # first maximum, like the strict > scan
        n, d = planes[kb]
        t = f(dot(n, pi) - d)
        point = np.array([pi[a] - f(n[a] * t) for a in range(3)], F32)
        sdf = dot(np.array([pi[a] - point[a] for a in range(3)], F32), n)
        dvec = np.array([pi[a] - pj[a] for a in range(3)], F32)
        total = f(w0 + W(dot(dvec, dvec)))
        if f(0.0) < sdf < h:
            q = np.array([pi[a] - dvec[a] for a in range(3)], F32)
            dn = dot(np.array([q[a] - point[a] for a in range(3)], F32), n)
            gpt = np.array([q[a] - f(n[a] * f(f(2.0) * dn)) for a in range(3)], F32)
            e = np.array([pi[a] - gpt[a] for a in range(3)], F32)
            rg2 = dot(e, e)
            if rg2 <= h2:
                total = f(total + W(rg2))
                ghosts += 1
        want.append(f(f(mass * total) + f(0.0)))
    assert ghosts == 2  # each particle's neighbour has a mirror image within h
    assert np.asarray(got, F32)[:2].tobytes() == np.array(want, F32).tobytes(), (got, want)
    o.close()


def _still_box(bid, half, pos):
    from vxl_sph import scenes
    return scenes.Body(bid, half, pos)


def test_boundary_particles_hold_fluid_column(oracle_mod):
    """tests.rs:439-476: a 12x12x10 block on an Akinci floor (a box body, no providers) for 60
    ticks stays finite and its core does not leak below -0.06."""
    o = _system(oracle_mod, (-0.3, 0.0, -0.3), (12, 12, 10), [])
    floor = [_still_box(0, (0.5, 0.05, 0.5), (0.0, -0.05, 0.0))]
    assert o.set_bodies(floor) > 0
    dt = float(F32(1.0) / F32(60.0))
    for _ in range(60):
        o.set_bodies(floor)
        o.step(dt)
    p = o.read_f32()["pos"][:o.n_fluid]
    assert np.all(np.isfinite(p))
    core = (np.abs(p[:, 0]) <= 0.25) & (np.abs(p[:, 2]) <= 0.25)
    assert p[core, 1].min() > -0.06, p[core, 1].min()
    o.close()


def test_submerged_box_gets_buoyant_reaction(oracle_mod):
    """tests.rs:492-561: a box (half 0.06) held in a 7^3 column in the Tank provider: over a
    60-tick window after 180 ticks of settling, the mean reaction on it is 0.5-2 rho V g up,
    its sideways components and torque near zero — the Akinci reactions and the provider
    walls together (the oracle gives 1.07 rho V g up)."""
    from vxl_sph import scenes
    o = _system(oracle_mod, (-0.15, 0.05, -0.15), (7, 7, 7), [scenes.tank_provider()], xsph_viscosity=0.05)
    half = 0.06
    body = [_still_box(7, (half, half, half), (0.0, 0.12, 0.0))]
    dt = float(F32(1.0) / F32(60.0))
    for _ in range(180):
        o.set_bodies(body)
        o.step(dt)
    f_sum, t_sum = np.zeros(3), np.zeros(3)
    for _ in range(60):
        o.set_bodies(body)
        o.step(dt)
        r = [x for x in o.reactions() if x[0] == 7][0]
        f_sum += r[1]
        t_sum += r[2]
    force, tau = f_sum / 60, t_sum / 60
    expect = 1000.0 * (2 * half) ** 3 * 9.81
    assert 0.5 * expect < force[1] < 2.0 * expect, (force, expect)
    assert abs(force[0]) < 0.5 * expect and abs(force[2]) < 0.5 * expect, force
    assert np.linalg.norm(tau) < 0.5 * expect * half, tau
    o.close()


class _FloorSdf:
    """A floor y = 0 answered as a host-side provider (closest point and normal), the same
    contacts the fluid crate's FloorY face provider reports (tests.rs:9-44, 81-110)."""

    def bounds(self, bid):
        return ((-50.0, -1.0, -50.0), (50.0, 0.0, 50.0))

    def contacts_point(self, bid, p, probe):
        if p[1] > F32(2) * F32(probe):
            return []
        return [(np.array([p[0], 0.0, p[2]], F32), np.array([0.0, 1.0, 0.0], F32))]


def test_contact_tables_equal_the_floor_provider_at_one_substep(oracle_mod):
    """With one substep per tick a table gathered each tick from the current positions is
    exactly the provider's answer for that substep, so the table-driven oracle (the GPU
    tier's gather, crates/vxl-phys-gpu/src/pipeline/walls.rs:164-215) and the oracle that
    queries FloorY itself give the same state bit for bit through landing and rest."""
    from vxl_sph import scenes, walls
    a = _system(oracle_mod, (-0.1, 0.3, -0.1), (5, 5, 5), [scenes.floor_provider()], xsph_viscosity=0.05,
                substeps=1)
    b = _system(oracle_mod, (-0.1, 0.3, -0.1), (5, 5, 5), [], xsph_viscosity=0.05, substeps=1)
    h = 0.1
    dt = float(F32(1.0) / F32(60.0))
    entries = 0
    for t in range(60):
        ps = b.read_f32()["pos"]
        for side in (walls.MIRROR, walls.PROJECT):
            ids, start, planes = walls.gather_contacts([0], h, ps, _FloorSdf(), side)
            entries = max(entries, ids.shape[0])
            b.set_wall_contacts(side, ids, start, planes)
        a.step(dt)
        b.step(dt)
        ra, rb = a.read_f32(), b.read_f32()
        assert ra["pos"].tobytes() == rb["pos"].tobytes(), f"tick {t}"
        assert ra["vel"].tobytes() == rb["vel"].tobytes(), f"tick {t}"
    assert entries > 20
    assert ra["pos"][:, 1].min() > -0.01
    a.close()
    b.close()


def test_gather_contacts_rules():
    """Mirror keeps 0 < sdf < h, projection sdf < h, at most 8 planes, bounds grown by h."""
    from vxl_sph import walls

    class Many:
        def bounds(self, bid):
            return ((-1.0, -1.0, -1.0), (1.0, 0.0, 1.0))

        def contacts_point(self, bid, p, probe):
            return [(np.array([p[0], 0.0, p[2]], F32), np.array([0.0, 1.0, 0.0], F32))] * 5

    ps = np.array([[0.0, 0.05, 0.0], [0.0, -0.02, 0.0], [0.0, 0.5, 0.0], [5.0, 0.05, 0.0]], F32)
    ids, start, planes = walls.gather_contacts([0, 1], 0.1, ps, Many(), walls.MIRROR)
    assert ids.tolist() == [0] and start.tolist() == [0, 8] and planes.shape == (8, 6)
    ids, start, _ = walls.gather_contacts([0], 0.1, ps, Many(), walls.PROJECT)
    assert ids.tolist() == [0, 1] and start.tolist() == [0, 5, 10]
