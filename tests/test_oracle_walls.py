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
