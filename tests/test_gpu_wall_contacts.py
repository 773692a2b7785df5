"""Provider walls of any ProviderColliders through contact tables, on a B200.

The reference's GPU tier serves providers it cannot evaluate on the device (voxel
terrain, meshes, splats) by gathering, once per tick on the host, each fluid particle's
contact planes and uploading two tables (crates/vxl-phys-gpu/src/pipeline/stepper.rs:
118-137, walls.rs:100-215). Here a test-only SDF provider set (a solid sphere and a
height-field floor, answered by closest-point queries in float32 like a terrain provider)
is gathered the same way every tick (vxl_sph.walls.gather_contacts) and uploaded with
vxl_sph_set_wall_contacts; the oracle is driven the same way (the same tables, set each
tick). The tables act as one more provider: mirror ghosts interleaved with the neighbour
terms in the CPU path's order (fluid_density.rs:25-47), projection and coincident
separation after integration (fluid_boundary.rs:45-128). Tolerance: zero (bitwise), tick
after tick, through the GpuFluidStepper mirror's gather_walls.
"""
import numpy as np
import pytest

from test_gpu_parity import _custom, assert_bits, pair

pytestmark = pytest.mark.gpu
F = np.float32


class SdfProviders:
    """bid 0: a height-field floor y = 0 (solid below); bid 1: a solid sphere."""

    def __init__(self, centre, radius):
        self.c = np.asarray(centre, F)
        self.r = F(radius)

    def bounds(self, bid):
        if bid == 0:
            return None  # unbounded terrain: always queried
        return (self.c - self.r, self.c + self.r)

    def contacts_point(self, bid, p, probe):
        p = np.asarray(p, F)
        if bid == 0:
            if p[1] > F(2) * probe:
                return []
            return [(np.array([p[0], 0.0, p[2]], F), np.array([0.0, 1.0, 0.0], F))]
        d = (p - self.c).astype(F)
        dist = F(np.sqrt(F(F(F(d[0] * d[0]) + F(d[1] * d[1])) + F(d[2] * d[2]))))
        if dist - self.r > probe or dist == F(0):
            return []
        n = (d / dist).astype(F)
        return [((self.c + n * self.r).astype(F), n)]

    def contacts_point_boundary(self, bid, p, probe):
        return self.contacts_point(bid, p, probe)


def _scene(vxl):
    from vxl_sph import scenes
    pos = scenes.jitter(scenes.fluid_block((-0.12, 0.18, -0.12), (6, 5, 6), 0.05), 0.05, 9)
    return _custom(vxl, pos, h=0.1, spacing=0.05, xsph_viscosity=0.05)


def test_sdf_provider_contact_tables_bit_exact(vxl, oracle_mod):
    """A block falling onto a sphere standing on a floor, 30 ticks: every tick the tables
    are gathered from the oracle's (bitwise equal) positions and given to both sides."""
    from vxl_sph import walls
    spec = _scene(vxl)
    prov = SdfProviders((0.0, 0.05, 0.0), 0.08)
    g, o = pair(vxl, oracle_mod, spec, threads=4)
    h = float(spec.params.smoothing_radius)
    dt = float(F(1.0) / F(60.0))
    touched = 0
    for t in range(30):
        ps = o.read_f32()["pos"][:spec.n_fluid]
        for side in (walls.MIRROR, walls.PROJECT):
            ids, start, planes = walls.gather_contacts([0, 1], h, ps, prov, side)
            g.set_wall_contacts(side, ids, start, planes)
            o.set_wall_contacts(side, ids, start, planes)
            touched = max(touched, ids.shape[0])
        g.step_tick(dt)
        o.step(dt)
        p, v = g.read_state()
        r = o.read_f32()
        assert_bits(p, r["pos"], f"tick {t} pos")
        assert_bits(v, r["vel"], f"tick {t} vel")
    assert touched > 20, "the block reached the providers"
    y = g.read_state()[0][:, 1]
    assert y.min() > -0.02, "projection kept the fluid above the floor"
    o.close()
    g.close()


def test_stepper_gather_walls_uses_contact_tables(vxl, oracle_mod):
    """GpuFluidStepper.gather_walls (read positions, gather, upload) once per tick before
    step, as the facade calls it (crates/vxl-phys/src/world_step/fluid_stepper.rs:66-79),
    tracks the oracle fed the tables gathered from its own positions."""
    from vxl_sph import walls
    spec = _scene(vxl)
    prov = SdfProviders((0.02, 0.04, -0.01), 0.07)
    st = vxl.GpuFluidStepper(spec.params, spec.n_fluid, spec.pos, spec.vel, spec.pmass, boundaries=[0, 1])
    o = oracle_mod.OracleSystem.from_scene(spec, threads=4)
    h = float(spec.params.smoothing_radius)
    dt = float(F(1.0) / F(60.0))
    for t in range(20):
        st.gather_walls(h, prov)
        ps = o.read_f32()["pos"][:spec.n_fluid]
        for side in (walls.MIRROR, walls.PROJECT):
            o.set_wall_contacts(side, *walls.gather_contacts([0, 1], h, ps, prov, side))
        st.step(dt, spec.n_fluid, spec.pos, spec.vel, spec.pmass, [])
        o.step(dt)
        assert_bits(st.scene.read_state()[0], o.read_f32()["pos"], f"tick {t} pos")
    o.close()


def test_contact_table_rejects_bad_tables(vxl):
    spec = _scene(vxl)
    g = vxl.Scene(spec.params, spec.pos, spec.vel, spec.pmass, spec.n_fluid)
    pl = np.zeros((2, 6), F)
    with pytest.raises(vxl.VxlError):
        g.set_wall_contacts(0, [3, 2], [0, 1, 2], pl)  # ids must ascend
    with pytest.raises(vxl.VxlError):
        g.set_wall_contacts(0, [spec.n_fluid], [0, 2], pl)  # not a fluid particle
    with pytest.raises(vxl.VxlError):
        g.set_wall_contacts(1, [0], [0, 9], np.zeros((9, 6), F))  # more than 8 planes
    g.set_wall_contacts(0, [], [0], np.zeros((0, 6), F))  # clearing is fine
    g.close()
