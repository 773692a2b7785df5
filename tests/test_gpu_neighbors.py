"""Neighbour lists and the 10M-particle configuration against the oracle, on a B200.

The neighbour lists the density pass records (and the force pass and boundary reactions
read) are exported through vxl_sph_export_neighbors and compared, entry for entry and in
order, with the oracle's UniformGrid::for_neighbors_in walk
(crates/vxl-phys-fluid/src/grid.rs:115-155) over the same positions: all neighbours of a
fluid particle, the fluid ones of a boundary particle (fluid_density.rs:59-69). Cases: the
16k dam break at h-sized bins, a doubled-bin tank (2h cells, half-cell culling), lists
longer than the 64 recorded entries (walked again), and a flowing state after a few ticks.

The 10M configuration (9,938,375 fluid particles in the 2.5 x 1.2 x 1.2 m tank, Akinci
walls, 64 boxes, c0 = 20, alpha = 0.05, eps = 0.5, bins doubled to 2h by the cell budget)
is stepped one substep from identical state on the GPU and on the oracle, and compared bit
for bit: cell table, density, pressure, acceleration, XSPH, per-boundary-particle
reaction, and the integrated positions and velocities
(crates/vxl-phys-fluid/src/fluid_step.rs:91-127).
"""
import os

import numpy as np
import pytest

from test_gpu_parity import F32, assert_bits, compare_grid, compare_state, f32_dt

pytestmark = pytest.mark.gpu


def _threads():
    return max(1, len(os.sched_getaffinity(0)))


def _compare_lists(g, o, label):
    go, ge = g.export_neighbors()
    oo, oe = o.neighbors()
    assert go.shape == oo.shape, label
    if not np.array_equal(go, oo):
        i = int(np.nonzero(go != oo)[0][0])
        raise AssertionError(f"{label}: list lengths differ first at particle {max(i - 1, 0)}")
    if not np.array_equal(ge, oe):
        k = int(np.nonzero(ge != oe)[0][0])
        i = int(np.searchsorted(oo, k, side="right") - 1)
        raise AssertionError(f"{label}: entry {k} (particle {i}) differs: {ge[k]} vs {oe[k]}")
    return go, ge


DENSITY = [0, 1]  # density kernels: per-particle walk, grouped segments


def _lists_after(vxl, oracle_mod, spec, warm_ticks=0, substeps_before=0, density=0):
    """GPU and oracle from identical state; optionally advanced together; then the oracle's
    lists from its current positions and the GPU's lists of its next substep."""
    g = vxl.Scene(spec.params, spec.pos, spec.vel, spec.pmass, spec.n_fluid)
    g.set_tuning(256, 256, 0, density)
    o = oracle_mod.OracleSystem.from_scene(spec, threads=_threads())
    dt_tick = float(F32(1) / F32(60))
    for _ in range(warm_ticks):
        g.step_tick(dt_tick, spec.spans)
        o.step(dt_tick)
    dt = f32_dt(spec.params.substeps)
    for _ in range(substeps_before):
        g.substep(dt)
        o.substep(dt)
    compare_state(g, o, "before the listed substep")
    g.substep(dt)
    return g, o


@pytest.mark.parametrize("density", DENSITY)
def test_neighbor_lists_dam0_bit_exact(vxl, oracle_mod, density):
    from vxl_sph import scenes
    spec = scenes.dam0()
    g, o = _lists_after(vxl, oracle_mod, spec, density=density)
    offs, ent = _compare_lists(g, o, "dam0")
    counts = np.diff(offs.astype(np.int64))
    assert counts[:spec.n_fluid].mean() > 20 and ent.size > 0


@pytest.mark.parametrize("density", DENSITY)
def test_neighbor_lists_flowing_state(vxl, oracle_mod, density):
    """After two ticks of the dam break (particles moved, cells reordered)."""
    from vxl_sph import scenes
    spec = scenes.dam0()
    g, o = _lists_after(vxl, oracle_mod, spec, warm_ticks=2, substeps_before=3, density=density)
    _compare_lists(g, o, "dam0 after 2 ticks + 3 substeps")


@pytest.mark.parametrize("density", DENSITY)
def test_neighbor_lists_doubled_bins(vxl, oracle_mod, density):
    """The 10M tank's grid rule with a 40^3 block: the budget doubles the bins to 2h, so the
    density pass culls half-cells and orders or groups particles by octant."""
    from vxl_sph import scenes
    spec = scenes.dam10m_block(40)
    g, o = _lists_after(vxl, oracle_mod, spec, density=density)
    _, _, _, info = g.export_grid()
    assert info.bin >= 2 * spec.params.smoothing_radius * 0.999
    _compare_lists(g, o, "dam10m tank, 40^3 block")


@pytest.mark.parametrize("density", DENSITY)
def test_neighbor_lists_longer_than_the_recorded_cap(vxl, oracle_mod, density):
    """h = 3 s: about 110 neighbours per particle, past the 64 recorded entries, so every
    interior list is walked again; boundary particles keep only their fluid neighbours."""
    from vxl_sph import scenes
    s = 0.02
    params = scenes.baseline_params(s, substeps=4, smoothing_radius=3 * s)
    fluid = scenes.jitter(scenes.fluid_block((0.0, 0.0, 0.0), (14, 12, 14), s), s, 5)
    spec = scenes.assemble("wide", params, fluid, scenes.tank_bodies((0.4, 0.4, 0.4), 2 * s), s, 2)
    g, o = _lists_after(vxl, oracle_mod, spec, density=density)
    offs, _ = _compare_lists(g, o, "h = 3 s")
    assert np.diff(offs.astype(np.int64)).max() > 64


def test_neighbor_lists_before_any_substep_is_not_ready(vxl):
    from vxl_sph import scenes
    spec = scenes.small_dam()
    g = vxl.Scene(spec.params, spec.pos, spec.vel, spec.pmass, spec.n_fluid)
    with pytest.raises(vxl.VxlError) as e:
        g.export_neighbors()
    assert e.value.status == vxl.NOT_READY


def test_dam10m_substep_bit_exact(vxl, oracle_mod):
    """The 10M configuration, one substep from identical state (doubled bins, walls, 64
    boxes, the configuration's constants): every per-particle quantity bit for bit, with
    either density kernel."""
    from vxl_sph import scenes
    spec = scenes.dam10m()
    assert spec.n_fluid == 9938375 and len(spec.spans) == 69
    o = oracle_mod.OracleSystem.from_scene(spec, threads=_threads())
    dt = f32_dt(spec.params.substeps)
    o.substep(dt)
    r = o.read_f32()
    nf = spec.n_fluid
    for density in DENSITY:
        g = vxl.Scene(spec.params, spec.pos, spec.vel, spec.pmass, spec.n_fluid)
        g.set_tuning(256, 256, 0, density)
        g.set_record(True)
        g.substep(dt)
        _, _, _, info = g.export_grid()
        assert info.bin >= 2 * spec.params.smoothing_radius * 0.999, "the cell budget doubles the bins"
        compare_grid(g, o, f"dam10m density kernel {density}")
        dens, press, acc, xsph, bf = g.read_fields()
        assert_bits(dens, r["dens"], "density")
        assert_bits(press, r["press"], "pressure")
        assert_bits(acc[:nf], r["acc"][:nf], "acceleration")
        assert_bits(xsph[:nf], r["xsph"][:nf], "xsph")
        assert_bits(bf, r["bforce"][nf:], "boundary reaction per particle")
        compare_state(g, o, f"dam10m after one substep, density kernel {density}")
        g.close()
    o.close()
