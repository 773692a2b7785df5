"""Batched and served forms on a B200, through the C ABI.

Batched: several independent scenes of different sizes, spacings and smoothing lengths in
one handle, stepped together (one launch per kernel per substep). Each scene must equal
the oracle and its own plain handle bit for bit — the segmented sort keeps scenes apart
and every per-scene sum keeps the reference's order — for every launch shape the
autotuner can choose. Served: requests that arrive while others run join at substep
boundaries; each finished request's state must equal the same scene stepped alone on a
plain handle for the same number of ticks (the alone-vs-mix check), bit for bit,
including when the budget forces requests to wait in the queue.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu
F32 = np.float32
DT_TICK = float(F32(1.0) / F32(60.0))


def _specs():
    from vxl_sph import scenes
    return [
        scenes.small_dam(n=(8, 10, 8), spacing=0.05, tank=(0.8, 0.7, 0.6), seed=11),
        scenes.small_dam(n=(12, 9, 7), spacing=0.04, tank=(0.7, 0.6, 0.5), seed=12),
        scenes.small_dam(n=(6, 6, 14), spacing=0.03, tank=(0.4, 0.5, 0.6), seed=13),
        scenes.small_dam(n=(10, 10, 10), spacing=0.05, tank=(0.9, 0.8, 0.7), seed=14),
    ]


def _assert_same(a, b, what):
    assert a.shape == b.shape and a.tobytes() == b.tobytes(), what


def test_batch_equals_oracle_and_plain(vxl, oracle_mod):
    specs = _specs()
    batch = vxl.Batch(specs)
    plain = [vxl.Scene(s.params, s.pos, s.vel, s.pmass, s.n_fluid) for s in specs]
    orc = [oracle_mod.OracleSystem.from_scene(s, threads=4) for s in specs]
    for t in range(3):
        rb = batch.step_tick(DT_TICK)
        rp = [p.step_tick(DT_TICK, s.spans) for p, s in zip(plain, specs)]
        for o in orc:
            o.step(DT_TICK)
        flat = [x for r in rp for x in r]
        assert len(rb) == len(flat)
        for (b1, f1, t1), (b2, f2, t2) in zip(rb, flat):
            assert b1 == b2 and f1.tobytes() == f2.tobytes() and t1.tobytes() == t2.tobytes()
    for q, (p, o) in enumerate(zip(plain, orc)):
        bp, bv = batch.read_state(q)
        pp, pv = p.read_state()
        r = o.read_f32()
        _assert_same(bp, pp, f"scene {q} pos vs plain")
        _assert_same(bv, pv, f"scene {q} vel vs plain")
        _assert_same(bp, r["pos"], f"scene {q} pos vs oracle")
        items, start, _, _ = batch.export_grid(q)
        og = o.grid()
        assert np.array_equal(items, og["items"]) and np.array_equal(start, og["start"])


@pytest.mark.parametrize("shape", [(128, 128, 0, 0), (256, 1024, 0, 1), (128, 128, 1, 1), (256, 256, 2, 0),
                                   (128, 4096, 1, 0), (256, 512, 1, 1)])
def test_batch_launch_shape_does_not_change_results(vxl, shape):
    specs = _specs()
    ref = vxl.Batch(specs)
    alt = vxl.Batch(specs)
    alt.set_tuning(*shape)
    assert alt.tuning() == shape
    for _ in range(2):
        ref.step_tick(DT_TICK)
        alt.step_tick(DT_TICK)
    for q in range(len(specs)):
        a, _ = ref.read_state(q)
        b, _ = alt.read_state(q)
        _assert_same(a, b, f"scene {q}")


def test_autotune_restores_state_and_keeps_results(vxl):
    specs = _specs()
    tuned = vxl.Batch(specs)
    plain = vxl.Batch(specs)
    tuned.step_tick(DT_TICK)
    plain.step_tick(DT_TICK)
    before = [tuned.read_state(q)[0].copy() for q in range(len(specs))]
    best = tuned.autotune(DT_TICK, trials=2)
    assert best["block"] in (128, 256) and best["tile"] % 128 == 0 and best["ms_per_substep"] > 0
    for q in range(len(specs)):
        _assert_same(tuned.read_state(q)[0], before[q], f"scene {q} after autotune")
    tuned.step_tick(DT_TICK)
    plain.step_tick(DT_TICK)
    for q in range(len(specs)):
        _assert_same(tuned.read_state(q)[0], plain.read_state(q)[0], f"scene {q}")


def _alone(vxl, spec, ticks):
    g = vxl.Scene(spec.params, spec.pos, spec.vel, spec.pmass, spec.n_fluid)
    for _ in range(ticks):
        g.step_tick(DT_TICK)
    return g.read_state()


def test_served_requests_equal_alone_runs(vxl):
    """Staggered arrivals with different tick counts: every result equals its alone run."""
    specs = _specs()
    ticks = [3, 2, 4, 1]
    srv = vxl.Server(budget_bytes=2 << 30)
    ids = []
    arrivals = {0: [0], 2: [1], 3: [2, 3]}  # substep index -> requests submitted before it
    step = 0
    while True:
        for r in arrivals.get(step, []):
            ids.append((r, srv.submit(specs[r], ticks[r])))
        rep = srv.step(DT_TICK)
        step += 1
        done = all(srv.poll(i).state == vxl.Server.DONE for _, i in ids) and len(ids) == len(specs)
        if done or step > 200:
            break
        if rep.active == 0 and rep.queued == 0 and len(ids) == len(specs):
            srv.step(DT_TICK)  # retire
            break
    for r, i in ids:
        st = srv.poll(i)
        assert st.state == vxl.Server.DONE and st.ticks_done == ticks[r]
        assert st.tick_p99_ms >= st.tick_p50_ms > 0
        tt = srv.tick_times(i)
        assert tt.shape == (ticks[r],) and np.all(tt > 0)
        assert tt.min() <= st.tick_p50_ms <= tt.max()
        p, v = srv.read(i)
        ap, av = _alone(vxl, specs[r], ticks[r])
        _assert_same(p, ap, f"request {r} pos")
        _assert_same(v, av, f"request {r} vel")


def test_served_budget_queues_then_admits(vxl):
    """A budget that fits one scene at a time: later requests wait, then run, same results."""
    from vxl_sph import scenes
    specs = [scenes.small_dam(n=(8, 8, 8), spacing=0.05, tank=(0.6, 0.5, 0.5), seed=21 + k) for k in range(3)]
    # every scene reserves its grid budget (2^21 cells x 8 B) out of the 15% of the budget
    # set aside for cells: 1.5 budgets of cells fit one scene at a time
    budget = int(1.5 * (1 << 21) * 8 / 0.15) + (1 << 20)
    srv = vxl.Server(budget_bytes=budget)
    ids = [srv.submit(s, 2) for s in specs]
    rep = srv.step(DT_TICK)
    assert rep.active == 1 and rep.queued == 2
    for _ in range(400):
        srv.step(DT_TICK)
        if all(srv.poll(i).state == vxl.Server.DONE for i in ids):
            break
    for s, i in zip(specs, ids):
        st = srv.poll(i)
        assert st.state == vxl.Server.DONE and st.admit_s >= st.submit_s
        p, _ = srv.read(i)
        ap, _ = _alone(vxl, s, 2)
        _assert_same(p, ap, "queued request")


def test_cell_capacity_overflow_is_reported_and_harmless(vxl):
    """A batch whose scenes need more cells than its cell capacity: the device flags it, every
    kernel of the tick returns without touching memory, the call reports
    VXL_DEVICE_FAULT_FLAG and the state is exactly the state before — repeatedly (no GPU
    fault involved; the flag is an ordinary word the host reads)."""
    specs = _specs()
    b = vxl.Batch(specs, cell_capacity=64)
    before = [b.read_state(q) for q in range(len(specs))]
    for _ in range(2):
        with pytest.raises(vxl.VxlError) as e:
            b.step_tick(DT_TICK)
        assert e.value.status == vxl.DEVICE_FAULT_FLAG and "cell capacity" in str(e.value)
        for q in range(len(specs)):
            p, v = b.read_state(q)
            _assert_same(p, before[q][0], f"scene {q} pos")
            _assert_same(v, before[q][1], f"scene {q} vel")


def test_served_request_that_never_fits_is_rejected(vxl):
    from vxl_sph import scenes
    srv = vxl.Server(budget_bytes=64 << 20)
    big = scenes.small_dam(n=(40, 40, 40), spacing=0.01, tank=(0.6, 0.6, 0.6), seed=1)
    with pytest.raises(vxl.VxlError) as e:
        srv.submit(big, 2)
    assert e.value.status == vxl.OUT_OF_MEMORY
    rep = srv.step(DT_TICK)
    assert rep.active == 0 and rep.queued == 0


def test_batch_with_boundary_only_and_single_particle_scenes(vxl):
    """Degenerate scenes inside a batch: a boundary-only scene stays exactly where it is
    (the reference does not drive a system without fluid, fluid_step.rs:93-95) and a
    one-particle scene falls like its own plain handle; the ordinary scenes around them are
    unaffected."""
    from vxl_sph import scenes
    specs = _specs()[:2]
    b_pos, b_vel, b_pm, b_spans = scenes.body_particles([scenes.Body(0, (0.1, 0.02, 0.1), (0.2, 0.1, 0.2))],
                                                        0.05, 0.1, 1, 1000.0)
    p = scenes.baseline_params(0.05, substeps=4)
    walls_only = scenes.SceneSpec("walls", p, b_pos, b_vel, b_pm, 0, [], 0.05, 1)
    one = scenes.SceneSpec("one", scenes.baseline_params(0.05, substeps=4), np.array([[0.3, 0.4, 0.2]], F32),
                           np.zeros((1, 3), F32), np.full(1, F32(p.particle_mass), F32), 1, [], 0.05, 1)
    mix = [specs[0], walls_only, one, specs[1]]
    batch = vxl.Batch(mix)
    plain = [vxl.Scene(s.params, s.pos, s.vel, s.pmass, s.n_fluid) for s in mix]
    for _ in range(3):
        batch.step_tick(DT_TICK)
        for q, (pl, s) in enumerate(zip(plain, mix)):
            pl.step_tick(DT_TICK, s.spans if q != 1 else ())
    for q, pl in enumerate(plain):
        bp, bv = batch.read_state(q)
        pp, pv = pl.read_state()
        _assert_same(bp, pp, f"scene {q} pos")
        _assert_same(bv, pv, f"scene {q} vel")
    wp, _ = batch.read_state(1)
    _assert_same(wp, b_pos, "boundary-only scene moved")
