#!/usr/bin/env python
"""Benchmark of the B200 WCSPH plain step (one JSON line on rank 0).

A step is one 60 Hz tick of the plain single-scene path: 10 substeps of grid
rebuild (cell keys + stable counting sort), density + EOS, and force + XSPH +
integration with the Akinci wall terms and per-body reactions, on a seeded dam-break
scene resident in HBM. value = fluid particle-updates per second (one update = one fluid
particle through one full substep), summed over ranks, divided by the slowest rank's
device time. Multi-GPU runs are independent replicas (each rank steps its own scene;
no collective on the data path), so scaling is weak.

The plain run also carries two comparisons (single GPU only): "batched", 256 uneven
tanks stepped in one handle against looping the plain step over them, and "served",
Poisson-arriving requests under continuous batching against running them one by one on
plain handles (p50/p99 per-tick latency beside aggregate throughput).

  python bench.py [--gpus N] [--steps K] [--warmup W] [--workload dam1|dam0|dam10m]
  python bench.py --workload batched|served ...   # the batched or served form as the headline
  python bench.py --impl reference ...   # the reference CPU path (C++ restatement) on the host cores
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import tempfile
import time
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parent
for p in (ROOT, ROOT / "rust-wl_b200"):
    if str(p) not in sys.path:
        sys.path.insert(0, str(p))

METRIC = "WCSPH particle-updates/s & %HBM roofline; batched/served p50/p99 vs plain"
UNIT = "particle-updates/s"
FALLBACK_HBM_GBS = 6650.0
# Kernels launched on the handle's second stream beside k_force: their event-timed spans
# include waiting for SMs that k_force holds, so they are not costs and are listed apart.
SIDE_STREAM = ("k_bforce", "k_react_long", "k_react_spans")

# Algorithmic bytes per launch of each substep kernel (per particle unless noted), the
# per-unit figures of the byte model B = 116 N_t + 72 N_f + 40 N_b + 8 C per substep:
#   k_keys     16 B position read + 4 B key write                       (N_t)
#   k_canon    4 B key + 32 B pos/vel read + 32 B write + 4 B index      (N_t)
#   k_density  16 B position read + 8 B (rho, p/rho^2) write            (N_t)
#   k_force    fluid 40 B read + 32 B write; boundary 40 B read once    (N_f, N_b)
#   scan       8 B per cell
def algorithmic_bytes(kernel: str, nf: int, nb: int, cells: int) -> float | None:
    nt = nf + nb
    return {
        "k_keys": 20.0 * nt,
        "k_canon": 72.0 * nt,
        "k_density": 24.0 * nt,
        "k_force": 72.0 * nf + 40.0 * nb,
        "k_scan_final": 8.0 * cells,
    }.get(kernel)


def substep_bytes(nf: int, nb: int, cells: int) -> float:
    return 116.0 * (nf + nb) + 72.0 * nf + 40.0 * nb + 8.0 * cells


def ncu_traffic(kernel: str, workload: str):
    """DRAM bytes per launch of `kernel` on `workload` from the committed ncu summary."""
    p = ROOT / "profiles" / "roofline_traffic.txt"
    try:
        for line in p.read_text().splitlines():
            f = line.split()
            if len(f) >= 3 and not line.startswith("#") and f[0] == kernel and f[1] == workload:
                return float(f[2])
    except OSError:
        pass
    return None


def ncu_issue(kernel: str, workload: str):
    """Issue-slot use of `kernel` on `workload` from the committed ncu summary: the resource
    that binds the neighbour passes (their DRAM throughput stays below 10%)."""
    p = ROOT / "profiles" / "roofline_issue.txt"
    try:
        for line in p.read_text().splitlines():
            f = line.split()
            if len(f) >= 5 and not line.startswith("#") and f[0] == kernel and f[1] == workload:
                return {"issue_active": float(f[2]), "threads_per_instruction": float(f[3]),
                        "source": "profiles/" + f[4]}
    except OSError:
        pass
    return None


def hbm_peak() -> tuple[float, str]:
    p = ROOT / "MEASURED_PEAKS.json"
    try:
        v = float(json.loads(p.read_text())["hbm_gbs"])
        return v, "measured"
    except Exception:
        return FALLBACK_HBM_GBS, "fallback"


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled every 200 ms during a region."""

    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,clocks_event_reasons.hw_slowdown,"
         "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
         "clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu: int):
        self.gpu = gpu
        self.proc = None
        self.path = None

    def start(self):
        try:
            fd, self.path = tempfile.mkstemp(suffix=".csv")
            os.close(fd)
            self.f = open(self.path, "w")
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.gpu), f"--query-gpu={self.Q}",
                                          "--format=csv,noheader,nounits", "-lms", "200"], stdout=self.f,
                                         stderr=subprocess.DEVNULL)
        except Exception:
            self.proc = None

    def stop(self) -> dict:
        if not self.proc:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unavailable"]}
        time.sleep(0.25)
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        self.f.close()
        sm, smax, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in Path(self.path).read_text().splitlines():
            f = [x.strip() for x in line.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                smax.append(float(f[2]))
            except ValueError:
                continue
            for n, v in zip(names, f[5:9]):
                if v.lower() == "active":
                    reasons.add(n)
        os.unlink(self.path)
        if not sm:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["no samples"]}
        loaded = [x for x in sm if x > 0.5 * max(sm)] or sm
        return {"sm_mhz": statistics.median(loaded), "sm_max_mhz": max(smax), "reasons": sorted(reasons),
                "samples": len(sm)}


def build_scene(workload: str):
    from vxl_sph import scenes
    return scenes.CONFIGS[workload]()


# The CPU path's bounded sample of each plain workload. dam10m: a 100^3 fluid block in the
# corner of the dam10m tank, its floor and two corner walls cropped around the block and two
# marker boxes at the tank's far corners (scenes.dam10m_sample): the same grid and doubled
# bins as the full scene, a boundary-to-fluid ratio close to its own, 1M fluid particles, so
# that a step of the reference arm (one substep) takes seconds instead of half a minute.
# dam0 and dam1 are sampled whole.
def cpu_sample_spec(workload: str):
    from vxl_sph import scenes
    if workload == "dam10m":
        return scenes.dam10m_sample(100)
    return build_scene(workload)


def workload_config(spec) -> dict:
    """The `config` object of both arms' lines for a plain workload (identical in each)."""
    tank = spec.meta.get("tank")
    return {"workload": spec.name, "n_fluid": spec.n_fluid, "n_boundary": spec.n_boundary,
            "substeps": int(spec.params.substeps), "h": float(spec.params.smoothing_radius),
            "spacing": float(spec.spacing), "tank": list(tank) if tank else None, "fill": spec.meta.get("fill"),
            "bodies": len(spec.spans), "dynamic_boxes": int(sum(spec.meta.get("dynamic", []))),
            "unit_of_work": "one fluid particle advanced through one full substep"}


def use_oracle_lattice() -> None:
    """Build scenes with the oracle's lattice restatement (the CPU arm loads no CUDA library)."""
    from oracle import oracle as orc
    from vxl_sph import scenes
    scenes.use_lattice_source(*orc.scene_lattice_source())


def measure_coupled(spec, local: int, steps: int, warmup: int, density: float = 500.0) -> dict:
    """The scene's boxes as dynamic rigid bodies kept on the device (vxl_sph_step_coupled:
    two rigid substeps from the previous tick's reactions, the boundary rebuilt from the new
    poses, the fluid tick; the tank walls static; no contact solver), `steps` coupled ticks
    from the initial state and the initial bodies, the reactions back on the host each tick."""
    import torch
    import vxl_sph
    from vxl_sph import scenes
    bodies, dynamic = spec.meta["bodies"], spec.meta["dynamic"]
    p = spec.params
    lat, idx = scenes.body_lattice(bodies, spec.spacing, p.smoothing_radius, p.boundary_layers)
    inv_mass, inertia = [], []
    for b, d in zip(bodies, dynamic):
        im, ii = scenes.box_mass_props(b.half, density) if d else (0.0, (0.0, 0.0, 0.0))
        inv_mass.append(im)
        inertia.append(ii)
    g = vxl_sph.Scene(spec.params, spec.pos, spec.vel, spec.pmass, spec.n_fluid, device=local)
    stream = torch.cuda.Stream(device=local)
    g.set_stream(stream.cuda_stream)
    g.set_body_lattice(lat, idx, len(bodies))
    g.set_spans(spec.spans)
    dt = float(np.float32(1.0) / np.float32(60.0))
    grav = (0.0, -9.81, 0.0)
    nspans = len(spec.spans)

    def reset():
        g.write_state(spec.pos, spec.vel)
        g.set_rigid_bodies(bodies, inv_mass, inertia, dynamic)

    reset()
    for _ in range(max(warmup, 2)):
        g.step_coupled(dt, 2, grav, 100.0, 50.0, nspans)
    reset()
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    with torch.cuda.stream(stream):
        e0.record(stream)
    for _ in range(steps):
        g.step_coupled(dt, 2, grav, 100.0, 50.0, nspans)
    with torch.cuda.stream(stream):
        e1.record(stream)
    torch.cuda.synchronize()
    ms = e0.elapsed_time(e1)
    g.close()
    upd = spec.n_fluid * spec.params.substeps * steps
    return {"workload": f"{spec.name} with its {sum(dynamic)} boxes dynamic (density {density} kg/m^3), "
                        "the coupling loop on the device, no contact solver",
            "value": upd / (ms / 1e3), "unit": UNIT, "ms_per_tick": ms / steps, "rigid_substeps": 2,
            "call": "vxl_sph_step_coupled per tick (reactions to the host; bodies stay on the device)"}


def cpu_baseline(workload: str, budget_s: float = 12.0) -> dict:
    """The oracle (C++ restatement of the reference's phase-parallel CPU path) on the host
    cores, on a bounded sample of the same workload (cpu_sample_spec): whole substeps from
    the sample's initial state until budget_s of wall time is used."""
    from oracle import oracle as orc
    spec = cpu_sample_spec(workload)
    cores = len(os.sched_getaffinity(0)) if hasattr(os, "sched_getaffinity") else os.cpu_count()
    o = orc.OracleSystem.from_scene(spec, threads=cores)
    dt = float(np.float32(np.float32(1.0) / np.float32(60.0)) / np.float32(spec.params.substeps))
    n = 0
    t0 = time.perf_counter()
    while True:
        o.substep(dt)
        n += 1
        el = time.perf_counter() - t0
        if el >= budget_s or n >= 10 * spec.params.substeps:
            break
    o.close()
    return {"value": spec.n_fluid * n / el, "unit": UNIT, "cores": cores, "kind": "port",
            "sample": f"{spec.name}: {n} substeps from the initial state ({spec.n_fluid} fluid + "
                      f"{spec.n_boundary} boundary particles), {el:.1f} s wall, {cores} threads"}


def run_reference(args) -> None:
    """The reference arm: the reference's CPU path (the oracle, its C++ restatement; Rust is
    not buildable here) on all host cores, rank 0 only. Scenes are built with the oracle's
    lattice, so this process loads no library of this repository's product."""
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    use_oracle_lattice()
    from oracle import oracle as orc
    cores = len(os.sched_getaffinity(0)) if hasattr(os, "sched_getaffinity") else os.cpu_count()
    if args.cpu_threads:
        cores = args.cpu_threads
    if args.workload in ("batched", "served"):
        run_reference_mix(args, orc, cores)
        return
    spec = build_scene(args.workload)
    config = workload_config(spec)
    del spec
    sample = cpu_sample_spec(args.workload)
    o = orc.OracleSystem.from_scene(sample, threads=cores)
    dt_sub = float(np.float32(np.float32(1.0) / np.float32(60.0)) / np.float32(sample.params.substeps))
    # one step = one substep of the bounded sample (the metric is per particle-update, so
    # it compares with the GPU arm's ticks of the whole workload)
    for _ in range(args.warmup):
        o.substep(dt_sub)
    times = []
    for _ in range(args.steps):
        t0 = time.perf_counter()
        o.substep(dt_sub)
        times.append(time.perf_counter() - t0)
    o.close()
    total = sum(times)
    value = sample.n_fluid * args.steps / total
    desc = (f"{args.steps} substeps of {sample.name} ({sample.n_fluid} fluid + {sample.n_boundary} boundary "
            f"particles) after {args.warmup} warm-up substeps, {cores} threads")
    line = {
        "impl": "reference", "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": args.gpus,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1e3 * total / args.steps,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
        "data": "synthetic: seeded dam break in an Akinci-walled tank (no public dataset exists)",
        "config": config,
        "step": "one substep of the bounded sample on the host cores (the reference CPU path restated in C++)",
        "cpu_baseline": {"value": value, "unit": UNIT, "cores": cores, "kind": "port", "sample": desc},
        "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


def run_reference_mix(args, orc, cores: int) -> None:
    """The reference CPU path scene by scene on the batched or served workload: each step is
    one substep of every scene of a bounded sample (the first `--scenes` tanks of the mix,
    at most 16, or the first 8 requests), the scenes stepped one after another as a host
    running one FluidSystem per scene would."""
    from vxl_sph import scenes
    if args.workload == "batched":
        specs = scenes.batched_mix(min(args.scenes, 16))
        sample = f"the first {len(specs)} of the 256 tanks"
    else:
        specs = [r.spec for r in scenes.served_stream(8, 1.0, tick_scale=args.tick_scale)]
        sample = f"the first {len(specs)} requests of the stream"
    systems = [orc.OracleSystem.from_scene(sp, threads=cores) for sp in specs]
    dts = [float(np.float32(np.float32(1.0) / np.float32(60.0)) / np.float32(sp.params.substeps)) for sp in specs]
    for _ in range(args.warmup):
        for o, dt in zip(systems, dts):
            o.substep(dt)
    t0 = time.perf_counter()
    for _ in range(args.steps):
        for o, dt in zip(systems, dts):
            o.substep(dt)
    total = time.perf_counter() - t0
    for o in systems:
        o.close()
    nf = sum(sp.n_fluid for sp in specs)
    value = nf * args.steps / total
    line = {
        "impl": "reference", "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": args.gpus,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1e3 * total / args.steps,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
        "data": "synthetic (seeded tanks)",
        "config": {"workload": args.workload, "scenes": len(specs), "n_fluid": nf,
                   "step": "one substep of every sampled scene, scene by scene, on the host cores"},
        "cpu_baseline": {"value": value, "unit": UNIT, "cores": cores, "kind": "port",
                         "sample": f"{args.steps} substeps of {sample} after {args.warmup} warm-up substeps"},
        "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


def run_ours(args) -> None:
    import torch
    import vxl_sph

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    dist = None
    if world > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))

    vxl_sph.load()
    spec = build_scene(args.workload)
    scene = vxl_sph.Scene(spec.params, spec.pos, spec.vel, spec.pmass, spec.n_fluid, device=local)
    stream = torch.cuda.Stream(device=local)
    scene.set_stream(stream.cuda_stream)
    dt_tick = float(np.float32(1.0) / np.float32(60.0))
    sub = spec.params.substeps

    tune = scene.autotune(dt_tick, trials=3)  # launch shape for this scene (state restored)
    for _ in range(max(args.warmup, 3)):
        scene.step_tick_async(dt_tick, spec.spans)
        scene.sync()

    l2_flush = torch.empty(256 << 20, dtype=torch.uint8, device=f"cuda:{local}")

    def timed_ticks(profiled: bool) -> list:
        """`args.steps` ticks from the workload's initial state (the states the CPU arm
        times), L2 flushed before each, one CUDA-event pair per tick on the scene's stream."""
        scene.write_state(spec.pos, spec.vel)
        evs = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True))
               for _ in range(args.steps)]
        torch.cuda.synchronize()
        if dist:
            dist.barrier()
        for k in range(args.steps):
            if profiled:
                scene.profile()  # collect the previous tick's kernel timers before enqueueing more
            with torch.cuda.stream(stream):
                l2_flush.zero_()
                evs[k][0].record(stream)
            scene.step_tick_async(dt_tick, spec.spans)
            with torch.cuda.stream(stream):
                evs[k][1].record(stream)
        torch.cuda.synchronize()
        scene.sync()
        if dist:
            dist.barrier()
        return [a.elapsed_time(b) for a, b in evs]

    # headline pass: the tick graph without per-kernel events
    clocks = ClockSampler(local)
    clocks.start()
    step_ms = timed_ticks(False)
    clk = clocks.stop()
    total_ms = sum(step_ms)
    stats = scene.stats()
    cells = int(stats.cells)
    launches_per_tick = int(stats.launches_last_tick)
    # roofline pass: the same ticks with a CUDA-event pair around every kernel launch
    scene.set_profile(True)
    scene.step_tick_async(dt_tick, spec.spans)  # capture the profiled graph outside the timed ticks
    scene.sync()
    scene.set_profile(True)  # reset accumulators
    prof_step_ms = timed_ticks(True)
    prof = scene.profile()

    from vxl_sph import placement
    t_max = placement.max_over_ranks(total_ms, dist, f"cuda:{local}")
    updates = spec.n_fluid * sub * args.steps * world
    value = updates / (t_max / 1e3)

    # dominant kernel and its roofline
    peak, peak_kind = hbm_peak()
    dom = max(((k, v) for k, v in prof.items() if k not in SIDE_STREAM), key=lambda kv: kv[1][0])
    dom_name, (dom_ms, dom_n) = dom
    prof_total = sum(v[0] for v in prof.values())
    bytes_launch = algorithmic_bytes(dom_name, spec.n_fluid, spec.n_boundary, cells)
    avg_ms = dom_ms / max(dom_n, 1)
    achieved = (bytes_launch / (avg_ms / 1e3) / 1e9) if bytes_launch else None
    roofline = {"kernel": dom_name, "bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                "frac": (achieved / peak) if achieved else None,
                "traffic": ncu_traffic(dom_name, spec.name),
                "issue": ncu_issue(dom_name, spec.name),
                "peak_source": f"{peak_kind} (MEASURED_PEAKS.json hbm_gbs)" if peak_kind == "measured"
                else "fallback 6650 GB/s",
                "avg_launch_ms": avg_ms, "launches": dom_n, "share": dom_ms / prof_total if prof_total else None,
                "algorithmic_bytes_per_launch": bytes_launch,
                "substep": {"bytes": substep_bytes(spec.n_fluid, spec.n_boundary, cells),
                            "ms": total_ms / (args.steps * sub)},
                "profiled_ms_per_tick": sum(prof_step_ms) / args.steps,
                "timing": "kernel times from a second pass over the same ticks with an event pair around "
                          "every launch; value from the pass without them. k_bforce runs on a second stream "
                          "beside k_force and k_react_* on a third beside the next substep's passes: their "
                          "spans include waiting for SMs, so they are listed apart "
                          "(side_stream_spans_ms_per_substep) and are not costs",
                "kernels_ms_per_substep": {k: v[0] / max(args.steps * sub, 1) for k, v in sorted(prof.items())
                                           if k not in SIDE_STREAM},
                "side_stream_spans_ms_per_substep": {k: v[0] / max(args.steps * sub, 1)
                                                     for k, v in sorted(prof.items()) if k in SIDE_STREAM}}
    sb = roofline["substep"]
    sb["achieved_gbs"] = sb["bytes"] / (sb["ms"] / 1e3) / 1e9
    sb["frac"] = sb["achieved_gbs"] / peak

    # e2e: the drop-in call pattern of the GPU tier's FluidStepper::step through the C ABI,
    # pinned host buffers. The backend owns the fluid state, so a step uploads the boundary
    # segment (the reference's per-tick upload, crates/vxl-phys-gpu/src/pipeline/coupling.rs:
    # 20-50), enqueues the tick, takes the previous tick's positions while this one runs
    # (the tier's deferred readback: Packet::run_deferred + take_deferred_state,
    # crates/vxl-phys-gpu/src/pipeline.rs:603-609, pipeline/readback.rs:229-262), waits for
    # this tick's per-body reactions and requests its positions. Every timed step's positions
    # reach the host inside the timed region (the last one after the loop).
    nf, nb = spec.n_fluid, spec.n_boundary
    pin_bp = torch.empty((max(nb, 1), 3), dtype=torch.float32, pin_memory=True).numpy()[:nb]
    pin_bv = torch.empty((max(nb, 1), 3), dtype=torch.float32, pin_memory=True).numpy()[:nb]
    pin_p = torch.empty((spec.n_total, 3), dtype=torch.float32, pin_memory=True).numpy()
    pin_bp[:] = spec.pos[nf:]
    pin_bv[:] = spec.vel[nf:]
    scene.set_profile(False)

    def e2e_steps(k: int) -> None:
        for q in range(k):
            if nb:
                scene.upload_boundary(pin_bp, pin_bv)
            scene.step_tick_async(dt_tick, spec.spans)
            if q:
                scene.take_state(pin_p)
            scene.sync()
            scene.request_state()
        if k:
            scene.take_state(pin_p)

    scene.write_state(spec.pos, spec.vel)
    e2e_steps(2)
    scene.write_state(spec.pos, spec.vel)  # the timed steps start from the initial state too
    torch.cuda.synchronize()
    if dist:
        dist.barrier()
    t0 = time.perf_counter()
    e2e_steps(args.steps)
    e2e_s = placement.max_over_ranks(time.perf_counter() - t0, dist, f"cuda:{local}")
    nspans = len(spec.spans)
    e2e = {"value": updates / e2e_s, "unit": UNIT, "h2d_bytes_per_step": nb * 24 + nspans * 24,
           "d2h_bytes_per_step": spec.n_total * 12 + nspans * 28,
           "api": "vxl_sph_upload_boundary (boundary segment) + vxl_sph_step_tick_async (spans in) + "
                  "vxl_sph_take_state (the previous tick's positions) + vxl_sph_sync (reactions out) + "
                  "vxl_sph_request_state, pinned host buffers: the GPU tier's FluidStepper::step pattern "
                  "with its deferred readback"}

    mix = {}
    if world == 1 and spec.meta.get("dynamic") and any(spec.meta["dynamic"]) and not args.no_coupled:
        mix["coupled"] = measure_coupled(spec, local, steps=args.steps, warmup=args.warmup)
    if not args.no_mix:
        # scene-parallel on several GPUs: each rank takes its share of the tanks / requests
        scene.close()
        mix["batched"] = measure_batched(local, steps=3, warmup=3, rank=rank, world=world, dist=dist)
        mix["served"] = measure_served(local, n_requests=args.requests, rates=args.rates, tick_scale=args.tick_scale,
                                       rank=rank, world=world, dist=dist)

    cpu = None
    if world == 1 and not args.no_cpu_baseline:
        cpu = cpu_baseline(args.workload)

    if rank == 0:
        line = {
            "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": t_max / args.steps, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f32",
            "data": "synthetic: seeded dam break in an Akinci-walled tank (no public dataset exists)",
            "config": workload_config(spec),
            "step": "one 60 Hz tick (10 substeps) of the whole workload on the GPU",
            "run": {"cells": cells, "l2": "flushed between steps (256 MiB write outside the timed events)",
                    "parallelism": f"replicas x{world} (each rank steps its own copy of the scene)",
                    "tuning": tune},
            "roofline": roofline,
            "cpu_baseline": cpu,
            "e2e": e2e,
            "gpu_launches": launches_per_tick * args.steps,
            "clocks": clk,
            "step_ms": step_ms,
            **mix,
        }
        print(json.dumps(line), flush=True)
    scene.close()
    if dist:
        dist.destroy_process_group()


def _pct(v, q):
    return float(np.percentile(np.asarray(v, np.float64), q)) if len(v) else None


def measure_batched(local: int, steps: int, warmup: int, n_scenes: int = 256, seed: int = 7,
                    plain_loop: bool = True, rank: int = 0, world: int = 1, dist=None) -> dict:
    """The batched workload (n_scenes uneven dam-break tanks in one handle, autotuned launch
    shape, one graph per tick) against looping the plain step scene by scene.

    Batched: device time of `steps` ticks (CUDA events on the handle's stream, L2 flushed
    between ticks) and the wall time of the same ticks through the synchronous C ABI call.
    Plain loop: `steps` ticks of every scene on its own plain handle, one synchronous
    vxl_sph_step_tick after another (the reference's per-stepper call pattern), wall time.
    On several GPUs each rank steps its share of the scenes (scene-parallel placement, no
    collective on the data path); rates are summed over ranks and divided by the slowest
    rank's time.
    """
    import torch
    import vxl_sph
    from vxl_sph import placement, scenes

    t_build = time.perf_counter()
    specs = scenes.batched_mix(n_scenes, seed)
    if world > 1:
        mine = placement.assign_scenes([s.n_total for s in specs], world)[rank]
        specs = [specs[q] for q in mine]
    t_build = time.perf_counter() - t_build
    nf = sum(s.n_fluid for s in specs)
    nb = sum(s.n_boundary for s in specs)
    sub = specs[0].params.substeps
    dt_tick = float(np.float32(1.0) / np.float32(60.0))
    batch = vxl_sph.Batch(specs, device=local)
    stream = torch.cuda.Stream(device=local)
    batch.set_stream(stream.cuda_stream)
    t0 = time.perf_counter()
    tune = batch.autotune(dt_tick, trials=2)
    tune_s = time.perf_counter() - t0
    for _ in range(max(warmup, 3)):
        batch.step_tick(dt_tick)
    l2_flush = torch.empty(256 << 20, dtype=torch.uint8, device=f"cuda:{local}")

    def timed_ticks(profiled: bool) -> float:
        for q, sp in enumerate(specs):  # timed ticks start from the initial state
            batch.write_state(q, sp.pos, sp.vel)
        evs = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(steps)]
        torch.cuda.synchronize()
        for k in range(steps):
            if profiled:
                batch.profile()
            with torch.cuda.stream(stream):
                l2_flush.zero_()
                evs[k][0].record(stream)
            batch.step_tick_async(dt_tick)
            with torch.cuda.stream(stream):
                evs[k][1].record(stream)
        torch.cuda.synchronize()
        batch.sync()
        return sum(a.elapsed_time(b) for a, b in evs)

    dev_ms = placement.max_over_ranks(timed_ticks(False), dist, f"cuda:{local}")
    stats = batch.stats()
    cells = int(stats.cells)
    launches = int(stats.launches_last_tick)
    batch.set_profile(True)
    batch.step_tick(dt_tick)  # capture the profiled graph outside the timed ticks
    batch.set_profile(True)
    timed_ticks(True)
    prof = batch.profile()
    batch.set_profile(False)
    batch.step_tick(dt_tick)  # re-capture the tick graph without profiling events
    for q, sp in enumerate(specs):
        batch.write_state(q, sp.pos, sp.vel)
    # wall time through the synchronous call (what a caller sees)
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    for _ in range(steps):
        batch.step_tick(dt_tick)
    wall_s = placement.max_over_ranks(time.perf_counter() - t0, dist, f"cuda:{local}")
    batch.close()
    del batch
    nf_all = int(placement.sum_over_ranks(nf, dist, f"cuda:{local}"))
    updates = nf_all * sub * steps
    peak, _ = hbm_peak()
    sb = substep_bytes(nf, nb, cells)
    out = {
        "workload": f"{n_scenes} dam-break tanks, N log-U[4096, 262144], aspect U[0.5, 2], fill U[0.2, 0.6], "
                    f"s U[0.005, 0.02] m, h = 2 s, closed tanks, seed {seed}",
        "scenes": n_scenes, "scenes_this_rank": len(specs), "n_fluid": nf_all, "n_boundary_this_rank": nb,
        "cells_this_rank": cells, "substeps": sub, "ticks": steps,
        "value": updates / (dev_ms / 1e3), "unit": UNIT, "ms_per_tick": dev_ms / steps,
        "wall_value": updates / wall_s, "wall_ms_per_tick": 1e3 * wall_s / steps,
        "tuning": tune, "autotune_s": tune_s, "build_s": t_build, "gpu_launches_per_tick": launches,
        "substep_roofline": {"bytes": sb, "ms": dev_ms / (steps * sub),
                             "achieved_gbs": sb / (dev_ms / (steps * sub) / 1e3) / 1e9, "peak": peak},
        "kernels_ms_per_substep": {k: v[0] / max(steps * sub, 1) for k, v in sorted(prof.items())
                                   if k not in SIDE_STREAM},
        "side_stream_spans_ms_per_substep": {k: v[0] / max(steps * sub, 1) for k, v in sorted(prof.items())
                                             if k in SIDE_STREAM},
    }
    out["substep_roofline"]["frac"] = out["substep_roofline"]["achieved_gbs"] / peak
    if plain_loop:
        plain = [vxl_sph.Scene(s.params, s.pos, s.vel, s.pmass, s.n_fluid, device=local) for s in specs]
        for sc, s in zip(plain, specs):
            sc.step_tick(dt_tick, s.spans)  # graph capture + warm-up
            sc.write_state(s.pos, s.vel)  # back to the initial state
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        for _ in range(steps):
            for sc, s in zip(plain, specs):
                sc.step_tick(dt_tick, s.spans)
        plain_s = placement.max_over_ranks(time.perf_counter() - t0, dist, f"cuda:{local}")
        for sc, s in zip(plain, specs):
            sc.write_state(s.pos, s.vel)
        torch.cuda.synchronize()
        # the same loop with every scene's tick enqueued before any is awaited
        t0 = time.perf_counter()
        for _ in range(steps):
            for sc, s in zip(plain, specs):
                sc.step_tick_async(dt_tick, s.spans)
            for sc in plain:
                sc.sync()
        plain_async_s = placement.max_over_ranks(time.perf_counter() - t0, dist, f"cuda:{local}")
        for sc in plain:
            sc.close()
        out["plain_loop"] = {"value": updates / plain_s, "ms_per_tick": 1e3 * plain_s / steps,
                             "call": "vxl_sph_step_tick per scene, synchronous, one after another"}
        out["plain_loop_async"] = {"value": updates / plain_async_s, "ms_per_tick": 1e3 * plain_async_s / steps,
                                   "call": "vxl_sph_step_tick_async on every scene, then vxl_sph_sync on each"}
        out["speedup_vs_plain_loop"] = plain_s / wall_s
        out["speedup_vs_plain_async"] = plain_async_s / wall_s
    return out


def _serve_once(reqs, local: int, budget_bytes: int, batch_cap: int = 0, dist=None, world: int = 1) -> dict:
    """One served run of `reqs`: Poisson arrivals submitted as wall time reaches them, one
    vxl_sph_serve_step (retire, admit, one substep of every admitted scene) after another
    until every request is done. Aggregate fluid particle-updates/s over the makespan (first
    arrival to last completion), per-tick latency pooled over every tick of every request,
    request latency (completion - arrival)."""
    import torch
    import vxl_sph
    from vxl_sph import placement
    dt_tick = float(np.float32(1.0) / np.float32(60.0))
    sub = reqs[0].spec.params.substeps
    updates = placement.sum_over_ranks(sum(r.spec.n_fluid * sub * r.ticks for r in reqs), dist, f"cuda:{local}")
    srv = vxl_sph.Server(budget_bytes=budget_bytes, device=local)
    if batch_cap:
        srv.set_batch_cap(batch_cap)
    torch.cuda.synchronize()
    ids, py_submit = [], []
    i = steps = peak_active = peak_queued = 0
    peak_bytes = 0
    t0 = time.perf_counter()
    while True:
        now = time.perf_counter() - t0
        while i < len(reqs) and reqs[i].arrival_s <= now:
            ids.append(srv.submit(reqs[i].spec, reqs[i].ticks))
            py_submit.append(time.perf_counter() - t0)
            i += 1
        rep = srv.step(dt_tick)
        steps += 1
        peak_active = max(peak_active, rep.active)
        peak_queued = max(peak_queued, rep.queued)
        peak_bytes = max(peak_bytes, int(rep.device_bytes_in_use))
        if rep.active == 0 and rep.queued == 0:
            if i >= len(reqs):
                break
            time.sleep(max(0.0, reqs[i].arrival_s - (time.perf_counter() - t0)))
    t_end = time.perf_counter() - t0
    if dist is not None and world > 1:
        dist.barrier()
    sts = [srv.poll(q) for q in ids]
    ticks_ms = np.concatenate([srv.tick_times(q) for q in ids])
    off = float(np.median([st.submit_s - ps for st, ps in zip(sts, py_submit)]))  # server clock -> ours
    done = [st.done_s - off for st in sts]
    admit_wait = [st.admit_s - st.submit_s for st in sts]
    makespan = placement.max_over_ranks(t_end - reqs[0].arrival_s, dist, f"cuda:{local}")
    req_lat = [d - r.arrival_s for d, r in zip(done, reqs)]
    assert all(st.state == vxl_sph.Server.DONE for st in sts)
    srv.close()
    del srv
    return {"value": updates / makespan, "unit": UNIT, "makespan_s": makespan, "serve_steps": steps,
            "peak_active": peak_active, "peak_queued": peak_queued, "peak_device_bytes": peak_bytes,
            "tick_p50_ms": _pct(ticks_ms, 50), "tick_p99_ms": _pct(ticks_ms, 99),
            "request_p50_s": _pct(req_lat, 50), "request_p99_s": _pct(req_lat, 99),
            "admit_wait_p99_s": _pct(admit_wait, 99)}


def _plain_runs(reqs, local: int) -> list:
    """The plain path on every request: its own handle, created (and returned to the
    request's initial state) outside the timed region; then, timed per request, its ticks
    of the synchronous vxl_sph_step_tick and the final vxl_sph_read_state. Returns the
    run time and the tick times of each request."""
    import torch
    import vxl_sph
    dt_tick = float(np.float32(1.0) / np.float32(60.0))
    out = []
    for r in reqs:
        sc = vxl_sph.Scene(r.spec.params, r.spec.pos, r.spec.vel, r.spec.pmass, r.spec.n_fluid, device=local)
        sc.step_tick(dt_tick, r.spec.spans)  # tick graph captured outside the timed run
        sc.write_state(r.spec.pos, r.spec.vel)
        torch.cuda.synchronize()
        ticks = []
        t0 = time.perf_counter()
        for _ in range(r.ticks):
            ta = time.perf_counter()
            sc.step_tick(dt_tick, r.spec.spans)
            ticks.append(1e3 * (time.perf_counter() - ta))
        sc.read_state()
        out.append((time.perf_counter() - t0, ticks))
        sc.close()
    return out


def _plain_schedule(reqs, runs, updates: float, dist, local: int) -> dict:
    """The plain path serving the stream: requests one after another in arrival order,
    each starting when it has arrived and the previous one is done, each taking its
    measured run time (a request's run on an otherwise idle GPU does not depend on when
    it arrives)."""
    from vxl_sph import placement
    free_at = 0.0
    lat = []
    for r, (run, _) in zip(reqs, runs):
        start = max(r.arrival_s, free_at)
        free_at = start + run
        lat.append(free_at - r.arrival_s)
    makespan = placement.max_over_ranks(free_at - reqs[0].arrival_s, dist, f"cuda:{local}")
    ticks = [t for _, tk in runs for t in tk]
    return {"value": updates / makespan, "makespan_s": makespan, "busy_s": sum(x for x, _ in runs),
            "tick_p50_ms": _pct(ticks, 50), "tick_p99_ms": _pct(ticks, 99),
            "request_p50_s": _pct(lat, 50), "request_p99_s": _pct(lat, 99)}


def measure_served(local: int, n_requests: int = 200, rates=(50.0, 200.0, 1000.0, 2000.0), tick_scale: float = 0.05,
                   budget_bytes: int = 150 * 10**9, seed: int = 11, plain: bool = True, rank: int = 0,
                   world: int = 1, dist=None, variants: bool = True) -> dict:
    """The served workload at each arrival rate: the same requests (one seed: particle
    counts, ticks, kinds, tanks), arriving as a Poisson process of that rate, served by
    continuous batching; against the plain path serving them one by one. With `variants`,
    at the highest rate also: a batch cap of 8M fluid particles per substep (the latency
    knob) and a 12 GB budget (admission limited by memory). On several GPUs each rank
    serves its share of the stream (placement by work, no collective on the data path);
    throughput is summed over ranks over the longest makespan."""
    from vxl_sph import placement, scenes

    base = scenes.served_stream(n_requests, 1.0, seed, tick_scale=tick_scale)
    if world > 1:
        mine = placement.assign_scenes([r.spec.n_fluid * r.ticks for r in base], world)[rank]
        base = [base[q] for q in mine]
    sub = base[0].spec.params.substeps
    updates = placement.sum_over_ranks(sum(r.spec.n_fluid * sub * r.ticks for r in base), dist, f"cuda:{local}")
    runs = _plain_runs(base, local) if plain else None
    points = []
    for rate in rates:
        reqs = [scenes.Request(r.arrival_s / rate, r.spec, r.ticks) for r in base]
        pt = {"rate_per_s": rate, **_serve_once(reqs, local, budget_bytes, dist=dist, world=world)}
        if runs is not None:
            pt["plain"] = _plain_schedule(reqs, runs, updates, dist, local)
            pt["speedup_vs_plain"] = pt["plain"]["makespan_s"] / pt["makespan_s"]
        points.append(pt)
    out = {
        "workload": f"{n_requests} requests, Poisson arrivals, N log-U[8192, 1048576], ticks U[60, 600] x "
                    f"{tick_scale}, dam-break or sloshing (closed tanks), budget {budget_bytes / 1e9:.0f} GB, seed {seed}",
        "requests": n_requests, "requests_this_rank": len(base),
        "fluid_particles_this_rank": sum(r.spec.n_fluid for r in base),
        "ticks_total": sum(r.ticks for r in base), "updates": updates, "unit": UNIT,
        "plain_call": "per request: a handle created before the timed run; its ticks of vxl_sph_step_tick and a "
                      "read_state, timed; the stream served one request after another in arrival order",
        "rates": points,
    }
    top = max(points, key=lambda q: q["rate_per_s"])
    out.update({k: top[k] for k in ("rate_per_s", "value", "makespan_s", "tick_p50_ms", "tick_p99_ms",
                                    "request_p50_s", "request_p99_s")})
    if "speedup_vs_plain" in top:
        out["speedup_vs_plain"] = top["speedup_vs_plain"]
    if variants:
        reqs = [scenes.Request(r.arrival_s / top["rate_per_s"], r.spec, r.ticks) for r in base]
        out["batch_cap"] = {"max_fluid_particles": 8_000_000, "rate_per_s": top["rate_per_s"],
                            **_serve_once(reqs, local, budget_bytes, batch_cap=8_000_000, dist=dist, world=world)}
        out["budget_limited"] = {"budget_bytes": 12 * 10**9, "rate_per_s": top["rate_per_s"],
                                 **_serve_once(reqs, local, 12 * 10**9, dist=dist, world=world)}
    return out


def run_mix(args) -> None:
    """--workload batched|served: the batched or served form as the headline line."""
    import torch
    import vxl_sph
    local = int(os.environ.get("LOCAL_RANK", "0"))
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    torch.cuda.set_device(local)
    dist = None
    if world > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300))
    vxl_sph.load()
    clocks = ClockSampler(local)
    clocks.start()
    if args.workload == "batched":
        m = measure_batched(local, args.steps, args.warmup, n_scenes=args.scenes, plain_loop=not args.no_plain,
                            rank=rank, world=world, dist=dist)
        value, ms = m["value"], m["ms_per_tick"]
        cfg = {"workload": "batched", **{k: m[k] for k in ("scenes", "n_fluid", "substeps")},
               "step": "one 60 Hz tick of every scene", "l2": "flushed between ticks",
               "parallelism": f"scenes packed in one handle per GPU, scene-parallel x{world}"}
    else:
        m = measure_served(local, n_requests=args.requests, rates=args.rates, tick_scale=args.tick_scale,
                           plain=not args.no_plain, rank=rank, world=world, dist=dist)
        value, ms = m["value"], None
        cfg = {"workload": "served", "requests": m["requests"], "rates_per_s": list(args.rates),
               "step": "one serve step = one substep of every admitted scene",
               "parallelism": f"continuous batching per GPU, request-parallel x{world}"}
    clk = clocks.stop()
    if rank == 0:
        line = {"metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
                "warmup": args.warmup, "ms_per_step": ms, "higher_is_better": True, "scaling": "weak",
                "vs_baseline": None, "dtype": "f32", "data": "synthetic: seeded tanks (no public dataset exists)",
                "config": cfg, args.workload: m, "clocks": clk}
        print(json.dumps(line), flush=True)
    if dist:
        dist.barrier()
        dist.destroy_process_group()


def run_ncu_case(args) -> None:
    """Smallest run of the workload for a profiler: build, `--warmup` ticks, exit."""
    import vxl_sph
    vxl_sph.load()
    dt_tick = float(np.float32(1.0) / np.float32(60.0))
    if args.workload == "batched":
        from vxl_sph import scenes
        specs = scenes.batched_mix(args.scenes)
        batch = vxl_sph.Batch(specs)
        for _ in range(max(args.warmup, 1)):
            batch.step_tick(dt_tick)
        batch.close()
        print(json.dumps({"ncu_case": "batched", "scenes": args.scenes, "ticks": max(args.warmup, 1),
                          "n_fluid": sum(s.n_fluid for s in specs), "n_boundary": sum(s.n_boundary for s in specs)}))
        return
    if args.workload == "dam10m" and args.ncu_block:
        from vxl_sph import scenes
        spec = scenes.dam10m_block(args.ncu_block)
    else:
        spec = build_scene(args.workload)
    scene = vxl_sph.Scene(spec.params, spec.pos, spec.vel, spec.pmass, spec.n_fluid)
    if args.ncu_density >= 0:
        block, tile, waves, _ = scene.tuning()
        scene.set_tuning(block, tile, waves, args.ncu_density)
    for _ in range(max(args.warmup, 1)):
        scene.step_tick(dt_tick, spec.spans)
    scene.close()
    print(json.dumps({"ncu_case": spec.name, "ticks": max(args.warmup, 1), "n_fluid": spec.n_fluid,
                      "n_boundary": spec.n_boundary}))


def launch_ranks(n: int, argv=None) -> int:
    """`--gpus N` started directly (no WORLD_SIZE in the environment): run N ranks of this
    script with the same arguments under torch.distributed.run on this node (one process
    per GPU, rendezvous on 127.0.0.1) and return the launcher's exit status."""
    import socket
    with socket.socket() as sk:
        sk.bind(("127.0.0.1", 0))
        port = sk.getsockname()[1]
    cmd = [sys.executable, "-m", "torch.distributed.run", "--nnodes=1", f"--nproc-per-node={n}",
           "--master-addr", "127.0.0.1", "--master-port", str(port), str(Path(__file__).resolve()),
           *(sys.argv[1:] if argv is None else argv)]
    return subprocess.call(cmd)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--workload", default="dam10m", choices=["dam0", "dam1", "dam10m", "batched", "served"])
    ap.add_argument("--requests", type=int, default=200, help="served: number of requests")
    ap.add_argument("--rates", type=float, nargs="+", default=[50.0, 200.0, 1000.0, 2000.0],
                    help="served: Poisson arrival rates swept (1/s)")
    ap.add_argument("--tick-scale", type=float, default=0.05, help="served: factor on the 60-600 tick counts")
    ap.add_argument("--no-mix", action="store_true", help="skip the batched/served comparison in the plain run")
    ap.add_argument("--scenes", type=int, default=256, help="batched: number of tanks")
    ap.add_argument("--no-plain", action="store_true", help="batched/served: skip the plain-path comparison")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-coupled", action="store_true", help="skip the coupled-bodies line of scenes with boxes")
    ap.add_argument("--cpu-threads", type=int, default=0, help="reference arm: host threads (default: all)")
    ap.add_argument("--ncu-case", action="store_true", help="build + warm-up ticks only (for ncu captures)")
    ap.add_argument("--ncu-density", type=int, default=-1,
                    help="ncu case: density kernel (0 walk, 1 grouped; default: the handle's)")
    ap.add_argument("--ncu-block", type=int, default=0,
                    help="ncu case of dam10m: an N^3 fluid block in the same tank (bins still doubled)")
    args = ap.parse_args()
    if args.gpus > 1 and "WORLD_SIZE" not in os.environ and not args.ncu_case:
        sys.exit(launch_ranks(args.gpus))
    if args.ncu_case:
        run_ncu_case(args)
    elif args.impl == "reference":
        run_reference(args)
    elif args.workload in ("batched", "served"):
        run_mix(args)
    else:
        run_ours(args)


if __name__ == "__main__":
    main()
