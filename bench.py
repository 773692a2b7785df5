#!/usr/bin/env python
"""Benchmark of the B200 WCSPH plain step (one JSON line on rank 0).

A step is one 60 Hz tick of the plain single-scene path: 10 substeps of grid
rebuild (cell keys + stable counting sort), density + EOS, and force + XSPH +
integration with the Akinci wall terms and per-body reactions, on a seeded dam-break
scene resident in HBM. value = fluid particle-updates per second (one update = one fluid
particle through one full substep), summed over ranks, divided by the slowest rank's
device time. Multi-GPU runs are independent replicas (each rank steps its own scene;
no collective on the data path), so scaling is weak.

  python bench.py [--gpus N] [--steps K] [--warmup W] [--workload dam1|dam0|dam10m]
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


def cpu_baseline(spec, budget_s: float = 12.0) -> dict:
    """The oracle (C++ restatement of the reference's phase-parallel CPU path) on the host
    cores, on a bounded sample of the same workload: whole substeps from the scene's
    initial state until budget_s of wall time is used."""
    from oracle import oracle as orc
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
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    spec = build_scene(args.workload)
    from oracle import oracle as orc
    cores = len(os.sched_getaffinity(0)) if hasattr(os, "sched_getaffinity") else os.cpu_count()
    o = orc.OracleSystem.from_scene(spec, threads=cores)
    dt_sub = float(np.float32(np.float32(1.0) / np.float32(60.0)) / np.float32(spec.params.substeps))
    # one step = one substep of the workload (a bounded sample of the tick the GPU arm
    # times; the metric is per particle-update so the two are comparable)
    for _ in range(args.warmup):
        o.substep(dt_sub)
    times = []
    for _ in range(args.steps):
        t0 = time.perf_counter()
        o.substep(dt_sub)
        times.append(time.perf_counter() - t0)
    total = sum(times)
    value = spec.n_fluid * args.steps / total
    line = {
        "impl": "reference", "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": args.gpus,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1e3 * total / args.steps,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
        "data": "synthetic (seeded dam break)",
        "config": {"workload": spec.name, "n_fluid": spec.n_fluid, "n_boundary": spec.n_boundary,
                   "step": "one substep on the host cores (reference CPU path restated in C++; Rust not buildable here)"},
        "cpu_baseline": {"value": value, "unit": UNIT, "cores": cores, "kind": "port",
                         "sample": f"{args.steps} substeps of {spec.name} after {args.warmup} warm-up substeps"},
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

    for _ in range(max(args.warmup, 3)):
        scene.step_tick_async(dt_tick, spec.spans)
        scene.sync()

    l2_flush = torch.empty(256 << 20, dtype=torch.uint8, device=f"cuda:{local}")
    evs = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(args.steps)]
    scene.set_profile(True)
    scene.step_tick_async(dt_tick, spec.spans)  # capture the profiled graph outside the timed region
    scene.sync()
    scene.set_profile(True)  # reset accumulators

    clocks = ClockSampler(local)
    torch.cuda.synchronize()
    if dist:
        dist.barrier()
    clocks.start()
    for k in range(args.steps):
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
    clk = clocks.stop()
    step_ms = [a.elapsed_time(b) for a, b in evs]
    total_ms = sum(step_ms)
    prof = scene.profile()
    stats = scene.stats()
    cells = int(stats.cells)

    t_max = total_ms
    if dist:
        t = torch.tensor([total_ms], device=f"cuda:{local}")
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        t_max = float(t.item())
    updates = spec.n_fluid * sub * args.steps * world
    value = updates / (t_max / 1e3)

    # dominant kernel and its roofline
    peak, peak_kind = hbm_peak()
    dom = max(prof.items(), key=lambda kv: kv[1][0])
    dom_name, (dom_ms, dom_n) = dom
    prof_total = sum(v[0] for v in prof.values())
    bytes_launch = algorithmic_bytes(dom_name, spec.n_fluid, spec.n_boundary, cells)
    avg_ms = dom_ms / max(dom_n, 1)
    achieved = (bytes_launch / (avg_ms / 1e3) / 1e9) if bytes_launch else None
    roofline = {"kernel": dom_name, "bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                "frac": (achieved / peak) if achieved else None,
                "traffic": ncu_traffic(dom_name, spec.name),
                "peak_source": f"{peak_kind} (MEASURED_PEAKS.json hbm_gbs)" if peak_kind == "measured"
                else "fallback 6650 GB/s",
                "avg_launch_ms": avg_ms, "launches": dom_n, "share": dom_ms / prof_total if prof_total else None,
                "algorithmic_bytes_per_launch": bytes_launch,
                "substep": {"bytes": substep_bytes(spec.n_fluid, spec.n_boundary, cells),
                            "ms": total_ms / (args.steps * sub)},
                "kernels_ms_per_substep": {k: v[0] / max(args.steps * sub, 1) for k, v in sorted(prof.items())}}
    sb = roofline["substep"]
    sb["achieved_gbs"] = sb["bytes"] / (sb["ms"] / 1e3) / 1e9
    sb["frac"] = sb["achieved_gbs"] / peak

    # e2e: through the C ABI with pinned host buffers: H2D state, one tick, D2H state
    pin_p = torch.empty((spec.n_total, 3), dtype=torch.float32, pin_memory=True).numpy()
    pin_v = torch.empty((spec.n_total, 3), dtype=torch.float32, pin_memory=True).numpy()
    scene.set_profile(False)
    scene.read_state(out=(pin_p, pin_v))
    for _ in range(2):
        scene.write_state(pin_p, pin_v)
        scene.step_tick(dt_tick, spec.spans)
        scene.read_state(out=(pin_p, pin_v))
    torch.cuda.synchronize()
    if dist:
        dist.barrier()
    t0 = time.perf_counter()
    for _ in range(args.steps):
        scene.write_state(pin_p, pin_v)
        scene.step_tick(dt_tick, spec.spans)
        scene.read_state(out=(pin_p, pin_v))
    e2e_s = time.perf_counter() - t0
    if dist:
        t = torch.tensor([e2e_s], device=f"cuda:{local}")
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        e2e_s = float(t.item())
    e2e = {"value": updates / e2e_s, "unit": UNIT, "h2d_bytes_per_step": spec.n_total * 24,
           "d2h_bytes_per_step": spec.n_total * 24,
           "api": "vxl_sph_write_state + vxl_sph_step_tick + vxl_sph_read_state, pinned host buffers"}

    cpu = None
    if world == 1 and not args.no_cpu_baseline:
        cpu = cpu_baseline(spec)

    if rank == 0:
        line = {
            "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": t_max / args.steps, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f32",
            "data": "synthetic: seeded dam break in an Akinci-walled tank (no public dataset exists)",
            "config": {"workload": spec.name, "n_fluid": spec.n_fluid, "n_boundary": spec.n_boundary,
                       "substeps": sub, "cells": cells, "step": "one 60 Hz tick (10 substeps)",
                       "l2": "flushed between steps (256 MiB write outside the timed events)",
                       "parallelism": f"replicas x{world}", "h": spec.params.smoothing_radius,
                       "spacing": spec.spacing, "fill": spec.meta.get("fill")},
            "roofline": roofline,
            "cpu_baseline": cpu,
            "e2e": e2e,
            "gpu_launches": int(stats.launches_last_tick) * args.steps,
            "clocks": clk,
            "step_ms": step_ms,
        }
        print(json.dumps(line), flush=True)
    scene.close()
    if dist:
        dist.destroy_process_group()


def run_ncu_case(args) -> None:
    """Smallest run of the workload for a profiler: build, `--warmup` ticks, exit."""
    import vxl_sph
    vxl_sph.load()
    spec = build_scene(args.workload)
    scene = vxl_sph.Scene(spec.params, spec.pos, spec.vel, spec.pmass, spec.n_fluid)
    dt_tick = float(np.float32(1.0) / np.float32(60.0))
    for _ in range(max(args.warmup, 1)):
        scene.step_tick(dt_tick, spec.spans)
    scene.close()
    print(json.dumps({"ncu_case": spec.name, "ticks": max(args.warmup, 1), "n_fluid": spec.n_fluid,
                      "n_boundary": spec.n_boundary}))


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--workload", default="dam1", choices=["dam0", "dam1", "dam10m"])
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--ncu-case", action="store_true", help="build + warm-up ticks only (for ncu captures)")
    args = ap.parse_args()
    if args.ncu_case:
        run_ncu_case(args)
    elif args.impl == "reference":
        run_reference(args)
    else:
        run_ours(args)


if __name__ == "__main__":
    main()
