#!/usr/bin/env python
"""Benchmark of the FDTD time stepping: Mcell-updates/s on the large
dispersive box (512³ cells, 0.5 mm, CPML 10, two-pole Lorentz sphere of
radius 80 cells, 20-cell Drude slab, soft E_x sheet source, leapfrog ADE),
with the share of the HBM roofline it reaches.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

One process per GPU (torchrun for N > 1): every rank steps its own replica
of the model (the configuration fits one GPU; there is no data exchange
between models), so ``scaling`` is weak and ``value`` counts the cell
updates of all ranks over the slowest rank's device time. Rank 0 prints
one JSON line.

* ``value``: device time of K steps (CUDA events on the engine's stream,
  barrier + synchronize on both sides, max over ranks). Inputs (3.2 GB of
  fields plus coefficients) are far larger than the 126 MB L2, so no flush
  is needed between steps.
* ``e2e``: the same metric through the C ABI step by step, as a host that
  feeds a source and reads a probe every step would: per step the source
  amplitude goes host→device, the step runs, and the probe's new sample
  comes back device→host.
* ``roofline``: the dominant kernel's algorithmic bytes per launch over its
  mean launch time (CUDA events around each launch inside the timed
  region), against the measured HBM copy bandwidth; ``traffic`` is the
  DRAM bytes of one launch from the committed ncu summary.
* ``cpu_baseline``: the oracle (the reference engine's step restated in
  C++, one thread per x-slab like the reference's pool) on a bounded sample
  of the same model on this host's cores.
* ``--impl reference`` times that CPU restatement alone (rank 0).
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "Mcell-updates/s"
ALGO_BYTES_CELL_FIELDS = 48.0  # read u, i and write u, i (f32 × 6 × 2)


def parse():
    ap = argparse.ArgumentParser(description=__doc__.split("\n")[0])
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=200)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--cells", type=int, default=512, help="cells per axis (default: the configuration's 512)")
    ap.add_argument("--schedule", type=int, default=0,
                    help="0 automatic, 1 per-operator, 2 fused, 3 two kernels, 4 split, 5 sweep, 6 interior, 7 marching")
    ap.add_argument("--interior-planes", type=int, default=0, help="planes per block of the interior kernel (0: default)")
    ap.add_argument("--march-shape", type=int, default=0, help="marching kernel tile shape (0..3)")
    ap.add_argument("--march-planes", type=int, default=32, help="planes per block of the marching kernel")
    ap.add_argument("--row-cpml", action="store_true", help="split schedule: the CPML inside the updates (opt-in)")
    ap.add_argument("--workload", choices=["box", "sweep", "learned"], default="box",
                    help="box: the 512^3 dispersive box (the headline line); sweep: the batched patch-variant "
                         "sweep; learned: training and held-out evaluation of the learned early stop")
    ap.add_argument("--models", type=int, default=64, help="sweep: number of patch variants")
    ap.add_argument("--sweep-cells", type=int, nargs=2, default=[60, 160], help="sweep: N range (N x N x N cells)")
    ap.add_argument("--max-steps", type=int, default=40000, help="sweep: step limit per model")
    ap.add_argument("--train", type=int, default=2000, help="learned: training variants")
    ap.add_argument("--test", type=int, default=256, help="learned: held-out variants")
    ap.add_argument("--learn-cells", type=int, nargs=2, default=[30, 50], help="learned: N range of the variants")
    ap.add_argument("--epochs", type=int, default=60, help="learned: training epochs")
    ap.add_argument("--threshold", type=float, default=0.1, help="learned: window residual threshold")
    return ap.parse_args()


def max_over_ranks(x: float, world: int, device=None) -> float:
    """The largest x over the ranks (the slowest rank's time): an all-reduce
    of one f64 on the process group (NCCL on the GPU, gloo on the CPU)."""
    if world <= 1:
        return x
    import torch
    import torch.distributed as dist

    t = torch.tensor([x], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def aggregate(world: int, cells: int, steps: int, seconds: float) -> float:
    """Whole-job Mcell-updates/s: every rank steps its own replica, so the
    job updates world × cells × steps cells in the slowest rank's time."""
    return world * cells * steps / seconds / 1e6


def dist_env():
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return rank, world, local


def workload(cells: int, steps: int):
    from ems_b200 import workloads as W

    if cells == 512:
        return W.dispersive_box(steps=steps)
    # Proportionally scaled box (for small trial runs only).
    s = cells / 512.0
    return W.dispersive_box(n=cells, radius=80 * s, slab=max(2, int(round(20 * s))), cpml=max(4, int(round(10 * s))),
                            steps=steps)


def algorithmic_bytes(w) -> dict:
    """Bytes a step must move at least (per step): fields 48 B per cell, the
    CPML ψ read and written (8 B per ψ per layer node), the pole state j, q
    (f64) read and written (32 B per pole) and the prev field value of each
    pole edge; coefficients count 0 (a handful of distinct rows)."""
    import ems_b200 as E

    m = w.model
    nx, ny, nz = m.nodes
    desc = E.EngineDesc.from_address(m.desc)
    psi = 0
    poles = 0
    pole_edges = 0
    for k in range(desc.n_ops):
        op = E.OpEntry.from_address(desc.ops + k * C_sizeof_op())
        if op.kind == E.OP_CPML:
            t = E.CpmlTable.from_address(op.table)
            for q in range(t.n_slabs):
                sl = E.CpmlSlab.from_address(t.slabs + q * E.C.sizeof(E.CpmlSlab))
                psi += int(np.prod([sl.hi[a] - sl.lo[a] for a in range(3)]))
        elif op.kind == E.OP_POLES:
            t = E.PolesTable.from_address(op.table)
            poles += t.electric.n_poles + t.magnetic.n_poles
            pole_edges += t.electric.n_edges + t.magnetic.n_edges
    cells = (nx - 1) * (ny - 1) * (nz - 1)
    b_fields = ALGO_BYTES_CELL_FIELDS * cells
    b_psi = 8.0 * psi
    b_poles = 32.0 * poles + 8.0 * pole_edges
    return {"cells": cells, "fields": b_fields, "psi": b_psi, "poles": b_poles, "total": b_fields + b_psi + b_poles,
            "psi_nodes": psi, "poles_n": poles, "pole_edges": pole_edges}


def C_sizeof_op():
    import ems_b200 as E

    return E.C.sizeof(E.OpEntry)


class Clocks:
    """Samples SM clocks and throttle reasons with nvidia-smi while running."""

    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index: int):
        self.index = index
        self.proc = None
        self.lines: list[str] = []

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.index), f"--query-gpu={self.Q}",
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except (OSError, ValueError):
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def __exit__(self, *a):
        if self.proc:
            time.sleep(0.25)
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()

    def summary(self) -> dict:
        sm, mx, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            p = [x.strip() for x in ln.split(",")]
            if len(p) < 9:
                continue
            try:
                sm.append(float(p[1]))
                mx.append(float(p[2]))
            except ValueError:
                continue
            for n, v in zip(names, p[5:9]):
                if v.lower() == "active":
                    reasons.add(n)
        if not sm:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": [], "samples": 0}
        return {"sm_mhz": statistics.median(sm), "sm_max_mhz": max(mx), "reasons": sorted(reasons),
                "samples": len(sm)}


def measured_peaks() -> dict:
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        with open(p) as f:
            d = json.load(f)
        return {"hbm_gbs": d.get("hbm_gbs"), "source": "measured"}
    return {"hbm_gbs": 6650.0, "source": "fallback"}


def profile_traffic(kernel: str, workload: str) -> float | None:
    """DRAM bytes per launch of `kernel` scaled to the full configuration,
    from the committed ncu summary (profiles/traffic.json), if present and
    recorded for this workload (None for other sizes)."""
    p = os.path.join(ROOT, "profiles", "traffic.json")
    if not os.path.exists(p):
        return None
    with open(p) as f:
        d = json.load(f).get(kernel, {})
    v = d.get("bytes_per_launch_full_config")
    return float(v) if v is not None and d.get("workload") == workload else None


def host_cpu() -> dict:
    """The host CPU model, its physical and logical core counts."""
    model = "unknown"
    try:
        with open("/proc/cpuinfo") as f:
            for line in f:
                if line.startswith("model name"):
                    model = line.split(":", 1)[1].strip()
                    break
    except OSError:
        pass
    try:
        import psutil

        phys = psutil.cpu_count(logical=False) or os.cpu_count() or 1
    except ImportError:
        phys = os.cpu_count() or 1
    return {"cpu_model": model, "physical_cores": phys, "logical_cpus": os.cpu_count() or 1}


def cpu_baseline(w, seconds: float = 15.0) -> dict:
    """The oracle on the same model, timed on this host's cores for about
    `seconds` (whole steps of the full model), with one thread per physical
    core (the reference's --numThreads at the full core count); the thread
    count the reference's default rule picks for this model
    (src/engine/mod.rs:404-428: physical cores, at most one per 4096 cells
    and one per five x-planes) is reported beside it, and timed too when it
    differs."""
    from oracle import OracleEngine

    cpu = host_cpu()

    def timed(threads):
        o = OracleEngine(w.model, threads=threads)
        t0 = time.perf_counter()
        o.run(1)
        per = max(time.perf_counter() - t0, 1e-6)
        n = max(1, min(200, int(seconds / per)))
        t0 = time.perf_counter()
        o.run(n)
        el = time.perf_counter() - t0
        th = o.threads
        o.close()
        return w.cells * n / el / 1e6, th, n

    v, th, n = timed(cpu["physical_cores"])
    o = OracleEngine(w.model, threads=0)
    rule = o.threads
    o.close()
    out = {"value": round(v, 3), "unit": METRIC, "cores": th, "kind": "port",
           "sample": f"{n} whole steps of the same {w.name} model after 1 untimed step "
                     f"(oracle: C++ restatement of the reference step, {th} threads)",
           "cpu_model": cpu["cpu_model"], "physical_cores": cpu["physical_cores"],
           "logical_cpus": cpu["logical_cpus"], "default_rule_threads": rule}
    if rule != th:
        vr, _, nr = timed(0)
        out["default_rule_value"] = round(vr, 3)
    return out


def run_reference(args):
    rank, world, _ = dist_env()
    if rank != 0:
        return 0
    w = workload(args.cells, max(args.steps + args.warmup + 10, 100))
    from oracle import OracleEngine

    cpu = host_cpu()
    o = OracleEngine(w.model, threads=cpu["physical_cores"])
    o.run(args.warmup)
    t0 = time.perf_counter()
    o.run(args.steps)
    el = time.perf_counter() - t0
    v = w.cells * args.steps / el / 1e6
    line = {
        "impl": "reference", "metric": METRIC, "value": round(v, 3), "unit": METRIC, "n_gpus": args.gpus,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": round(1e3 * el / args.steps, 3),
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
        "config": config(w, args),
        "cpu_baseline": {"value": round(v, 3), "unit": METRIC, "cores": o.threads, "kind": "port",
                         "sample": f"{args.steps} whole steps after {args.warmup} warm-up steps, "
                                   f"{o.threads} threads (C++ restatement of the reference step)",
                         **cpu},
        "e2e": {"value": round(v, 3), "unit": METRIC, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)
    return 0


def config(w, args) -> dict:
    i = w.info
    return {"workload": f"{w.name}: {i['cells']}^3 cells of {i['cell_m'] * 1e3:g} mm, CPML {i['cpml']}, "
                        f"2-pole Lorentz sphere r={i['radius']:g} cells (eps_inf 2.0), Drude slab {i['slab']} cells, "
                        f"soft E_x sheet ({i['sheet_edges']} edges), {i['scheme']} ADE, dt = "
                        f"{i['courant']} x Courant limit",
            "cells": w.cells, "seed": "0x5eed",
            "l2": "inputs larger than L2 (fields alone 3.2 GB at 512^3); no flush between steps",
            "parallelism": f"replicas x{args.gpus}"}


def run_ours(args):
    import torch

    import ems_b200 as E

    rank, world, local = dist_env()
    if world > 1:
        import torch.distributed as dist
        from datetime import timedelta

        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=timedelta(seconds=600))
    dev = local if world > 1 else 0
    total_steps = args.warmup + args.steps
    w = workload(args.cells, total_steps + 10)
    eng = E.Engine(w.model, device=dev)
    eng.set_schedule(args.schedule)
    if args.interior_planes:
        eng.set_interior_planes(args.interior_planes)
    eng.set_march(args.march_shape, args.march_planes)
    if args.row_cpml:
        eng.set_row_cpml(True)
    stream = torch.cuda.ExternalStream(eng.stream, device=dev)
    eng.run(args.warmup)
    torch.cuda.synchronize(dev)

    def barrier():
        if world > 1:
            torch.distributed.barrier()

    # --- timed region (no per-kernel events inside it)
    launches0 = eng.launches
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    with Clocks(dev) as clk:
        barrier()
        torch.cuda.synchronize(dev)
        e0.record(stream)
        eng.run(args.steps)
        e1.record(stream)
        torch.cuda.synchronize(dev)
        barrier()
    ms = e0.elapsed_time(e1)
    launches = eng.launches - launches0
    # Per-kernel device times from a separate pass with events around the
    # field-update kernels.
    eng.profile(True)
    eng.run(min(args.steps, 20))
    torch.cuda.synchronize(dev)
    kern = {k: eng.profile_read(k) for k in (0, 1, 2)}
    eng.profile(False)
    ms = max_over_ranks(ms, world, f"cuda:{dev}")
    value = aggregate(world, w.cells, args.steps, ms * 1e-3)

    # --- end to end through the C ABI: per step, amplitude H2D, step, probe sample D2H
    amp_op = w.source
    probe_op = w.probes[0]
    from ems_b200 import waveform_value

    t_src = lambda n: waveform_value(w.info["f0"], w.info["fc"], (n + 0.5) * w.model.dt)  # noqa: E731
    k_e2e = max(1, min(args.steps, 100))
    first = eng.timestep
    host_amp = np.array([t_src(first + q) for q in range(k_e2e)], dtype=np.float64)
    barrier()
    torch.cuda.synchronize(dev)
    t0 = time.perf_counter()
    for q in range(k_e2e):
        eng.source_amplitude(amp_op, first + q, host_amp[q:q + 1])
        eng.run(1)
        eng.last_sample(probe_op)
    el = time.perf_counter() - t0
    el = max_over_ranks(el, world, f"cuda:{dev}")
    e2e = aggregate(world, w.cells, k_e2e, el)

    if rank != 0:
        eng.close()
        if world > 1:
            torch.distributed.destroy_process_group()
        return 0

    ab = algorithmic_bytes(w)
    peaks = measured_peaks()
    # Dominant kernel: the fused step if it ran; else the H update: of the
    # two-kernel schedule (H update, CPML H, magnetic poles: reads u, reads
    # and writes i, reads and writes the H half of ψ), or the streaming H
    # update of the split and per-operator schedules (reads u, reads and
    # writes i: 36 B per cell).
    schedule = eng.schedule
    nodes = float(np.prod(w.model.nodes))
    if schedule == 7:
        # The marching kernel: reads u and i, writes both (48 B per node),
        # and reads and writes the ψ of every layer node.
        kname, (kms, kn) = "march", kern[2]
        per_launch = 48.0 * nodes + ab["psi"]
    elif schedule == 6:
        # The one-pass kernel over the interior box: reads u and i, writes
        # both (48 B per node).
        (blo, bhi) = eng.interior_box
        kname, (kms, kn) = "interior", kern[2]
        per_launch = 48.0 * float(np.prod([h - l for l, h in zip(blo, bhi)]))
    elif kern[2][1] > 0:
        kname, (kms, kn) = "fused_step", kern[2]
        per_launch = ab["total"]
    elif schedule == 5:
        # The sweep: one timed span per step over all chunks' updates and
        # slab hooks (everything but the serial hooks).
        kname, (kms, kn) = "sweep_chunks", kern[0]
        per_launch = ab["total"]
    else:
        # The H update: 36 B per cell; with the H half of ψ where the CPML
        # runs inside it (the two-kernel schedule; the split schedule's row
        # CPML, timed as one span over its launches).
        kname, (kms, kn) = ("step_h" if schedule == 3 else "update_h"), kern[0]
        inside = schedule == 3 or (schedule == 4 and eng.row_cpml)
        per_launch = 36.0 * ab["cells"] + (0.5 * ab["psi"] if inside else 0.0)
    achieved = per_launch / (kms * 1e-3 / kn) / 1e9 if kn else None
    step_gbs = ab["total"] / (ms * 1e-3 / args.steps) / 1e9 / (world)
    traffic = profile_traffic(kname, w.name)
    line = {
        "metric": METRIC, "value": round(value, 1), "unit": METRIC, "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": round(ms / args.steps, 4), "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f32 fields, f64 pole state", "data": "synthetic",
        "config": config(w, args),
        "roofline": {"bound": "hbm", "kernel": kname, "achieved": round(achieved, 1) if achieved else None,
                     "peak": peaks["hbm_gbs"], "unit": "GB/s",
                     "frac": round(achieved / peaks["hbm_gbs"], 4) if achieved else None,
                     "traffic": traffic, "peak_source": peaks["source"],
                     "algorithmic_bytes_per_launch": per_launch,
                     "mean_launch_ms": round(kms / kn, 4) if kn else None},
        "step_roofline": {"algorithmic_bytes_per_step": ab["total"], "bytes_per_cell": round(ab["total"] / ab["cells"], 2),
                          "achieved_gbs": round(step_gbs, 1), "frac": round(step_gbs / peaks["hbm_gbs"], 4)},
        "kernels_ms": {("h_update", "e_update", {6: "interior", 7: "march"}.get(schedule, "fused_step"))[k]:
                       {"ms": round(v[0], 3), "launches": v[1]} for k, v in kern.items() if v[1]},
        "schedule": {1: "per-operator kernels", 2: "fused single pass", 3: "two kernels", 4: "split",
                     5: "sweep", 6: "interior", 7: "marching"}[schedule],
        "e2e": {"value": round(e2e, 1), "unit": METRIC, "h2d_bytes_per_step": 8, "d2h_bytes_per_step": 8,
                "steps": k_e2e},
        "gpu_launches": launches,
        "clocks": clk.summary(),
    }
    if world == 1:
        line["cpu_baseline"] = cpu_baseline(w)
    eng.close()
    print(json.dumps(line), flush=True)
    if world > 1:
        torch.distributed.destroy_process_group()
    return 0


def run_sweep(args):
    """The batched sweep: seeded patch variants of uneven sizes run to the
    −40 dB energy criterion (checked every 50 steps), batched (one graph per
    step over all models, models frozen as they stop) and one at a time on
    the same GPU; both must give every model the same outcome."""
    import torch

    import ems_b200 as E
    from ems_b200 import workloads as W

    ws = [W.sweep_variant(s, cells=tuple(args.sweep_cells), steps=args.max_steps) for s in range(args.models)]
    t_exc = E.waveform_duration(2e9, 1.5e9)
    lims = [E.energy_decay_limits(args.max_steps, -40.0, w.model.dt, excitation_end=t_exc, interval=50) for w in ws]
    cells = [w.info["cells"] for w in ws]
    t0 = time.perf_counter()
    b = E.Batch([w.model for w in ws], max_steps=args.max_steps)
    t1 = time.perf_counter()
    with Clocks(0) as clk:
        outs_b = E.run_until_batch(b, lims)
        torch.cuda.synchronize(0)
    t2 = time.perf_counter()
    b.close()
    upd_b = sum(c * o.steps for c, o in zip(cells, outs_b))
    t_one, outs_1 = 0.0, []
    for w, lim in zip(ws, lims):
        g = E.Engine(w.model)
        ta = time.perf_counter()
        outs_1.append(E.run_until(g, lim))
        torch.cuda.synchronize(0)
        t_one += time.perf_counter() - ta
        g.close()
    # The same outcome per model: stop reason, step and number of checks,
    # and the final energy (a reduction in another order: within 1e-12).
    same = all((x.reason, x.steps, x.checks) == (y.reason, y.steps, y.checks) and
               abs(x.energy - y.energy) <= 1e-12 * max(abs(y.energy), 1e-300) for x, y in zip(outs_b, outs_1))
    line = {
        "metric": "sweep wall time", "value": round(t2 - t1, 3), "unit": "s", "higher_is_better": False,
        "n_gpus": 1, "data": "synthetic",
        "config": {"workload": f"{args.models} seeded patch variants, each on its own graded N x N x N mesh, "
                               f"N in {args.sweep_cells}, -40 dB energy criterion every 50 steps, "
                               f"max {args.max_steps} steps",
                   "total_cells": sum(cells), "cells_min": min(cells), "cells_max": max(cells)},
        "clocks": clk.summary(),
        "batched": {"s": round(t2 - t1, 3), "create_s": round(t1 - t0, 3),
                    "mcell_updates_per_s": round(upd_b / (t2 - t1) / 1e6, 1)},
        "one_at_a_time": {"s": round(t_one, 3), "mcell_updates_per_s": round(upd_b / t_one / 1e6, 1)},
        "speedup": round(t_one / (t2 - t1), 3),
        "steps": {"min": min(o.steps for o in outs_b), "max": max(o.steps for o in outs_b),
                  "reasons": sorted({o.reason for o in outs_b})},
        "same_outcomes": same,
    }
    print(json.dumps(line), flush=True)
    return 0 if same else 1


def run_learned(args):
    """The learned early stop: train the network on port records of seeded
    patch variants generated by the batched solver, then run held-out
    variants to the −40 dB criterion plainly and with the learned stop (both
    batched); report steps saved, sweep times and the |S11| error over
    1-3 GHz of the stopped runs against the plain ones (and, for contrast,
    of stopping at the same step without the network's tail)."""
    import torch

    import ems_b200 as E
    from ems_b200 import learn as Lr
    from ems_b200 import workloads as W

    cells = tuple(args.learn_cells)
    t0 = time.perf_counter()
    X, Y = [], []
    phase = {"build_s": 0.0, "create_s": 0.0, "run_s": 0.0, "extract_s": 0.0}
    for c0 in range(0, args.train, 1000):
        ta = time.perf_counter()
        ws = [W.patch_variant(10_000 + q, cells=cells, steps=args.max_steps) for q in range(c0, min(args.train, c0 + 1000))]
        need = [Lr.steps_needed(w.model.dt) for w in ws]
        tb_ = time.perf_counter()
        bb = E.Batch([w.model for w in ws], max_steps=max(need))
        tc = time.perf_counter()
        done = 0
        for target in sorted(set(need)):  # each model runs the steps its record needs, then is frozen
            bb.run(target - done)
            done = target
            for q, nq in enumerate(need):
                if nq == target:
                    bb.set_active(q, False)
        torch.cuda.synchronize()
        td = time.perf_counter()
        for q, w in enumerate(ws):
            x, y = Lr.example(bb.samples(q, w.port, 1), bb.samples(q, w.port, 2), w.model.dt)
            X.append(x)
            Y.append(y)
        bb.close()
        te = time.perf_counter()
        for k, v in zip(phase, (tb_ - ta, tc - tb_, td - tc, te - td)):
            phase[k] += v
        del ws
    t_data = time.perf_counter() - t0
    Xd, Yd = torch.from_numpy(np.stack(X)).cuda(), torch.from_numpy(np.stack(Y)).cuda()
    net = Lr.Net(seed=0)
    t1 = time.perf_counter()
    hist = Lr.train(net, Xd, Yd, epochs=args.epochs, batch=64, lr=2e-3)
    torch.cuda.synchronize()
    t_train = time.perf_counter() - t1

    ws = [W.patch_variant(20_000 + q, cells=cells, steps=args.max_steps) for q in range(args.test)]
    models, ports = [w.model for w in ws], [w.port for w in ws]
    t_exc = E.waveform_duration(2e9, 1.5e9)
    lims = [E.energy_decay_limits(args.max_steps, -40.0, m.dt, excitation_end=t_exc, interval=50) for m in models]
    b = E.Batch(models, max_steps=args.max_steps)
    ta = time.perf_counter()
    plain = E.run_until_batch(b, lims)
    torch.cuda.synchronize()
    t_plain = time.perf_counter() - ta
    recs = [(b.samples(q, ports[q], 1), b.samples(q, ports[q], 2)) for q in range(len(models))]
    b.close()
    b = E.Batch(models, max_steps=args.max_steps)
    ls = Lr.LearnedStop(b, ports, [m.dt for m in models], net, threshold=args.threshold)
    tb = time.perf_counter()
    learned = E.run_until_batch(ls, lims)
    torch.cuda.synchronize()
    t_learned = time.perf_counter() - tb
    lrecs = [(b.samples(q, ports[q], 1), b.samples(q, ports[q], 2)) for q in range(len(models))]
    b.close()

    freqs = np.linspace(1e9, 3e9, 81)
    err, err_cut, steps_l, fallback_same = [], [], [], True
    for q, m in enumerate(models):
        v, i = recs[q]
        full = Lr.s11_db(np.arange(len(v)), v, i, m.dt, freqs)
        if q in ls.stopped:
            stop = ls.stopped[q]
            st, vv, ii = Lr.spliced(lrecs[q][0], lrecs[q][1], ls.pred[q], stop, m.dt)
            err.append(float(np.max(np.abs(Lr.s11_db(st, vv, ii, m.dt, freqs) - full))))
            cut = Lr.s11_db(np.arange(stop), lrecs[q][0][:stop], lrecs[q][1][:stop], m.dt, freqs)
            err_cut.append(float(np.max(np.abs(cut - full))))
            steps_l.append(stop)
        else:
            steps_l.append(learned[q].steps)
            fallback_same &= learned[q].steps == plain[q].steps and np.array_equal(lrecs[q][0], v)
    steps_p = [o.steps for o in plain]
    upd = lambda st: sum(w.info["cells"] * n for w, n in zip(ws, st))  # noqa: E731
    e = np.array(err) if err else np.zeros(0)
    line = {
        "metric": "sweep wall time, learned stop vs plain", "value": round(t_learned, 3), "unit": "s",
        "higher_is_better": False, "n_gpus": 1, "data": "synthetic",
        "config": {"workload": f"patch variants N x N x N/2, N in {list(cells)}; {args.train} training and "
                               f"{args.test} held-out variants; -40 dB criterion every 50 steps, max {args.max_steps}",
                   "k_in": Lr.K_IN, "t_out": Lr.T_OUT, "stride": Lr.STRIDE, "window": Lr.WINDOW,
                   "dt_ref_ps": Lr.DT_REF * 1e12,
                   "threshold": args.threshold, "params": int(net.p.numel()), "dtype": "bf16 GEMM, f32 accumulate"},
        "plain": {"s": round(t_plain, 3), "steps": int(sum(steps_p)), "mcell_updates": round(upd(steps_p) / 1e6, 1)},
        "learned": {"s": round(t_learned, 3), "steps": int(sum(steps_l)), "stopped": len(ls.stopped),
                    "fallback": args.test - len(ls.stopped), "fallback_identical": bool(fallback_same)},
        "speedup": round(t_plain / t_learned, 3),
        "steps_saved": round(1.0 - sum(steps_l) / max(1, sum(steps_p)), 4),
        "s11_err_db": {"median": round(float(np.median(e)), 4) if e.size else None,
                       "p90": round(float(np.percentile(e, 90)), 4) if e.size else None,
                       "max": round(float(e.max()), 4) if e.size else None,
                       "within_0.5dB": round(float(np.mean(e <= 0.5)), 4) if e.size else None},
        "s11_err_db_truncated_without_net": {"median": round(float(np.median(err_cut)), 4) if err_cut else None,
                                             "max": round(float(np.max(err_cut)), 4) if err_cut else None},
        "training": {"data_s": round(t_data, 2), "data_phases_s": {k: round(v, 2) for k, v in phase.items()},
                     "train_s": round(t_train, 2), "loss_first": round(hist[0], 6),
                     "loss_last": round(hist[-1], 6), "epochs": args.epochs},
    }
    print(json.dumps(line), flush=True)
    return 0


def main():
    args = parse()
    if args.impl == "reference":
        return run_reference(args)
    if args.workload == "sweep":
        return run_sweep(args)
    if args.workload == "learned":
        return run_learned(args)
    return run_ours(args)


if __name__ == "__main__":
    sys.exit(main())
