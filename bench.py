#!/usr/bin/env python
"""Gillespie transitions/s of the B200 trajectory engine on a synthetic Boolean network.

One step = one complete simulation of the workload (all trajectories from t=0 to max_time with
window, final-state and fixed-point statistics). Default workload: the 1000-node network
(32 state words, 10 non-internal nodes, 1e6 trajectories, max_time 50, tick 0.5).

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference] [--workload c3]
                  [--mode fast|exact|epoch|epoch_dense]

Multi-GPU (torchrun, one process per GPU): every rank simulates its own block of trajectories
(random streams first_traj = rank * n), no collective on the data path (weak scaling); the step
time is the maximum over ranks.

The default line also carries, measured after its timed region, the two other targets of the
engine: `batched` (the 256-variant sweep in one persistent launch against running the variants one
by one through the NVRTC-specialised kernel, with and without the per-variant compilation the
reference needs) and `gradient` (the score-function gradient of the 50-node network against its
forward simulation). `cpu_baseline` is the CPU restatement of the measured mode's own algorithm
(fast mode: the incremental integer-rate process; exact mode: the reference's dense per-step
algorithm) on all host cores.

--impl reference runs the reference's own CUDA path (oracle/_ref/ref_run, built from its sources)
on the same B200 and workload, through simulation_runner::run_simulation with its statistics.
"""
from __future__ import annotations

import argparse
import json
import os
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

# algorithmic bytes per transition of the trajectory path: state words + time + entropy written
# by simulate, plus the non-internal words + time + entropy read back by the window statistics
# (4W + 8) + (4 W_ni + 8)
def bytes_per_transition(words: int, ni_words: int) -> int:
    return 4 * words + 8 + 4 * ni_words + 8


EXTRA_WORKLOADS = {
    "c5": "batched sweep: 256 rate-perturbed variants (lognormal sigma 0.3) of 8 networks of 20-500 nodes, "
          "1e3-1e5 trajectories each, max_time 20-200, one persistent launch",
    "c4grad": "score-function gradient of the 50-node network w.r.t. 40 rate parameters, 1e6 trajectories",
}

WORKLOADS = {
    # name: (generator, kwargs, description)
    "c1": ("c1", {}, "10-node random network, 1e5 trajectories, max_time 5, tick 0.2"),
    "c2": ("c2", {}, "100-node network, 20 % internal nodes (77 non-internal: sparse window bins), 1e6 trajectories, "
                   "max_time 100, tick 1"),
    "c2disc": ("c2", dict(discrete=True), "the same in discrete time"),
    "c2b": ("c2", dict(noninternal=20), "100-node network, 20 non-internal nodes, 1e6 trajectories, max_time 100"),
    "c3": ("c3", {}, "1000-node power-law network, 10 non-internal nodes, 1e6 trajectories, max_time 50, tick 0.5"),
    "c4": ("c4", {}, "50-node network with 40 rate parameters, 8 outputs, 1e6 trajectories"),
}


def load_peaks() -> dict:
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            return json.load(f)
    except OSError:
        return {}


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled every 200 ms during the timed region."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device: int):
        self.device = device
        self.proc = None
        self.lines: list[str] = []
        self.thread = None

    def start(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--id={self.device}", f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits",
                 "-lms", "200"], stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
        except OSError:
            self.proc = None
            return
        self.thread = threading.Thread(target=self._read, daemon=True)
        self.thread.start()

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def stop(self) -> dict:
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        if self.thread:
            self.thread.join(timeout=2)
        sm, smax, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in self.lines:
            parts = [p.strip() for p in line.split(",")]
            if len(parts) < 9:
                continue
            try:
                sm.append(float(parts[1]))
                smax.append(float(parts[2]))
            except ValueError:
                continue
            for name, flag in zip(names, parts[5:9]):
                if flag.lower() == "active":
                    reasons.add(name)
        return {"sm_mhz": float(np.median(sm)) if sm else None, "sm_max_mhz": max(smax) if smax else None,
                "reasons": sorted(reasons), "samples": len(sm)}


def dist_env() -> tuple[int, int, int]:
    return int(os.environ.get("RANK", 0)), int(os.environ.get("WORLD_SIZE", 1)), int(os.environ.get("LOCAL_RANK", 0))


def make_workload(name: str, samples: int | None):
    from maboss.gpu_b200 import synth
    gen, kw, desc = WORKLOADS[name]
    bnd, cfg = getattr(synth, gen)(**kw)
    return bnd, cfg, desc


ORACLE_MODES = {0: "exact (the reference's dense per-step algorithm, XORWOW)",
                1: "fast process, every rate re-evaluated each step",
                2: "fast process computed incrementally as the GPU fast kernel does (unstable sets, word sums, "
                   "dependents only)"}


def cpu_baseline(bnd: str, cfg: str, sample: int, mode: int, threads: int) -> dict:
    """The oracle (C++/OpenMP restatement of the path) on a bounded sample."""
    from oracle.oracle import OracleModel, build
    build()
    o = OracleModel(bnd, cfg)
    t = time.perf_counter()
    r = o.run(n=sample, mode=mode, threads=threads)
    dt = time.perf_counter() - t
    return {"value": r["transitions"] / dt, "transitions": r["transitions"], "seconds": dt, "trajectories": sample}


def cpu_baseline_sized(bnd: str, cfg: str, mode: int, threads: int, target_s: float, cap: int) -> dict:
    """cpu_baseline on a sample sized from a short probe to take about target_s seconds."""
    probe = cpu_baseline(bnd, cfg, max(64, threads * 8), mode, threads)
    per_traj = probe["seconds"] / probe["trajectories"]
    sample = int(max(64, min(cap, target_s / max(per_traj, 1e-9))))
    return cpu_baseline(bnd, cfg, sample, mode, threads)


def reference_sample(n: int, state_words: int) -> int:
    """Trajectories of the reference arm's runs: the workload's count, capped below the size at which
    the reference's int buffer sizes and indices overflow (batch * 100 * state words <= INT_MAX,
    simulation_runner.cu:68, window_average_small.cu:71), rounded down to a multiple of 10,000."""
    cap = (2147483647 // (100 * state_words)) // 10_000 * 10_000
    return min(n, cap)


def run_reference(args) -> None:
    """The reference's own CUDA build (oracle/_ref/ref_run) on this workload: W warm-up runs, then K
    timed runs of simulation_runner::run_simulation with its three statistics plugins (device time
    by CUDA events on the legacy stream it launches on; e2e: the host clock around run_simulation +
    finalize, which includes its allocations, initial-state upload and result copies)."""
    rank, world, _ = dist_env()
    if rank != 0:
        return
    from oracle import reference

    bnd, cfg, desc = make_workload(args.workload, args.samples)
    import torch

    if not torch.cuda.is_available():
        print(json.dumps({"impl": "reference", "unavailable": "no GPU on this host: the reference's path is CUDA "
                                                              "code (its CUDA build runs on the B200)"}))
        return
    if not reference.available():
        print(json.dumps({"impl": "reference", "unavailable": "the reference build oracle/_ref/ref_run is absent "
                                                              "(built by oracle/refbuild from the reference sources)"}))
        return
    import maboss.gpu_b200 as mb

    model = mb.Model(bnd, cfg)
    n_work = int(args.samples or model.constant("sample_count"))
    words = (model.num_nodes + 31) // 32
    n = args.ref_samples or reference_sample(n_work, words)
    try:
        r = reference.run_text(bnd, cfg, samples=n, warmup=args.warmup, runs=args.steps, dump=False, timeout=3000)
    except reference.Refused as e:
        print(json.dumps({"impl": "reference", "unavailable": f"the reference refuses this input: {e}"}))
        return
    dev_ms, host_ms = r["device_ms"], r["host_ms"]
    value = r["transitions"] * len(dev_ms) / (sum(dev_ms) / 1e3)
    e2e = r["transitions"] * len(host_ms) / (sum(host_ms) / 1e3)
    if n == n_work:
        which = "the whole workload"
    else:
        which = (f"of the workload's {n_work}: the largest multiple of 10,000 below the reference's int "
                 f"overflow at batch * 100 * {words} state words")
    sample = f"{n} trajectories per run ({which}), the reference's CUDA path on the B200"
    line = {
        "impl": "reference", "metric": "Gillespie transitions/s", "value": value, "unit": "transitions/s",
        "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": float(np.mean(dev_ms)), "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "f32", "data": "synthetic",
        "config": {"workload": f"{args.workload}: {desc}", "trajectories": n, "workload_trajectories": n_work,
                   "transitions_per_step": r["transitions"], "nvrtc_nvjitlink_compile_s": round(r["compile_s"], 2),
                   "build": "reference sources (src/) compiled by oracle/refbuild, MAX_NODES=1024, sm_100, "
                            "kernels NVRTC + nvJitLink LTO-linked at run time as the reference does",
                   "l2": "not flushed (every run allocates and writes a trajectory buffer of "
                         f"{n * 100 * (4 * words + 8) / 1e9:.1f} GB, larger than L2)"},
        "cpu_baseline": {"value": value, "unit": "transitions/s", "cores": 0, "kind": "reference",
                         "sample": sample + " (a GPU run: the reference has no CPU implementation of the path)"},
        "e2e": {"value": e2e, "unit": "transitions/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0,
                "host_ms_per_step": float(np.mean(host_ms))},
    }
    print(json.dumps(line), flush=True)


def _timed_line(args, value, ms_per_step, config, extra) -> dict:
    line = {"metric": "Gillespie transitions/s", "value": value, "unit": "transitions/s", "n_gpus": 1,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms_per_step, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic", "config": config}
    line.update(extra)
    return line


def batched_record(ctx, warmup: int, steps: int, per_variant_sample: int = 8) -> dict:
    """C5: the 256-variant sweep in one persistent launch (graph replay) against the variants run one
    by one through the NVRTC-specialised fast kernel of each variant (the reference bakes
    $variables into its generated code, expressions.cpp:211-214, so every variant is a compilation:
    timed with and without it) on a stated sample of variants (one per base network)."""
    import maboss.gpu_b200 as mb
    from maboss.gpu_b200 import synth

    bases, variants = synth.c5_sweep()
    models = [mb.Model(*b) for b in bases]
    batch = mb.Batch(ctx)
    nets = [batch.add_model(m) for m in models]
    for net, params, n in variants:
        batch.add_variant(nets[net], n, params)
    for _ in range(max(1, warmup)):
        batch.run(0)  # the first run tunes the launch shape and captures the CUDA graph
    ms, trans = [], 0
    for step in range(steps):
        ms.append(batch.run(step))
        trans += sum(batch.result(v).transitions for v in range(len(variants)))
    value = trans / (sum(ms) / 1e3)
    info = batch.info

    # end to end: whole runs through the public API (graph launch: clears, kernel, extraction, copies
    # to pinned memory; then every variant's result), wall clock
    d2h = 0
    t0 = time.perf_counter()
    reps = max(1, steps)
    for i in range(reps):
        batch.run(100 + i)
        d2h = 0
        for v in range(len(variants)):
            r = batch.result(v)
            d = r.dims
            _ = r.window_probs, r.final_counts, r.fixed
            d2h += d.windows * d.bins * 8 + d.windows * 8 + d.bins * 4 + len(r.fixed) * (4 * d.state_words + 4) + 64
    e2e_s = (time.perf_counter() - t0) / reps

    # one variant per base network, each through its own NVRTC-specialised module
    sample = [next(k for k, v in enumerate(variants) if v[0] == net) for net in range(len(bases))]
    sample = sample[:per_variant_sample]
    comp_s, comp_trans, run_ms, run_trans = 0.0, 0, 0.0, 0
    for k in sample:
        net, params, n = variants[k]
        m = mb.Model(*bases[net])
        for name, val in params.items():
            m.set_variable(name, val)
        t = time.perf_counter()
        mod = ctx.compile(m)
        res = mod.run(mode="fast", sample_count=n)
        comp_s += time.perf_counter() - t
        comp_trans += res.transitions
        runner = mod.runner(mode="fast", sample_count=n)
        runner.launch()
        runner.result()
        runner.launch()
        r2 = runner.result()
        run_ms += r2.timing[0]
        run_trans += r2.transitions
    precompiled = run_trans / (run_ms / 1e3)
    with_compile = comp_trans / comp_s
    return {
        "workload": f"c5: {EXTRA_WORKLOADS['c5']}", "value": value, "unit": "transitions/s",
        "ms_per_step": sum(ms) / steps, "steps": steps, "variants": len(variants),
        "trajectories": sum(v[2] for v in variants), "transitions_per_step": trans // steps,
        "launch": {"block": info["block"], "blocks_per_sm": info["blocks_per_sm"],
                   "graph_nodes": info["graph_nodes"], "tuned": info["tuning"]},
        "per_variant_precompiled": {"value": precompiled, "variants": len(sample),
                                    "note": "one variant of each base network, each with its own NVRTC-specialised "
                                            "fast kernel compiled beforehand; device time of its launch"},
        "per_variant_with_compile": {"value": with_compile, "variants": len(sample),
                                     "compile_and_run_s": comp_s,
                                     "note": "the same variants, NVRTC compilation + fast run per variant, wall "
                                             "time (the reference's workflow: $variables are compiled in)"},
        "ratio_vs_precompiled": value / precompiled, "ratio_vs_with_compile": value / with_compile,
        "e2e": {"value": (trans / steps) / e2e_s, "unit": "transitions/s", "wall_ms_per_run": 1e3 * e2e_s,
                "h2d_bytes_per_step": 8, "d2h_bytes_per_step": d2h,
                "api": "Batch.run (graph replay with the new seed) + Batch.result of every variant "
                       "(window probabilities, final counts, fixed points)"},
        "gpu_launches": 1 + len(variants),
    }


def run_batched(args) -> None:
    import maboss.gpu_b200 as mb

    mb.build()
    ctx = mb.Context(0)
    clocks = ClockSampler(0)
    clocks.start()
    rec = batched_record(ctx, args.warmup, args.steps)
    clk = clocks.stop()
    line = _timed_line(args, rec["value"], rec["ms_per_step"],
                       {"workload": rec["workload"], "mode": "fast (batched kernel)", "variants": rec["variants"],
                        "trajectories": rec["trajectories"], "transitions_per_step": rec["transitions_per_step"],
                        "l2": "not flushed (the per-variant statistics are a few MB; the inputs are tables)",
                        "launch": rec["launch"]},
                       {k: rec[k] for k in ("per_variant_precompiled", "per_variant_with_compile",
                                            "ratio_vs_precompiled", "ratio_vs_with_compile", "e2e")}
                       | {"gpu_launches": args.steps * rec["gpu_launches"], "clocks": clk})
    print(json.dumps(line), flush=True)


def gradient_record(ctx, warmup: int, steps: int, n: int = 1_000_000) -> dict:
    """C4: the score-function gradient (VJP) of the 50-node network's window probabilities with
    respect to its 40 rate parameters, 1e6 trajectories, against the forward simulation: the
    NVRTC-specialised fast kernel of the same model (the plain forward pass) and the batched kernel
    that the gradient kernel extends (same runtime tables, without the score)."""
    import maboss.gpu_b200 as mb
    from maboss.gpu_b200 import synth

    model = mb.Model(*synth.c4())
    names = sorted(model.variables)
    theta = {k: model.variable(k) for k in names}
    b = mb.Batch(ctx)
    v = b.add_variant(b.add_model(model), n, theta)
    for _ in range(max(1, warmup)):
        b.run(0)
    dims = b.result(v).dims
    cot = np.zeros((dims.windows, dims.bins))
    cot[:, [s for s in range(dims.bins) if s & 1]] = 1.0
    # a gradient batch kept across calls (the way repeated gradients are taken: device buffers, launch
    # shape and graphs reused)
    kept = mb.Batch(ctx)
    kv = kept.add_variant(kept.add_model(model), n, theta, grad_params=names)
    mod = ctx.compile(model)
    runner = mod.runner(mode="fast", sample_count=n)
    for _ in range(max(1, warmup)):
        runner.launch()
        runner.result()
        kept.run_gradient(0, {kv: cot})
    fwd_ms, nvrtc_ms, grad_ms, call_ms, trans = [], [], [], [], 0
    for step in range(steps):
        fwd_ms.append(b.run(step))
        runner.launch()
        nvrtc_ms.append(runner.result().timing[0])
        t = time.perf_counter()
        grad_ms.append(kept.run_gradient(step, {kv: cot}))
        kept.gradient(kv)
        trans += kept.result(kv).transitions
        call_ms.append(1e3 * (time.perf_counter() - t))
    g_ms, f_ms, nv_ms = float(np.mean(grad_ms)), float(np.mean(fwd_ms)), float(np.mean(nvrtc_ms))
    return {"workload": f"c4grad: {EXTRA_WORKLOADS['c4grad']}", "parameters": len(names), "trajectories": n,
            "value": trans / (sum(grad_ms) / 1e3), "unit": "transitions/s",
            "gradient_ms": g_ms, "forward_nvrtc_fast_ms": nv_ms, "forward_batched_ms": f_ms,
            "gradient_over_nvrtc_forward": g_ms / nv_ms, "gradient_over_batched_forward": g_ms / f_ms,
            "gradient_call_ms": float(np.mean(call_ms)), "steps": steps,
            "note": "device times (CUDA events) of the launches; gradient_call_ms is the host-to-host time of "
                    "run_gradient + gradient on a batch kept across calls"}


def run_gradient(args) -> None:
    import maboss.gpu_b200 as mb

    mb.build()
    ctx = mb.Context(0)
    clocks = ClockSampler(0)
    clocks.start()
    rec = gradient_record(ctx, args.warmup, args.steps, args.samples or 1_000_000)
    clk = clocks.stop()
    line = _timed_line(args, rec["value"], rec["gradient_ms"],
                       {"workload": rec["workload"], "parameters": rec["parameters"], "trajectories": rec["trajectories"]},
                       {k: rec[k] for k in ("forward_nvrtc_fast_ms", "forward_batched_ms", "gradient_ms",
                                            "gradient_over_nvrtc_forward", "gradient_over_batched_forward",
                                            "gradient_call_ms")}
                       | {"gpu_launches": args.steps, "clocks": clk})
    print(json.dumps(line), flush=True)


def run_ours(args) -> None:
    import torch
    import torch.distributed as dist

    import maboss.gpu_b200 as mb

    rank, world, local = dist_env()
    torch.cuda.set_device(local)
    if world > 1:
        dist.init_process_group("nccl", timeout=__import__("datetime").timedelta(seconds=600))
    mb.build()
    bnd, cfg, desc = make_workload(args.workload, args.samples)
    model = mb.Model(bnd, cfg)
    n = int(args.samples or model.constant("sample_count"))
    ctx = mb.Context(local)
    t0 = time.perf_counter()
    mod = ctx.compile(model)
    compile_s = time.perf_counter() - t0
    tuned = None
    if args.block == 0 and args.mode in ("fast", "exact"):
        # launch shape from the autotuner (probe runs on a slice of this workload, outside the timing)
        tuned = mod.autotune(mode=args.mode, sample_count=n, first_traj=rank * n)
        launch_kw = dict(block=tuned["block"], blocks_per_sm=tuned["blocks_per_sm"])
    else:
        launch_kw = dict(block=args.block or 256, blocks_per_sm=args.blocks_per_sm)
    runner = mod.runner(mode=args.mode, sample_count=n, first_traj=rank * n, **launch_kw)
    stream = torch.cuda.ExternalStream(ctx.stream, device=local)
    flush = torch.empty(256 << 20, dtype=torch.uint8, device=local)  # 256 MiB > 126 MB L2

    def barrier():
        torch.cuda.synchronize()
        if world > 1:
            dist.barrier()

    # warm-up
    for _ in range(args.warmup):
        runner.launch()
        r = runner.result()
    trans_per_step = r.transitions

    # timed region: K steps, each preceded by an L2 flush outside its events
    starts = [torch.cuda.Event(enable_timing=True) for _ in range(args.steps)]
    ends = [torch.cuda.Event(enable_timing=True) for _ in range(args.steps)]
    kernel_ms, trans = [], 0
    clocks = ClockSampler(local)
    clocks.start()
    barrier()
    for i in range(args.steps):
        with torch.cuda.stream(stream):
            flush.fill_(i & 0xff)
            starts[i].record(stream)
        runner.launch()
        ends[i].record(stream)
        r = runner.result()  # waits; copies statistics back (outside the events)
        trans += r.transitions
        kernel_ms.append(r.timing[0])
    barrier()
    clk = clocks.stop()
    step_ms = [s.elapsed_time(e) for s, e in zip(starts, ends)]
    total_s = sum(step_ms) / 1e3
    local_time = torch.tensor([total_s], dtype=torch.float64, device=local)
    total_trans = torch.tensor([trans], dtype=torch.float64, device=local)
    if world > 1:
        dist.all_reduce(local_time, op=dist.ReduceOp.MAX)
        dist.all_reduce(total_trans, op=dist.ReduceOp.SUM)
    value = float(total_trans.item()) / float(local_time.item())

    # end to end through the public API: mb_run with host-side results (H2D of the initial
    # probabilities, D2H of every statistic), each step synchronised on both sides; with several
    # ranks each step is one job of n * world trajectories whose statistics are summed over the
    # ranks (maboss.gpu_b200.distributed.sharded_run: one all-reduce + one all-gather)
    from maboss.gpu_b200.distributed import sharded_run

    def api_run():
        if world > 1:
            return sharded_run(mod, mode=args.mode, sample_count=n * world, **launch_kw)
        return mod.run(mode=args.mode, sample_count=n, **launch_kw)

    # W untimed calls first, as for the device-timed steps: the module keeps the runner (device
    # buffers) of its last run for the next call with the same configuration
    for _ in range(args.warmup):
        api_run()
    barrier()
    t = time.perf_counter()
    e2e_trans = 0
    for _ in range(args.steps):
        res = api_run()
        # with several ranks res is the job's merged result: its total counted once over the ranks
        e2e_trans += res.transitions / world if world > 1 else res.transitions
        # host copy of the result: the entries when the windows are sparse (more than 20 non-internal
        # nodes, or a large histogram's non-zero cells), else the dense window probabilities
        probs = res.sparse()["probs"] if res.windows_sparse else res.window_probs
    barrier()
    e2e_s = time.perf_counter() - t
    e2e_time = torch.tensor([e2e_s], dtype=torch.float64, device=local)
    e2e_total = torch.tensor([e2e_trans], dtype=torch.float64, device=local)
    if world > 1:
        dist.all_reduce(e2e_time, op=dist.ReduceOp.MAX)
        dist.all_reduce(e2e_total, op=dist.ReduceOp.SUM)
    d = res.dims
    h2d = model.num_nodes * 4
    if res.is_sparse:  # compacted bins: 16-byte key + 8-byte value each
        sp = res.sparse()
        d2h = (len(sp["raw"]) + len(sp["final_counts"])) * 24 + d.windows * 8 + len(res.fixed) * (4 * d.state_words + 4) + 64
    elif res.windows_sparse:  # a large histogram's non-zero cells: 8-byte cell index + 8-byte value each
        sp = res.sparse()
        d2h = len(sp["raw"]) * 16 + d.windows * 8 + d.bins * 4 + len(res.fixed) * (4 * d.state_words + 4) + 64
    else:
        d2h = d.windows * d.bins * 8 + d.windows * 8 + d.bins * 4 + len(res.fixed) * (4 * d.state_words + 4) + 64

    if world > 1:
        dist.destroy_process_group()
    if rank != 0:
        return

    # roofline of the simulation kernel (algorithmic bytes per transition x transitions per launch)
    peaks = load_peaks()
    words = d.state_words
    ni_words = len({i // 32 for i in model.noninternal_nodes}) or 1
    bpt = bytes_per_transition(words, ni_words)
    avg_kernel_s = float(np.mean(kernel_ms)) / 1e3
    achieved = trans_per_step * bpt / avg_kernel_s / 1e9
    peak = peaks.get("hbm_gbs")
    traffic = None
    prof = os.path.join(ROOT, "profiles", "traffic.json")
    if os.path.exists(prof):
        with open(prof) as f:
            traffic = json.load(f).get(f"{args.workload}:{args.mode}")
    issue = None
    if os.path.exists(prof):
        with open(prof) as f:
            issue = json.load(f).get("issue", {}).get(f"{args.workload}:{args.mode}")
    # CPU baselines on all host cores, each on a sample sized to about 10 s: the measured mode's own
    # algorithm (fast: the incremental integer-rate process, oracle mode 2; exact: the reference's
    # dense per-step algorithm, mode 0) feeds cpu_baseline; the other is reported beside it
    cores = os.cpu_count() or 1
    cpu = cpu_other = None
    same_mode = 2 if args.mode == "fast" else 0
    other_mode = 0 if same_mode == 2 else 2
    if not args.no_cpu:
        cpu = cpu_baseline_sized(bnd, cfg, same_mode, cores, args.cpu_seconds, n)
        cpu_other = cpu_baseline_sized(bnd, cfg, other_mode, cores, args.cpu_seconds / 2, n)
    # the batched sweep and the gradient, measured after the timed region (their own device timing)
    extras = {}
    if not args.no_extras and world == 1:
        extras["batched"] = batched_record(ctx, 3, 5)
        extras["gradient"] = gradient_record(ctx, 3, 5)
    line = {
        "metric": "Gillespie transitions/s",
        "value": value,
        "unit": "transitions/s",
        "n_gpus": world,
        "steps": args.steps,
        "warmup": args.warmup,
        "ms_per_step": 1e3 * float(local_time.item()) / args.steps,
        "higher_is_better": True,
        "scaling": "weak",
        "vs_baseline": None,
        "dtype": "f32",
        "data": "synthetic",
        "config": {"workload": f"{args.workload}: {desc}", "mode": args.mode, "trajectories_per_gpu": n,
                   "nodes": model.num_nodes, "state_words": words, "transitions_per_step": trans_per_step,
                   "l2": "flushed between steps (256 MiB write outside the step events)",
                   "nvrtc_compile_s": round(compile_s, 2), "block": launch_kw["block"],
                   "blocks_per_sm": launch_kw["blocks_per_sm"] or "occupancy calculator",
                   "launch_shape": "autotuned (mb_autotune)" if tuned else "given"},
        "e2e": {"value": float(e2e_total.item()) / float(e2e_time.item()), "unit": "transitions/s",
                "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": d2h,
                "api": "mb_run (Module.run) after W untimed calls (the module keeps its last run's device "
                       "buffers): H2D of the inputs, accumulator clears, kernel, D2H of all statistics"
                       + ("; statistics summed over the ranks (distributed.sharded_run)" if world > 1 else "")},
        "gpu_launches": runner.kernel_launches * args.steps,
        "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                     "frac": (achieved / peak) if peak else None, "traffic": traffic,
                     "bytes_per_transition": bpt, "kernel_ms_avg": float(np.mean(kernel_ms)),
                     "peak_source": "MEASURED_PEAKS.json hbm_gbs (measured)" if peak else "absent"},
        "cpu_baseline": None if cpu is None else {
            "value": cpu["value"], "unit": "transitions/s", "cores": cores, "kind": "port",
            "sample": f"{cpu['trajectories']} trajectories of the same workload, {ORACLE_MODES[same_mode]}, "
                      f"{cores} OpenMP threads ({cpu['seconds']:.1f} s; the CPU oracle)"},
        "cpu_baseline_other_algorithm": None if cpu_other is None else {
            "value": cpu_other["value"], "unit": "transitions/s", "cores": cores, "kind": "port",
            "sample": f"{cpu_other['trajectories']} trajectories, {ORACLE_MODES[other_mode]} "
                      f"({cpu_other['seconds']:.1f} s)"},
        "clocks": clk,
    }
    if issue:
        line["roofline"]["issue"] = issue
    line.update(extras)
    print(json.dumps(line), flush=True)


def main() -> None:
    p = argparse.ArgumentParser()
    p.add_argument("--gpus", type=int, default=1)
    p.add_argument("--steps", type=int, default=5)
    p.add_argument("--warmup", type=int, default=3)
    p.add_argument("--impl", choices=["ours", "reference"], default="ours")
    p.add_argument("--workload", choices=sorted(WORKLOADS) + sorted(EXTRA_WORKLOADS), default="c3")
    p.add_argument("--mode", choices=["fast", "exact", "epoch", "epoch_dense"], default="fast")
    p.add_argument("--samples", type=int, default=None, help="trajectories per GPU (default: the workload's)")
    p.add_argument("--block", type=int, default=0,
                   help="threads per block (0: chosen by the engine's autotuner, fused modes; 256 otherwise)")
    p.add_argument("--blocks-per-sm", type=int, default=0, help="resident blocks per SM (0: occupancy calculator)")
    p.add_argument("--cpu-seconds", type=float, default=10.0, help="CPU baseline sample size, in seconds of work")
    p.add_argument("--no-cpu", action="store_true", help="skip the CPU baselines")
    p.add_argument("--no-extras", action="store_true", help="skip the batched and gradient records")
    p.add_argument("--ref-samples", type=int, default=0,
                   help="trajectories of the reference arm's runs (0: the workload's, capped below the "
                        "reference's int overflow)")
    args = p.parse_args()
    if args.impl == "reference":
        run_reference(args)
    elif args.workload == "c5":
        run_batched(args)
    elif args.workload == "c4grad":
        run_gradient(args)
    else:
        run_ours(args)


if __name__ == "__main__":
    main()
