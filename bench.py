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
    "c5": "batched sweep: 256 rate-perturbed variants (lognormal sigma 0.3) of 8 networks of 20-144 nodes, "
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


def cpu_baseline(bnd: str, cfg: str, sample: int, mode: int, threads: int) -> dict:
    """The oracle (C++/OpenMP restatement of the reference algorithm) on a bounded sample."""
    from oracle.oracle import OracleModel, build
    build()
    o = OracleModel(bnd, cfg)
    t = time.perf_counter()
    r = o.run(n=sample, mode=mode, threads=threads)
    dt = time.perf_counter() - t
    return {"value": r["transitions"] / dt, "transitions": r["transitions"], "seconds": dt, "trajectories": sample}


def run_reference(args) -> None:
    rank, world, _ = dist_env()
    if rank != 0:
        return
    bnd, cfg, desc = make_workload(args.workload, args.samples)
    cores = os.cpu_count() or 1
    sample = args.cpu_sample
    for _ in range(args.warmup):
        cpu_baseline(bnd, cfg, max(1, sample // 10), 0, cores)
    vals, trans, secs = [], 0, 0.0
    for _ in range(args.steps):
        b = cpu_baseline(bnd, cfg, sample, 0, cores)
        vals.append(b["value"])
        trans += b["transitions"]
        secs += b["seconds"]
    value = trans / secs
    line = {
        "impl": "reference", "metric": "Gillespie transitions/s", "value": value, "unit": "transitions/s",
        "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1e3 * secs / args.steps,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
        "config": {"workload": f"{args.workload}: {desc}", "sample_trajectories_per_step": sample},
        "cpu_baseline": {"value": value, "unit": "transitions/s", "cores": cores, "kind": "port",
                         "sample": f"{sample} trajectories of the workload per step (CPU oracle, exact mode, "
                                   f"{cores} OpenMP threads); the reference ships no CPU implementation"},
        "e2e": {"value": value, "unit": "transitions/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


def _timed_line(args, value, ms_per_step, config, extra) -> dict:
    line = {"metric": "Gillespie transitions/s", "value": value, "unit": "transitions/s", "n_gpus": 1,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms_per_step, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic", "config": config}
    line.update(extra)
    return line


def run_batched(args) -> None:
    """C5: one persistent launch over 256 variants, against running the variants one by one."""
    import maboss.gpu_b200 as mb
    from maboss.gpu_b200 import synth

    mb.build()
    ctx = mb.Context(0)
    bases, variants = synth.c5_sweep()
    models = [mb.Model(*b) for b in bases]
    batch = mb.Batch(ctx)
    nets = [batch.add_model(m) for m in models]
    for net, params, n in variants:
        batch.add_variant(nets[net], n, params)
    for _ in range(args.warmup):
        batch.run(0)  # the first run tunes the launch shape and captures the CUDA graph
    clocks = ClockSampler(0)
    clocks.start()
    ms, trans = [], 0
    for step in range(args.steps):
        ms.append(batch.run(step))
        trans += sum(batch.result(v).transitions for v in range(len(variants)))
    clk = clocks.stop()
    value = trans / (sum(ms) / 1e3)
    info = batch.info

    # end to end: whole runs through the public API (graph launch: clears, kernel, extraction, copies
    # to pinned memory; then every variant's result), wall clock, with and without the graph
    def wall(b, reps=3):
        t0 = time.perf_counter()
        for i in range(reps):
            b.run(100 + i)
            for v in range(len(variants)):
                b.result(v).final_counts
        return (time.perf_counter() - t0) / reps

    e2e_s = wall(batch)
    nograph = mb.Batch(ctx)
    nograph.set_options(use_graph=False, autotune=False)
    ng_nets = [nograph.add_model(m) for m in models]
    for net, params, n in variants:
        nograph.add_variant(ng_nets[net], n, params)
    nograph.run(0)
    e2e_nograph_s = wall(nograph)
    # the same variants one launch each (first 32 variants), and with one compilation per variant
    # as the reference needs ($variables are baked into its generated code)
    single_ms, single_trans = 0.0, 0
    for net, params, n in variants[:32]:
        b = mb.Batch(ctx)
        b.set_options(use_graph=False, autotune=False)
        k = b.add_model(models[net])
        v = b.add_variant(k, n, params)
        b.run(0)
        single_ms += b.run(0)
        single_trans += b.result(v).transitions
    t0 = time.perf_counter()
    comp_trans = 0
    for net, params, n in variants[:4]:
        m = mb.Model(*bases[net])
        for k2, val in params.items():
            m.set_variable(k2, val)
        comp_trans += ctx.compile(m).run(mode="fast", sample_count=n).transitions
    comp_s = time.perf_counter() - t0
    line = _timed_line(args, value, sum(ms) / args.steps,
                       {"workload": f"c5: {EXTRA_WORKLOADS['c5']}", "mode": "fast (batched kernel)",
                        "variants": len(variants), "trajectories": sum(v[2] for v in variants),
                        "transitions_per_step": trans // args.steps,
                        "l2": "not flushed (the per-variant statistics are a few MB; the inputs are tables)",
                        "launch": {"block": info["block"], "blocks_per_sm": info["blocks_per_sm"],
                                   "graph_nodes": info["graph_nodes"], "tuned": info["tuning"]}},
                       {"per_variant_launch": {"value": single_trans / (single_ms / 1e3), "variants": 32,
                                               "note": "the first 32 variants, one batched launch each"},
                        "per_variant_compile_and_run": {"value": comp_trans / comp_s, "variants": 4,
                                                        "note": "NVRTC compile + fused fast run per variant, wall time"},
                        "e2e": {"value": (trans / args.steps) / e2e_s, "unit": "transitions/s",
                                "wall_ms_per_run": 1e3 * e2e_s, "wall_ms_per_run_without_graph": 1e3 * e2e_nograph_s,
                                "h2d_bytes_per_step": 0, "d2h_bytes_per_step": None,
                                "api": "Batch.run + Batch.result of every variant (graph replay)"},
                        "gpu_launches": args.steps * (1 + len(variants)), "clocks": clk})
    print(json.dumps(line), flush=True)


def run_gradient(args) -> None:
    """C4: cost of the score-function gradient against the forward simulation."""
    import maboss.gpu_b200 as mb
    from maboss.gpu_b200 import synth

    mb.build()
    ctx = mb.Context(0)
    model = mb.Model(*synth.c4())
    names = sorted(model.variables)
    theta = {k: model.variable(k) for k in names}
    n = args.samples or 1_000_000
    b = mb.Batch(ctx)
    v = b.add_variant(b.add_model(model), n, theta)
    dims = None
    for _ in range(args.warmup):
        b.run(0)
    dims = b.result(v).dims
    cot = np.zeros((dims.windows, dims.bins))
    cot[:, [s for s in range(dims.bins) if s & 1]] = 1.0
    for _ in range(args.warmup):
        mb.gradient(ctx, model, theta, cot, n, 0)
    fwd_ms, grad_ms, call_ms, trans = [], [], [], 0
    clocks = ClockSampler(0)
    clocks.start()
    for step in range(args.steps):
        fwd_ms.append(b.run(step))
        t = time.perf_counter()
        g, res = mb.gradient(ctx, model, theta, cot, n, step)
        call_ms.append(1e3 * (time.perf_counter() - t))
        grad_ms.append(res.timing[0])
        trans += res.transitions
    clk = clocks.stop()
    line = _timed_line(args, trans / (sum(grad_ms) / 1e3), sum(grad_ms) / args.steps,
                       {"workload": f"c4grad: {EXTRA_WORKLOADS['c4grad']}", "parameters": len(names),
                        "trajectories": n},
                       {"forward_ms": float(np.mean(fwd_ms)), "gradient_ms": float(np.mean(grad_ms)),
                        "gradient_call_ms": float(np.mean(call_ms)),  # wall time of mb_gradient, host to host
                        "gradient_over_forward": float(np.mean(grad_ms) / np.mean(fwd_ms)),
                        "gpu_launches": args.steps, "clocks": clk})
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
        probs = res.sparse()["probs"] if res.is_sparse else res.window_probs  # host copy of the result
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
    cores = os.cpu_count() or 1
    cpu = cpu_baseline(bnd, cfg, args.cpu_sample, 0, cores) if not args.no_cpu else None
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
            "sample": f"{args.cpu_sample} trajectories of the same workload, exact mode, {cores} OpenMP threads "
                      f"({cpu['seconds']:.1f} s)"},
        "clocks": clk,
    }
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
    p.add_argument("--cpu-sample", type=int, default=2000, help="trajectories of the CPU baseline sample")
    p.add_argument("--no-cpu", action="store_true", help="skip the CPU baseline")
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
