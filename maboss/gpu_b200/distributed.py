"""Runs over several processes (one per GPU) with torch.distributed.

Trajectories are independent, and trajectory i of a job always uses random stream i, so a job of n
trajectories splits into contiguous shards [first, first + count) run on different GPUs with no
communication. The one exchange of the path is at the end: the sum of the per-shard statistics
(window sums, entropy sums, final-state counts, transitions: one all-reduce of int64) and the union
of the fixed points (an all-gather of the short fixed-point lists). Every shard runs with the job's
fixed-point scale (mb_run_config.stats_trajectories = n), so the merged result equals a single run
of all n trajectories bit for bit.

With the NCCL backend each process must have selected its GPU (torch.cuda.set_device) before the
exchange; with gloo the exchange goes through host memory.
"""
from __future__ import annotations

import numpy as np

from .engine import Module, Result


def shard(total: int, rank: int, world: int) -> tuple[int, int]:
    """(first trajectory, count) of `rank`'s contiguous block; the first total % world ranks get one more."""
    if world <= 0 or not 0 <= rank < world or total < 0:
        raise ValueError("need 0 <= rank < world and total >= 0")
    base, extra = divmod(total, world)
    first = rank * base + min(rank, extra)
    return first, base + (1 if rank < extra else 0)


def _layout(result: Result) -> tuple:
    d, info, raw = result.dims, result.info(), result.raw()
    return (d.windows, d.bins, d.nodes, info["discrete"], info["time_tick"], info["max_time"],
            tuple(info["noninternal"]), raw["occ_exp"], raw["ent_exp"])


def allreduce_result(result: Result, group=None) -> Result:
    """The statistics of the whole job on every rank, from each rank's shard `result`."""
    import torch
    import torch.distributed as dist

    if not dist.is_available() or not dist.is_initialized():
        return result
    world = dist.get_world_size(group)
    info, raw = result.info(), result.raw()
    discrete = info["discrete"]
    win = (raw["cnt"] if discrete else raw["occ"]).reshape(-1).astype(np.int64)
    T = result.dims.windows
    final = result.final_counts.astype(np.int64)
    dense = np.concatenate([win, raw["h"].astype(np.int64), final,
                            np.array([result.transitions, info["n_trajectories"]], np.int64)])
    device = "cpu"
    if dist.get_backend(group) == "nccl":
        device = torch.device("cuda", torch.cuda.current_device())
    t = torch.from_numpy(dense).to(device)
    dist.all_reduce(t, op=dist.ReduceOp.SUM, group=group)
    dense = t.cpu().numpy()

    mine = (_layout(result), [(st.tolist(), int(c)) for st, c in result.fixed])
    gathered = [None] * world
    dist.all_gather_object(gathered, mine, group=group)
    if any(g[0] != mine[0] for g in gathered):
        raise ValueError("allreduce_result: the shards differ in model, windows or fixed-point scale "
                         "(run every shard with stats_trajectories = the job's trajectory count)")
    states, counts = [], []
    for _, fixed in gathered:
        for st, c in fixed:
            states.append(st)
            counts.append(c)

    n_win = win.size
    o = 0
    win_sum = dense[o:o + n_win]; o += n_win
    h_sum = dense[o:o + T]; o += T
    fin_sum = dense[o:o + final.size]; o += final.size
    transitions, n_total = int(dense[o]), int(dense[o + 1])
    return Result.from_raw(
        n_nodes=result.dims.nodes, n_windows=T, discrete=discrete, time_tick=info["time_tick"],
        max_time=info["max_time"], noninternal=info["noninternal"], n_trajectories=n_total,
        occ_exp=raw["occ_exp"], ent_exp=raw["ent_exp"],
        occ=None if discrete else win_sum, cnt=win_sum if discrete else None, h=h_sum, final=fin_sum,
        fixed_states=np.array(states, np.uint32).reshape(len(counts), -1) if counts else None,
        fixed_counts=np.array(counts, np.uint32) if counts else None, transitions=transitions)


def sharded_run(module: Module, mode: str = "exact", sample_count: int | None = None, group=None,
                **kw) -> Result:
    """simulation_runner::run_simulation of one job split over the ranks of `group`: this rank runs its
    block of trajectories, then the statistics are summed over the ranks (every rank returns the
    job's result)."""
    import torch.distributed as dist

    total = int(sample_count if sample_count is not None else module.model.constant("sample_count"))
    if not dist.is_available() or not dist.is_initialized():
        return module.run(mode=mode, sample_count=total, **kw)
    rank, world = dist.get_rank(group), dist.get_world_size(group)
    first, count = shard(total, rank, world)
    base = kw.pop("first_traj", 0)
    res = module.run(mode=mode, sample_count=count, first_traj=base + first, stats_trajectories=total, **kw)
    return allreduce_result(res, group)
