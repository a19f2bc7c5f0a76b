"""Rank process for tests/test_distributed.py, started by torch.distributed.run with the gloo backend.

Each rank computes its shard of a job with the CPU oracle (test infrastructure), wraps it as an engine
Result (mb_result_create) and sums the shards with maboss.gpu_b200.distributed.allreduce_result; rank 0
writes the merged statistics to OUT.npz and the CSV files OUT_probtraj.csv / OUT_fp.csv. With
--leave-rank r, rank r exits before the exchange (a rank that leaves between steps): the others must
end with an error within the process group's timeout instead of waiting."""
import argparse
import datetime
import os
import sys

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)

import numpy as np  # noqa: E402
import torch.distributed as dist  # noqa: E402

import maboss.gpu_b200 as mb  # noqa: E402
from maboss.gpu_b200.distributed import allreduce_result, shard  # noqa: E402
from oracle.oracle import OracleModel, entropy_exponent, occupancy_exponent  # noqa: E402


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--model-name", required=True)
    ap.add_argument("--trajectories", type=int, required=True)
    ap.add_argument("--out-prefix", required=True)
    ap.add_argument("--leave-rank", type=int, default=-1)
    a = ap.parse_args()
    dist.init_process_group("gloo", timeout=datetime.timedelta(seconds=20))
    rank, world = dist.get_rank(), dist.get_world_size()
    models = os.path.join(ROOT, "tests", "golden", "models")
    name = a.model_name
    with open(os.path.join(models, name + ".bnd")) as f, open(os.path.join(models, name + ".cfg")) as g:
        bnd, cfg = f.read(), g.read()
    o = OracleModel(bnd, cfg)
    first, count = shard(a.trajectories, rank, world)
    n = a.trajectories
    e_occ, e_h = occupancy_exponent(n, o.tick, o.discrete), entropy_exponent(n, o.tick, o.discrete)
    r = o.run(n=count, first=first, occ_exp=e_occ, ent_exp=e_h, threads=2)
    if rank == a.leave_rank:
        sys.exit(3)
    part = mb.Result.from_raw(
        n_nodes=o.nodes, n_windows=o.windows, discrete=o.discrete, time_tick=o.tick, max_time=o.max_time,
        noninternal=o.noninternal, n_trajectories=count, occ_exp=e_occ, ent_exp=e_h, occ=r["occ"], cnt=r["cnt"],
        h=r["h"], final=r["final"], fixed_states=r["fixed_states"], fixed_counts=r["fixed_counts"],
        transitions=r["transitions"])
    total = allreduce_result(part)
    if rank == 0:
        raw = total.raw()
        states = np.array([s for s, _ in total.fixed], np.uint32).reshape(len(total.fixed), total.dims.state_words)
        counts = np.array([c for _, c in total.fixed], np.uint32)
        np.savez(a.out_prefix + ".npz", occ=raw["occ"], cnt=raw["cnt"], h=raw["h"], final=total.final_counts,
                 fixed_states=states, fixed_counts=counts, transitions=total.transitions,
                 n=total.info()["n_trajectories"])
        total.write_csv(mb.Model(bnd, cfg), a.out_prefix)
    dist.destroy_process_group()


if __name__ == "__main__":
    main()
