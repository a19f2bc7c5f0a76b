"""Sharded jobs: the shard split, the merge of shard statistics (mb_result_create / mb_result_merge)
and the exchange over torch.distributed (maboss.gpu_b200.distributed) with world_size 2 gloo ranks
on the CPU, each computing its shard with the oracle. The merged statistics must equal those of one
run over all trajectories bit for bit (integer sums at the job's fixed-point scale)."""
import os
import socket
import subprocess
import sys
import time

import numpy as np
import pytest

import maboss.gpu_b200 as mb
from conftest import ROOT, model_text
from maboss.gpu_b200.distributed import shard
from oracle.oracle import OracleModel, entropy_exponent, occupancy_exponent


def _free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _oracle_result(o, n, first, total):
    e_occ, e_h = occupancy_exponent(total, o.tick, o.discrete), entropy_exponent(total, o.tick, o.discrete)
    r = o.run(n=n, first=first, occ_exp=e_occ, ent_exp=e_h)
    return r, mb.Result.from_raw(
        n_nodes=o.nodes, n_windows=o.windows, discrete=o.discrete, time_tick=o.tick, max_time=o.max_time,
        noninternal=o.noninternal, n_trajectories=n, occ_exp=e_occ, ent_exp=e_h, occ=r["occ"], cnt=r["cnt"],
        h=r["h"], final=r["final"], fixed_states=r["fixed_states"], fixed_counts=r["fixed_counts"],
        transitions=r["transitions"])


@pytest.mark.parametrize("total,world", [(10, 3), (7, 8), (1_000_000, 8), (0, 2), (5, 1)])
def test_shards_cover_the_job_once(total, world):
    blocks = [shard(total, r, world) for r in range(world)]
    assert sum(c for _, c in blocks) == total
    pos = 0
    for first, count in blocks:
        assert first == pos
        pos += count
    assert max(c for _, c in blocks) - min(c for _, c in blocks) <= 1


def _assert_same(a: mb.Result, b: mb.Result):
    ra, rb = a.raw(), b.raw()
    for k in ("occ", "cnt", "h", "occ_exp", "ent_exp"):
        assert np.array_equal(ra[k], rb[k]), k
    assert np.array_equal(a.final_counts, b.final_counts)
    assert [(s.tolist(), c) for s, c in a.fixed] == [(s.tolist(), c) for s, c in b.fixed]
    assert a.transitions == b.transitions and a.info() == b.info()


@pytest.mark.parametrize("name,n", [("sizek", 600), ("cellcycle", 1_500)])
def test_merge_of_shards_equals_one_run(tmp_path, name, n):
    bnd, cfg = model_text(name)
    o = OracleModel(bnd, cfg)
    _, full = _oracle_result(o, n, 0, n)
    parts = [_oracle_result(o, c, f, n)[1] for f, c in (shard(n, r, 3) for r in range(3))]
    merged = mb.merge_results(parts)
    _assert_same(merged, full)
    model = mb.Model(bnd, cfg)
    merged.write_csv(model, str(tmp_path / "m"))
    full.write_csv(model, str(tmp_path / "f"))
    for suffix in ("_probtraj.csv", "_fp.csv"):
        assert (tmp_path / ("m" + suffix)).read_text() == (tmp_path / ("f" + suffix)).read_text()
    assert merged.visualize(model) == full.visualize(model)


def test_merge_rejects_different_scales():
    bnd, cfg = model_text("sizek")
    o = OracleModel(bnd, cfg)
    a = _oracle_result(o, 100, 0, 100)[1]
    b = _oracle_result(o, 100, 100, 1_000_000)[1]  # another fixed-point scale
    with pytest.raises(mb.EngineError, match="scale"):
        mb.merge_results([a, b])


def _torchrun(args, timeout):
    cmd = [sys.executable, "-m", "torch.distributed.run", "--nnodes=1", "--nproc-per-node", "2",
           "--master-addr", "127.0.0.1", "--master-port", str(_free_port()),
           os.path.join(ROOT, "tests", "distributed_worker.py")] + args
    env = dict(os.environ, OMP_NUM_THREADS="2", CUDA_VISIBLE_DEVICES="")
    return subprocess.run(cmd, capture_output=True, text=True, timeout=timeout, env=env)


@pytest.mark.parametrize("name,n", [("sizek", 500), ("cellcycle", 1_200)])
def test_gloo_two_ranks_allreduce_equals_one_run(tmp_path, name, n):
    out = str(tmp_path / "job")
    p = _torchrun(["--model-name", name, "--trajectories", str(n), "--out-prefix", out], timeout=300)
    assert p.returncode == 0, p.stderr[-3000:]
    got = np.load(out + ".npz")
    bnd, cfg = model_text(name)
    o = OracleModel(bnd, cfg)
    r, full = _oracle_result(o, n, 0, n)
    assert np.array_equal(got["occ"], full.raw()["occ"]) and np.array_equal(got["cnt"], full.raw()["cnt"])
    assert np.array_equal(got["h"], r["h"]) and np.array_equal(got["final"], r["final"])
    assert np.array_equal(got["fixed_states"].reshape(-1), np.asarray(r["fixed_states"]).reshape(-1))
    assert np.array_equal(got["fixed_counts"], r["fixed_counts"])
    assert int(got["transitions"]) == r["transitions"] and int(got["n"]) == n
    model = mb.Model(bnd, cfg)
    full.write_csv(model, str(tmp_path / "full"))
    for suffix in ("_probtraj.csv", "_fp.csv"):
        assert open(out + suffix).read() == (tmp_path / ("full" + suffix)).read_text()


def test_rank_that_leaves_before_the_exchange_ends_the_job(tmp_path):
    """Rank 1 exits between steps; rank 0's collective ends with an error (process-group timeout or
    closed connection) and the job exits non-zero instead of waiting forever."""
    t0 = time.time()
    p = _torchrun(["--model-name", "sizek", "--trajectories", "200", "--out-prefix", str(tmp_path / "x"),
                   "--leave-rank", "1"], timeout=240)
    assert p.returncode != 0
    assert time.time() - t0 < 200
    assert not os.path.exists(str(tmp_path / "x.npz"))


@pytest.mark.gpu
@pytest.mark.parametrize("name,mode", [("sizek", "exact"), ("sizek", "fast"), ("cellcycle", "exact"),
                                       ("metastasis", "epoch")])
def test_gpu_shards_merge_to_one_run(gpu, name, mode):
    """Three shards run with the job's fixed-point scale (stats_trajectories) and merged equal one run
    of all trajectories bit for bit: the multi-GPU result without the collective."""
    model = mb.Model(*model_text(name))
    mod = gpu.compile(model)
    n = 3_000
    full = mod.run(mode=mode, sample_count=n)
    parts = [mod.run(mode=mode, sample_count=c, first_traj=f, stats_trajectories=n)
             for f, c in (shard(n, r, 3) for r in range(3))]
    _assert_same(mb.merge_results(parts), full)
