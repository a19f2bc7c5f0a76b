"""GPU parity against the reference's own CUDA build (oracle/_ref/ref_run: the reference sources
compiled by oracle/refbuild/Makefile, run on the same B200 with the same inputs).

Exact mode (MB_MODE_FUSED_EXACT) draws the reference's XORWOW streams (curand_init(seed, i, 0),
simulation.cu:31) and performs its fp32 operations in its order, including the 100-slot epoch
boundary (simulation.cu:143-147). So on the same model, seed and trajectory count:

* transitions (recorded slots s >= 1 with time > 0), final-state counts (final_states.cu:9-21),
  fixed points with their counts in std::map order (fixed_states.cu:84-125) and discrete window
  counts (window_average_small.cu:101-136) are identical integers;
* continuous window probabilities agree within |p - p_ref| <= 1e-6 + 2e-4 * p_ref and the
  per-window transition entropy within 2e-4 relative (+1e-6). The reference accumulates the
  window sums with fp32 atomicAdd in an order that changes from run to run
  (window_average_small.cu:79-84), so its own sums carry a rounding error of about
  sqrt(adds) * 2^-24 relative (up to ~1e5 adds per bin here: ~2e-5), while the engine sums in
  int64 fixed point.
"""
import os
import subprocess

import numpy as np
import pytest

import maboss.gpu_b200 as mb
from conftest import ROOT, model_files
from maboss.gpu_b200 import synth
from oracle import reference

pytestmark = [pytest.mark.gpu,
              pytest.mark.skipif(not reference.available(), reason="reference build absent (oracle/_ref)")]

P_ABS, P_REL, H_ABS, H_REL = 1e-6, 2e-4, 1e-6, 2e-4


def _compare(gpu, bnd_path, cfg_path, n, seed=None):
    ref = reference.run(bnd_path, cfg_path, samples=n, seed=seed)["result"]
    model = mb.Model.from_files(bnd_path, cfg_path)
    res = gpu.compile(model).run(mode="exact", sample_count=n, seed=seed)
    assert res.transitions == ref["transitions"] > 0
    assert np.array_equal(res.final_counts.astype(np.int64), ref["final"].astype(np.int64))
    fx = res.fixed
    assert len(fx) == len(ref["fixed_counts"])
    for (st, c), st2, c2 in zip(fx, ref["fixed_states"], ref["fixed_counts"]):
        assert np.array_equal(st, st2) and c == c2
    if ref["discrete"]:
        assert np.array_equal(res.raw()["cnt"].astype(np.int64), ref["window"].astype(np.int64))
    else:
        p, q = res.window_probs, ref["probs"]
        assert np.all(np.abs(p - q) <= P_ABS + P_REL * q), float(np.abs(p - q).max())
    th, th2 = res.window_entropy, ref["th"]
    assert np.all(np.abs(th - th2) <= H_ABS + H_REL * np.abs(th2)), float(np.abs(th - th2).max())
    return res, ref


@pytest.mark.parametrize("name,n", [("cellcycle", 20_000), ("sizek", 5_000), ("metastasis", 2_000),
                                    ("Montagud2022_Prostate_Cancer", 5_000)])
def test_exact_mode_equals_reference_build_on_example_models(gpu, name, n):
    _compare(gpu, *model_files(name), n)


@pytest.mark.parametrize("gen,kw,n", [(synth.c1, {}, 20_000), (synth.c2, dict(noninternal=20), 2_000),
                                      (synth.c2, dict(noninternal=20, discrete=True), 2_000),
                                      (synth.c3, {}, 1_000), (synth.c4, {}, 10_000)],
                         ids=["c1", "c2b", "c2b_discrete", "c3", "c4"])
def test_exact_mode_equals_reference_build_on_benchmark_networks(gpu, gen, kw, n, tmp_path):
    bnd, cfg = gen(**kw)
    (tmp_path / "m.bnd").write_text(bnd)
    (tmp_path / "m.cfg").write_text(cfg)
    _compare(gpu, str(tmp_path / "m.bnd"), str(tmp_path / "m.cfg"), n)


def test_exact_mode_equals_reference_build_with_other_seeds(gpu):
    for seed in (1, 12345):
        _compare(gpu, *model_files("sizek"), 3_000, seed=seed)


def test_csv_files_equal_reference_build(gpu, tmp_path):
    """The command-line front-end's out_probtraj.csv / out_fp.csv against the reference's writers
    (window_average_small.cpp:181-250, fixed_states.cu:154-187) on a discrete-time model: equal
    counts print equal text. The fixed-point file is equal byte for byte; in the trajectory file
    every column but TH is (times, entropies, states and probabilities come from the same integer
    counts), and TH, which the reference sums with fp32 atomics in a run-dependent order, agrees
    within 2e-4 relative."""
    bnd, cfg = model_files("cellcycle")
    (tmp_path / "m.cfg").write_text(open(cfg).read() + "\nsample_count = 30000;\n")
    reference.run(bnd, str(tmp_path / "m.cfg"), dump=False, csv_prefix=str(tmp_path / "ref"))
    cli = os.path.join(ROOT, "maboss", "gpu_b200", "MaBoSS.GPU")
    subprocess.run([cli, "--mode", "exact", "-o", str(tmp_path / "ours"), bnd, str(tmp_path / "m.cfg")],
                   check=True, capture_output=True)
    assert (tmp_path / "ref_fp.csv").read_bytes() == (tmp_path / "ours_fp.csv").read_bytes()
    a = (tmp_path / "ref_probtraj.csv").read_text().splitlines()
    b = (tmp_path / "ours_probtraj.csv").read_text().splitlines()
    assert len(a) == len(b) and a[0] == b[0]
    for la, lb in zip(a[1:], b[1:]):
        fa, fb = la.split("\t"), lb.split("\t")
        assert len(fa) == len(fb)
        assert fa[0] == fb[0] and fa[2:] == fb[2:], (la, lb)
        assert abs(float(fa[1]) - float(fb[1])) <= 2e-4 * abs(float(fa[1])) + 1e-6, (fa[1], fb[1])


@pytest.mark.parametrize("name", ["c1", "cellcycle"])
def test_refill_beyond_one_batch_equals_reference_build(gpu, name, tmp_path):
    """More trajectories than one batch (1.1e6 > 1e6): the reference refills the slots freed in an
    epoch with new trajectories that continue the random states the finished ones left there, in
    the order thrust::partition leaves them (simulation_runner.cu:126-153; quirk Q2). Epoch mode
    with refill_reuse_rng does the same: transitions, final states, fixed points and (cellcycle,
    discrete time) window counts identical to the reference build."""
    if name == "c1":
        bnd_path, cfg_path = str(tmp_path / "m.bnd"), str(tmp_path / "m.cfg")
        bnd, cfg = synth.c1()
        (tmp_path / "m.bnd").write_text(bnd)
        (tmp_path / "m.cfg").write_text(cfg)
    else:
        bnd_path, cfg_path = model_files(name)
    n = 1_100_000
    ref = reference.run(bnd_path, cfg_path, samples=n)["result"]
    model = mb.Model.from_files(bnd_path, cfg_path)
    mod = gpu.compile(model)
    res = mod.run(mode="epoch", sample_count=n, refill_reuse_rng=True)
    assert res.transitions == ref["transitions"]
    assert np.array_equal(res.final_counts.astype(np.int64), ref["final"].astype(np.int64))
    fx = res.fixed
    assert len(fx) == len(ref["fixed_counts"])
    for (st, c), st2, c2 in zip(fx, ref["fixed_states"], ref["fixed_counts"]):
        assert np.array_equal(st, st2) and c == c2
    if ref["discrete"]:
        assert np.array_equal(res.raw()["cnt"].astype(np.int64), ref["window"].astype(np.int64))
    else:
        # 1.1e6 trajectories put ~1e7 fp32 atomic adds into the reference's largest window bins:
        # its rounding error grows to a few 1e-4 relative there (the engine sums in int64)
        p, q = res.window_probs, ref["probs"]
        assert np.all(np.abs(p - q) <= P_ABS + 5 * P_REL * q), float(np.abs(p - q).max())
    # fresh streams for the refills (the default) give other trajectories
    other = mod.run(mode="epoch", sample_count=n)
    assert other.transitions != res.transitions or not np.array_equal(other.final_counts, res.final_counts)
