"""GPU parity tests: the CUDA engine against the CPU oracle, through the C ABI.

Exact mode draws the same XORWOW streams as the reference (curand_init(seed, trajectory, 0)) and
performs the reference's fp32 operations in the same order, so integer results (final-state and
discrete window counts, fixed points, number of transitions) must be identical to the oracle's.
Continuous-time waiting times use logf, whose device and host implementations may differ in the
last ulp; window occupancies are therefore compared with a tolerance of
    |p_gpu - p_oracle| <= 1e-5 + 1e-4 * p_oracle     (probabilities per window and bin)
and the per-window transition entropy (log2f on both sides) with a relative tolerance of 1e-4.
"""
import numpy as np
import pytest

import maboss.gpu_b200 as mb
from conftest import assert_statistically_equal, model_text
from maboss.gpu_b200 import synth
from oracle.oracle import OracleModel

pytestmark = pytest.mark.gpu

P_ABS, P_REL, H_REL = 1e-5, 1e-4, 1e-4


def _run_both(gpu, bnd, cfg, n, mode="exact", **kw):
    model = mb.Model(bnd, cfg)
    mod = gpu.compile(model)
    res = mod.run(mode=mode, sample_count=n, **kw)
    raw = res.raw()
    o = OracleModel(bnd, cfg)
    ref = o.run(n=n, mode=0 if mode in ("exact", "epoch") else 1, occ_exp=raw["occ_exp"], ent_exp=raw["ent_exp"],
                seed=kw.get("seed"))
    return model, res, raw, o, ref


def _assert_same(res, raw, ref, discrete):
    assert res.transitions == ref["transitions"]
    assert np.array_equal(res.final_counts, ref["final"])
    fx = res.fixed
    assert len(fx) == len(ref["fixed_counts"])
    for (st, c), st2, c2 in zip(fx, ref["fixed_states"], ref["fixed_counts"]):
        assert np.array_equal(st, st2) and c == c2
    assert res.fixed_overflow == 0
    if discrete:
        assert np.array_equal(raw["cnt"], ref["cnt"])
    else:
        p, q = res.window_probs, ref["probs"]
        assert np.all(np.abs(p - q) <= P_ABS + P_REL * q), np.abs(p - q).max()
    th, th2 = res.window_entropy, ref["th"]
    assert np.all(np.abs(th - th2) <= 1e-6 + H_REL * np.abs(th2)), np.abs(th - th2).max()


@pytest.mark.parametrize("name,n", [("cellcycle", 20_000), ("sizek", 2_000), ("metastasis", 1_000),
                                    ("Montagud2022_Prostate_Cancer", 3_000)])
def test_exact_mode_matches_oracle_on_reference_models(gpu, name, n):
    bnd, cfg = model_text(name)
    model, res, raw, o, ref = _run_both(gpu, bnd, cfg, n)
    _assert_same(res, raw, ref, o.discrete)


@pytest.mark.parametrize("gen,kw,n", [(synth.c1, {}, 20_000), (synth.c2, dict(noninternal=20), 300),
                                      (synth.c2, dict(noninternal=12, discrete=True), 2_000),
                                      (synth.c4, {}, 2_000), (synth.c3, {}, 300),
                                      (synth.c3, dict(n=3000, n_out=12), 24)])
def test_exact_mode_matches_oracle_on_synthetic_networks(gpu, gen, kw, n):
    bnd, cfg = gen(**kw)
    model, res, raw, o, ref = _run_both(gpu, bnd, cfg, n)
    _assert_same(res, raw, ref, o.discrete)


@pytest.mark.parametrize("name,n", [("cellcycle", 5_000), ("sizek", 1_000), ("metastasis", 1_000),
                                    ("Montagud2022_Prostate_Cancer", 2_000)])
def test_fast_mode_matches_oracle_fast_mode(gpu, name, n):
    """Fast mode (incremental kernel: Philox streams, integer rates) against the oracle's
    restatement of the same algorithm."""
    bnd, cfg = model_text(name)
    model, res, raw, o, ref = _run_both(gpu, bnd, cfg, n, mode="fast")
    _assert_same(res, raw, ref, o.discrete)


@pytest.mark.parametrize("gen,kw,n", [(synth.c1, {}, 20_000), (synth.c2, dict(noninternal=20), 500),
                                      (synth.c2, dict(noninternal=12, discrete=True), 2_000),
                                      (synth.c4, {}, 3_000), (synth.c3, {}, 300),
                                      (synth.c3, dict(n=3000, n_out=12), 24)])
def test_fast_mode_matches_oracle_on_synthetic_networks(gpu, gen, kw, n):
    bnd, cfg = gen(**kw)
    model, res, raw, o, ref = _run_both(gpu, bnd, cfg, n, mode="fast")
    _assert_same(res, raw, ref, o.discrete)


def test_fast_mode_dense_kernel_for_general_rates(gpu):
    """Rates that are not of the @logic form use the dense fast kernel (float rates)."""
    bnd = "".join(f"node Z{i} {{ logic = !Z{(i + 1) % 6}; rate_up = Z{(i + 2) % 6} ? 2 : 0.5; "
                  f"rate_down = @logic ? 0 : 1.5; }}\n" for i in range(6))
    cfg = "max_time = 4; time_tick = 0.25; sample_count = 3000;"
    model, res, raw, o, ref = _run_both(gpu, bnd, cfg, 3000, mode="fast")
    _assert_same(res, raw, ref, False)


def test_fast_mode_dense_kernel_for_a_wide_rate_span(gpu):
    """@logic-form rates spanning 1e-3 ... 1e3 are too wide for the integer rates: fast mode runs the
    dense kernel, equal to the oracle's restatement of it on the same Philox streams."""
    from test_codegen_host import wide_span_model

    bnd, cfg = wide_span_model()
    model, res, raw, o, ref = _run_both(gpu, bnd, cfg, 20_000, mode="fast")
    _assert_same(res, raw, ref, False)


def _assert_identical(a, b):
    ra, rb = a.raw(), b.raw()
    for k in ("occ", "cnt", "h"):
        assert np.array_equal(ra[k], rb[k]), k
    assert np.array_equal(a.final_counts, b.final_counts)
    assert a.transitions == b.transitions
    assert [(s.tolist(), c) for s, c in a.fixed] == [(s.tolist(), c) for s, c in b.fixed]


@pytest.mark.parametrize("name,n", [("cellcycle", 3_000), ("metastasis", 1_000), ("sizek", 1_500)])
def test_epoch_mode_is_identical_to_fused_exact(gpu, name, n):
    """Buffered epochs (SoA trajectory buffers + stats kernels; incremental unstable sets for
    @logic-form models, or every rate function per step in epoch_dense) and the fused kernel agree
    bit for bit."""
    model = mb.Model(*model_text(name))
    mod = gpu.compile(model)
    a = mod.run(mode="exact", sample_count=n)
    for mode in ("epoch", "epoch_dense"):
        _assert_identical(a, mod.run(mode=mode, sample_count=n))


@pytest.mark.parametrize("gen,kw,n", [(synth.c1, {}, 5_000), (synth.c2, dict(noninternal=12, discrete=True), 2_000),
                                      (synth.c3, {}, 200)])
def test_epoch_mode_is_identical_to_fused_exact_on_synthetic_networks(gpu, gen, kw, n):
    """The same identity on @logic-form networks, whose exact kernel keeps incremental unstable sets."""
    model = mb.Model(*gen(**kw))
    mod = gpu.compile(model)
    a = mod.run(mode="exact", sample_count=n)
    for mode in ("epoch", "epoch_dense"):
        _assert_identical(a, mod.run(mode=mode, sample_count=n))


@pytest.mark.parametrize("name,traj_len", [("metastasis", 2), ("metastasis", 7), ("Montagud2022_Prostate_Cancer", 5)])
def test_exact_mode_epoch_boundary_length(gpu, name, traj_len):
    """The epoch boundary (every traj_len-1 steps the reference re-evaluates the current state with a
    fresh draw) is part of the exact semantics; other lengths than the default must match too."""
    bnd, cfg = model_text(name)
    model = mb.Model(bnd, cfg)
    mod = gpu.compile(model)
    n = 1_000
    res = mod.run(mode="exact", sample_count=n, traj_len=traj_len)
    raw = res.raw()
    o = OracleModel(bnd, cfg)
    ref = o.run(n=n, mode=0, traj_len=traj_len, occ_exp=raw["occ_exp"], ent_exp=raw["ent_exp"])
    _assert_same(res, raw, ref, o.discrete)
    for mode in ("epoch", "epoch_dense"):
        _assert_identical(res, mod.run(mode=mode, sample_count=n, traj_len=traj_len))


def test_epoch_refill_beyond_batch_limit(gpu):
    """More trajectories than the batch: refilled slots start the streams of their trajectory ids, so
    the run equals the fused exact run bit for bit."""
    model = mb.Model(*model_text("metastasis"))
    mod = gpu.compile(model)
    exact = mod.run(mode="exact", sample_count=2_500)
    for mode in ("epoch", "epoch_dense"):
        r = mod.run(mode=mode, sample_count=2_500, batch_limit=1_000)
        assert r.final_counts.sum() == 2_500
        assert r.timing[2] >= 3
        p = r.window_probs
        assert np.allclose(p.sum(axis=1), 1.0, atol=1e-5)
        _assert_identical(exact, r)


def test_fast_mode_statistically_equivalent_to_exact(gpu):
    bnd, cfg = synth.c1()
    model = mb.Model(bnd, cfg)
    mod = gpu.compile(model)
    n = 100_000
    a, b = mod.run(mode="exact", sample_count=n), mod.run(mode="fast", sample_count=n)
    assert_statistically_equal(a.window_probs, n, b.window_probs, n)
    assert_statistically_equal(a.final_counts / n, n, b.final_counts / n, n)


def test_results_are_reproducible(gpu):
    model = mb.Model(*model_text("sizek"))
    mod = gpu.compile(model)
    a, b = mod.run(mode="fast", sample_count=4_000), mod.run(mode="fast", sample_count=4_000)
    assert np.array_equal(a.raw()["occ"], b.raw()["occ"])
    assert np.array_equal(a.final_counts, b.final_counts)


def test_low_level_kernel_entry_points(gpu):
    """init_random -> init_state -> simulate -> window/final/fixed stats through the C ABI on
    caller-owned device buffers reproduces the whole-run result (one epoch suffices here)."""
    import torch

    bnd, cfg = model_text("cellcycle")  # 25 discrete steps < one epoch of 100 slots
    model = mb.Model(bnd, cfg)
    mod = gpu.compile(model)
    n, L = 4_096, 100
    N, W = mod.state_size
    dev = torch.device("cuda", 0)
    rands = torch.empty(n * mb.rand_state_size(), dtype=torch.uint8, device=dev)
    last = torch.empty(W * n, dtype=torch.int32, device=dev)
    times = torch.empty(n, dtype=torch.float32, device=dev)
    istate = torch.tensor([model.node_info(i)[0] for i in range(N)], dtype=torch.float32, device=dev)
    ts = torch.empty(L * W * n, dtype=torch.int32, device=dev)
    tt = torch.empty(L * n, dtype=torch.float32, device=dev)
    th = torch.empty(L * n, dtype=torch.float32, device=dev)
    stat = torch.empty(n, dtype=torch.uint8, device=dev)
    trans = torch.zeros(1, dtype=torch.int64, device=dev)
    torch.cuda.synchronize()
    seed = int(model.constant("seed_pseudorandom"))
    mod.launch_initialize_random(n, seed, 0, rands.data_ptr())
    mod.launch_initialize_initial_state(n, n, istate.data_ptr(), last.data_ptr(), times.data_ptr(), rands.data_ptr())
    mod.launch_simulate(n, n, L, last.data_ptr(), times.data_ptr(), rands.data_ptr(), ts.data_ptr(), tt.data_ptr(),
                        th.data_ptr(), stat.data_ptr(), trans.data_ptr())
    st = mod.stats(model.constant("time_tick"), model.constant("max_time"), bool(model.constant("discrete_time")),
                   model.noninternal_nodes, n)
    st.final(n, n, last.data_ptr(), stat.data_ptr())
    st.fixed(n, n, last.data_ptr(), stat.data_ptr())
    st.window(n, n, L, ts.data_ptr(), tt.data_ptr(), th.data_ptr())
    r = st.finalize(n)
    assert int((stat == 0).sum()) == 0  # every trajectory finished in one epoch
    ref = mod.run(mode="exact", sample_count=n)
    assert np.array_equal(r.raw()["cnt"], ref.raw()["cnt"])
    assert np.array_equal(r.final_counts, ref.final_counts)
    assert int(trans.item()) == ref.transitions
    # slot 0 holds the start time, recorded times are tick multiples
    assert float(tt[:n].abs().max()) == 0.0
    assert float(tt[n:2 * n].min()) == pytest.approx(model.constant("time_tick"))


def test_edge_cases(gpu):
    bnd, cfg = model_text("metastasis")
    model = mb.Model(bnd, cfg)
    mod = gpu.compile(model)
    r0 = mod.run(sample_count=0)
    assert r0.final_counts.sum() == 0 and r0.transitions == 0
    r1 = mod.run(sample_count=1)
    assert r1.final_counts.sum() == 1
    # every node internal: a single bin (the first is_internal attribute of a node wins, so the
    # model's own declarations are removed first)
    import re
    stripped = re.sub(r"(?m)^\s*\w+\.is_internal\s*=.*$", "", cfg)
    allint = "\n".join(f"{n}.is_internal = 1;" for n in model.node_names)
    m2 = mb.Model(bnd, stripped + allint)
    r2 = gpu.compile(m2).run(sample_count=500)
    assert r2.dims.bins == 1 and r2.final_counts[0] == 500
    assert np.allclose(r2.window_probs[:, 0], 1.0, atol=1e-5)


def test_window_edge_ticks(gpu):
    """tick not dividing max_time, single window, and word-boundary network sizes (32/33 nodes)."""
    for n_nodes in (32, 33):
        names = [f"Y{i}" for i in range(n_nodes)]
        bnd = "".join(f"node {names[i]} {{ logic = !{names[(i + 1) % n_nodes]}; rate_up = @logic ? 1 : 0; "
                      f"rate_down = @logic ? 0 : 2; }}\n" for i in range(n_nodes))
        outs = {0, 31, n_nodes - 1}
        internal = "".join(f"{names[i]}.is_internal = 1;\n" for i in range(n_nodes) if i not in outs)
        for tail in ("max_time = 3; time_tick = 0.7;", "max_time = 0.5; time_tick = 1;"):
            cfg = internal + tail + " sample_count = 500;"
            model, res, raw, o, ref = _run_both(gpu, bnd, cfg, 500)
            _assert_same(res, raw, ref, False)


def test_runner_reports_its_kernel_launches(gpu):
    """Exact mode: the parallel XORWOW initialisation + the fused kernel; fast mode: the fused kernel;
    epoch mode: initialisation, then per epoch simulate, three statistics and three partition kernels."""
    mod = gpu.compile(mb.Model(*model_text("metastasis")))
    for mode, ok in (("exact", lambda k: k == 2), ("fast", lambda k: k == 1), ("epoch", lambda k: k >= 9)):
        r = mod.runner(mode=mode, sample_count=1_000)
        r.launch()
        r.result()
        assert ok(r.kernel_launches), (mode, r.kernel_launches)


def test_autotuner_picks_a_timed_shape_and_results_do_not_depend_on_it(gpu):
    """mb_autotune times shapes on a slice of the run; exact-mode results are the same whatever the
    launch shape (every trajectory has its own random stream)."""
    mod = gpu.compile(mb.Model(*synth.c2(noninternal=12)))
    t = mod.autotune(mode="exact", sample_count=20_000)
    shapes = {(c["block"], c["blocks_per_sm"]) for c in t["candidates"]}
    assert (t["block"], t["blocks_per_sm"]) in shapes and len(shapes) >= 2
    assert all(c["transitions_per_s"] > 0 for c in t["candidates"])
    a = mod.run(mode="exact", sample_count=3_000, block=t["block"], blocks_per_sm=t["blocks_per_sm"])
    b = mod.run(mode="exact", sample_count=3_000, block=64, blocks_per_sm=1)
    _assert_identical(a, b)


def test_large_histograms_come_back_as_their_non_zero_cells(gpu):
    """A dense histogram of >= 2^24 cells (the 100-node network with 20 outputs: 100 windows x 2^20
    states) is returned as its non-zero cells, selected in cell order on the device. The dense
    getters rebuild exactly the oracle's integers, the sparse getters give the same cells, the CSV
    writer and shard merges read them, and a small histogram stays dense."""
    bnd, cfg = synth.c2(noninternal=20)
    model, res, raw, o, ref = _run_both(gpu, bnd, cfg, 1_500)
    assert res.windows_sparse and not res.is_sparse
    _assert_same(res, raw, ref, o.discrete)
    # the same trajectories occupy the same cells (their sums agree to the slices' last ulp: device
    # and host logf, compared as probabilities above)
    nz = np.nonzero(ref["occ"].ravel())[0]
    assert np.array_equal(np.nonzero(raw["occ"].ravel())[0], nz)
    sp = res.sparse()
    assert len(sp["raw"]) == len(nz)
    cells = sp["windows"].astype(np.int64) * res.dims.bins + sp["states"][:, 0].astype(np.int64)
    assert np.array_equal(cells, nz) and np.array_equal(sp["raw"], raw["occ"].ravel()[nz])
    # discrete time: counts
    bnd_d, cfg_d = synth.c2(noninternal=20, discrete=True)
    _, res_d, raw_d, o_d, ref_d = _run_both(gpu, bnd_d, cfg_d, 1_000)
    assert res_d.windows_sparse and np.array_equal(raw_d["cnt"], ref_d["cnt"])
    # shards of one job merge to the whole run
    mod = gpu.compile(model)
    a = mod.run(mode="exact", sample_count=600, stats_trajectories=1_500)
    b = mod.run(mode="exact", sample_count=900, first_traj=600, stats_trajectories=1_500)
    m = mb.merge_results([a, b])
    assert m.windows_sparse and np.array_equal(m.raw()["occ"], raw["occ"])
    # a small histogram stays dense
    small = gpu.compile(mb.Model(*synth.c1())).run(mode="fast", sample_count=1_000)
    assert not small.windows_sparse
