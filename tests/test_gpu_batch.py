"""Batched variants and score-function gradients (kernels/batched.cuh through the C ABI)."""
import math

import numpy as np
import pytest

import maboss.gpu_b200 as mb
from conftest import force_node, model_text
from maboss.gpu_b200 import synth
from oracle.oracle import OracleModel

pytestmark = pytest.mark.gpu


def _same(a: "mb.Result", b: "mb.Result"):
    ra, rb = a.raw(), b.raw()
    for k in ("occ", "cnt", "h"):
        assert np.array_equal(ra[k], rb[k]), k
    assert np.array_equal(a.final_counts, b.final_counts)
    assert a.transitions == b.transitions
    assert [(s.tolist(), c) for s, c in a.fixed] == [(s.tolist(), c) for s, c in b.fixed]


@pytest.mark.parametrize("name,n", [("metastasis", 2_000), ("sizek", 1_000), ("cellcycle", 3_000)])
def test_batch_variant_without_overrides_equals_fast_mode(gpu, name, n):
    model = mb.Model(*model_text(name))
    b = mb.Batch(gpu)
    net = b.add_model(model)
    v = b.add_variant(net, n)
    b.run(int(model.constant("seed_pseudorandom")))
    _same(b.result(v), gpu.compile(model).run(mode="fast", sample_count=n))


def test_batch_of_networks_and_variants_matches_oracle(gpu):
    """Two networks of different sizes, rate variants and stream offsets in one launch; each
    variant equals the oracle's integer-rate fast mode with the same exact rates."""
    meta = model_text("metastasis")
    base = synth.c5_base(2)
    b = mb.Batch(gpu)
    nets = [b.add_model(mb.Model(*meta)), b.add_model(mb.Model(*base))]
    rng = np.random.default_rng(7)
    cases = []
    for net, (bnd, cfg) in zip(nets, [meta, base]):
        o = OracleModel(bnd, cfg)
        names = [k for k in mb.Model(bnd, cfg).variables][:6]
        for first in (0, 5_000):
            params = {k: float(np.float32(mb.Model(bnd, cfg).variable(k) * math.exp(rng.normal(0, 0.3))))
                      for k in names}
            n = int(rng.integers(300, 900))
            cases.append((b.add_variant(net, n, params, first_traj=first), bnd, cfg, params, n, first))
    seed = 11
    b.run(seed)
    for v, bnd, cfg, params, n, first in cases:
        o = OracleModel(bnd, cfg)
        o.set_variables(params)
        r = b.result(v)
        raw = r.raw()
        ref = o.run(n=n, mode=1, seed=seed, first=first, occ_exp=raw["occ_exp"], ent_exp=raw["ent_exp"])
        assert r.transitions == ref["transitions"]
        assert np.array_equal(r.final_counts, ref["final"])
        assert len(r.fixed) == len(ref["fixed_counts"])
        assert np.all(np.abs(r.window_probs - ref["probs"]) <= 1e-5 + 1e-4 * ref["probs"])


TWO_STATE = """
node A { logic = !A; rate_up = @logic ? $u : 0; rate_down = @logic ? 0 : $d; }
"""


def _two_state_window_mean(u, d, p0, a, b):
    lam = u + d
    pi = u / lam
    return pi + (p0 - pi) * (math.exp(-lam * a) - math.exp(-lam * b)) / (lam * (b - a))


def test_gradient_of_two_state_chain_matches_analytic(gpu):
    """A single node switching on at rate u and off at rate d: window probabilities and their
    derivatives have closed forms; the score-function estimate must agree within its own spread
    (4 independent seeds)."""
    u, d, p0, tick, tmax = 1.3, 0.7, 0.25, 0.5, 3.0
    cfg = f"$u = {u}; $d = {d}; A.istate = {p0}; max_time = {tmax}; time_tick = {tick};"
    model = mb.Model(TWO_STATE, cfg)
    T = int(round(tmax / tick))
    cot = np.zeros((T, 2))
    cot[:, 1] = 1.0  # L = sum over windows of P(A on)
    est = []
    for seed in range(4):
        g, fwd = mb.gradient(gpu, model, {"$u": u, "$d": d}, cot, 400_000, seed)
        est.append(g)
        # forward probabilities of the same run
        p = fwd.window_probs[:, 1]
        exact = np.array([_two_state_window_mean(u, d, p0, w * tick, (w + 1) * tick) for w in range(T)])
        assert np.all(np.abs(p - exact) < 5 * np.sqrt(exact * (1 - exact) / 400_000) + 1e-6)
    est = np.array(est)
    h = 1e-6

    def L(uu, dd):
        return sum(_two_state_window_mean(uu, dd, p0, w * tick, (w + 1) * tick) for w in range(T))

    exact = np.array([(L(u + h, d) - L(u - h, d)) / (2 * h), (L(u, d + h) - L(u, d - h)) / (2 * h)])
    mean, sem = est.mean(axis=0), est.std(axis=0, ddof=1) / 2.0
    assert np.all(np.abs(mean - exact) < 4 * sem + 0.01 * np.abs(exact)), (mean, exact, sem)


@pytest.mark.parametrize("discrete", [False, True], ids=["continuous", "discrete"])
def test_gradient_matches_common_random_number_finite_differences(gpu, discrete):
    """C4-style network: score-function gradients of sum_w P_w(output node 0 on) against central
    finite differences with common random numbers (variants with the same random streams in one
    batched launch). Both are Monte-Carlo estimates: over 4 seeds, the means must agree within 4
    combined standard errors plus 2% of |FD|. The step is 1% of each parameter: with 1e3-fold
    smaller steps the finite-difference noise at this sample size exceeds most of the gradients.
    Discrete time: one transition per tick, chosen with probability rate / a0."""
    bnd, cfg = synth.c4()
    if discrete:
        cfg += "\ndiscrete_time = 1;\n"
    model = mb.Model(bnd, cfg)
    names = [f"$u_{i}" for i in range(4)] + [f"$d_{i}" for i in range(4)]
    theta = {k: model.variable(k) for k in names}
    n = 500_000
    dims = gpu.compile(model).run(mode="fast", sample_count=10).dims
    T, S = dims.windows, dims.bins
    cot = np.zeros((T, S))
    cot[:, [s for s in range(S) if s & 1]] = 1.0  # output node 0 on
    sf, fd = [], []
    for seed in range(4):
        g, _ = mb.gradient(gpu, model, theta, cot, n, seed=seed)
        sf.append(g)
        b = mb.Batch(gpu)
        net = b.add_model(model)
        pairs = []
        for k in names:
            hk = 1e-2 * theta[k]
            pairs.append((b.add_variant(net, n, dict(theta, **{k: theta[k] + hk})),
                          b.add_variant(net, n, dict(theta, **{k: theta[k] - hk})), 2 * hk))
        b.run(seed)
        fd.append([((b.result(p).window_probs - b.result(m).window_probs) * cot).sum() / span
                   for p, m, span in pairs])
    sf, fd = np.array(sf), np.array(fd)
    se = np.sqrt(sf.var(axis=0, ddof=1) / 4 + fd.var(axis=0, ddof=1) / 4)
    diff = np.abs(sf.mean(axis=0) - fd.mean(axis=0))
    assert np.all(diff <= 4 * se + 0.02 * np.abs(fd.mean(axis=0))), (sf.mean(axis=0), fd.mean(axis=0), se)


def _fd_and_sf(gpu, model, names, cot, n, rel_step, seeds):
    theta = {k: model.variable(k) for k in names}
    sf, fd = [], []
    for seed in seeds:
        g, _ = mb.gradient(gpu, model, theta, cot, n, seed=seed)
        sf.append(g)
        b = mb.Batch(gpu)
        net = b.add_model(model)
        pairs = []
        for k in names:
            hk = rel_step * theta[k]
            pairs.append((b.add_variant(net, n, dict(theta, **{k: theta[k] + hk})),
                          b.add_variant(net, n, dict(theta, **{k: theta[k] - hk})), 2 * hk))
        b.run(seed)
        fd.append([((b.result(p).window_probs - b.result(m).window_probs) * cot).sum() / span
                   for p, m, span in pairs])
    return np.array(sf), np.array(fd)


def test_gradient_at_the_gradient_configuration(gpu):
    """The gradient configuration itself: the 50-node network, all 40 rate parameters, 1e6
    trajectories, central finite differences with common random numbers at h = 1e-3 relative
    (variants sharing random streams in one batched launch), 4 seeds. Criterion per parameter:
    |SF - FD| <= 4 combined standard errors + 2 % of |FD| (both are Monte-Carlo estimates). The
    measured standard errors at h = 1e-3 and h = 1e-2 and the largest relative deviation among the
    parameters whose finite difference is resolved (standard error below 2 % of its value) are
    printed."""
    model = mb.Model(*synth.c4())
    names = sorted(model.variables)
    assert len(names) == 40
    n = 1_000_000
    dims = gpu.compile(model).run(mode="fast", sample_count=10).dims
    cot = np.zeros((dims.windows, dims.bins))
    cot[:, [s for s in range(dims.bins) if s & 1]] = 1.0
    seeds = range(4)
    sf, fd = _fd_and_sf(gpu, model, names, cot, n, 1e-3, seeds)
    m_sf, m_fd = sf.mean(axis=0), fd.mean(axis=0)
    se_sf, se_fd = sf.std(axis=0, ddof=1) / 2.0, fd.std(axis=0, ddof=1) / 2.0
    se = np.sqrt(se_sf ** 2 + se_fd ** 2)
    diff = np.abs(m_sf - m_fd)
    _, fd2 = _fd_and_sf(gpu, model, names, cot, n, 1e-2, seeds)
    se_fd2 = fd2.std(axis=0, ddof=1) / 2.0
    resolved = se_fd < 0.02 * np.abs(m_fd)
    rel = diff / np.maximum(np.abs(m_fd), 1e-30)
    # the same estimate against the ten times wider step, whose finite differences resolve more
    m_fd2 = fd2.mean(axis=0)
    resolved2 = se_fd2 < 0.02 * np.abs(m_fd2)
    rel2 = np.abs(m_sf - m_fd2) / np.maximum(np.abs(m_fd2), 1e-30)
    print(f"\ngradient configuration: median |SF| {np.median(np.abs(m_sf)):.4g}, median SE(SF) "
          f"{np.median(se_sf):.3g}, median SE(FD) at h=1e-3 {np.median(se_fd):.3g}, at h=1e-2 "
          f"{np.median(se_fd2):.3g}; resolved at h=1e-3: {int(resolved.sum())} of 40; max relative deviation "
          f"among them {rel[resolved].max() if resolved.any() else float('nan'):.4f}; resolved at h=1e-2: "
          f"{int(resolved2.sum())} of 40, max relative deviation among them "
          f"{rel2[resolved2].max() if resolved2.any() else float('nan'):.4f}; max deviation in "
          f"combined standard errors {np.max(diff[se > 0] / se[se > 0]):.2f}")
    assert np.all(diff <= 4 * se + 0.02 * np.abs(m_fd)), (m_sf, m_fd, se)


@pytest.mark.parametrize("discrete", [False, True], ids=["continuous", "discrete"])
def test_gradient_equals_oracle_on_the_same_trajectories(gpu, discrete):
    """The kernel's gradient (incremental d a0 / d theta, slices summed by parts, fp32 scores)
    against the oracle's direct restatement (d a0 / d theta recomputed from every unstable node at
    every step, each slice integrated on its own, fp64) over the same fast-mode trajectories: equal
    up to rounding, far inside the estimator's own spread at this sample size."""
    bnd, cfg = synth.c4()
    if discrete:
        cfg += "\ndiscrete_time = 1;\n"
    model = mb.Model(bnd, cfg)
    names = [f"$u_{i}" for i in range(0, 20, 3)] + [f"$d_{i}" for i in range(1, 20, 4)]
    theta = {k: model.variable(k) for k in names}
    n, seed = 3_000, 11
    o = OracleModel(bnd, cfg)
    o.set_variables(theta)
    T, S = o.windows, 1 << o.k
    rng = np.random.default_rng(5)
    cot = rng.normal(size=(T, S))
    deriv = [[] for _ in range(2 * o.nodes)]
    for p, k in enumerate(names):
        node = int(k[3:])
        deriv[2 * node + (0 if k[1] == "u" else 1)].append((p, 1.0))
    ref = o.gradient(n, cot, deriv, len(names), seed=seed)
    g, fwd = mb.gradient(gpu, model, theta, cot, n, seed)
    assert np.array_equal(fwd.final_counts, o.run(n, mode=1, seed=seed)["final"])
    tol = 1e-3 * np.abs(ref) + 1e-4 * np.abs(ref).max()
    assert np.all(np.abs(g - ref) <= tol), (g, ref)


def _c4_gradient_case():
    bnd, cfg = synth.c4()
    model = mb.Model(bnd, cfg)
    names = [f"$u_{i}" for i in range(4)] + [f"$d_{i}" for i in range(4)]
    theta = {k: model.variable(k) for k in names}
    return model, names, theta


def test_forward_and_gradient_runs_share_one_batch(gpu):
    """One batch runs forward, then with cotangents, then forward again: the statistics of all three
    runs are identical (the two kinds of run share the variant's buffers, each keeps its own
    descriptors), and the gradient equals mb_gradient's on the same trajectories."""
    model, names, theta = _c4_gradient_case()
    n, seed = 20_000, 3
    b = mb.Batch(gpu)
    v = b.add_variant(b.add_model(model), n, theta, grad_params=names)
    b.run(seed)
    r1 = b.result(v)
    cot = np.random.default_rng(1).normal(size=r1.window_probs.shape)
    b.run_gradient(seed, {v: cot})
    g1, r2 = b.gradient(v), b.result(v)
    b.run(seed)
    r3 = b.result(v)
    _same(r1, r2)
    _same(r1, r3)
    b.run_gradient(seed, {v: cot})
    g2 = b.gradient(v)
    ref, _ = mb.gradient(gpu, model, theta, cot, n, seed)
    assert len(g1) == len(names)
    assert np.allclose(g1, ref, rtol=1e-9, atol=1e-12) and np.allclose(g2, ref, rtol=1e-9, atol=1e-12)


def test_set_variables_equals_a_fresh_batch(gpu):
    """New variable values on a prepared batch (tables re-uploaded in place, graphs replayed) give
    the statistics and the gradient of a batch built with those values."""
    model, names, theta = _c4_gradient_case()
    n, seed = 20_000, 5
    b = mb.Batch(gpu)
    v = b.add_variant(b.add_model(model), n, theta, grad_params=names)
    b.run(seed)
    cot = np.random.default_rng(2).normal(size=b.result(v).window_probs.shape)
    b.run_gradient(seed, {v: cot})
    theta2 = {k: float(np.float32(x * (1.3 if i % 2 else 0.8))) for i, (k, x) in enumerate(theta.items())}
    b.set_variables(v, theta2)
    b.run(seed)
    fresh = mb.Batch(gpu)
    fv = fresh.add_variant(fresh.add_model(model), n, theta2)
    fresh.run(seed)
    _same(b.result(v), fresh.result(fv))
    b.run_gradient(seed, {v: cot})
    ref, _ = mb.gradient(gpu, model, theta2, cot, n, seed)
    assert np.allclose(b.gradient(v), ref, rtol=1e-9, atol=1e-12)


def test_autograd_function_reuses_its_batch(gpu):
    import torch

    from maboss.gpu_b200.autograd import window_probabilities

    model, names, theta = _c4_gradient_case()
    n = 20_000
    for scale in (1.0, 1.2, 0.9):
        t = torch.tensor([theta[k] * scale for k in names], dtype=torch.float64, requires_grad=True)
        probs = window_probabilities(t, gpu, model, names, n, seed=7)
        w = torch.linspace(0.0, 1.0, probs.shape[1], dtype=torch.float64)
        (probs * w).sum().backward()
        params = {k: float(x) for k, x in zip(names, t.detach().tolist())}
        cot = np.tile(w.numpy(), (probs.shape[0], 1))
        g, fwd = mb.gradient(gpu, model, params, cot, n, 7)
        assert np.array_equal(probs.detach().numpy(), fwd.window_probs)
        assert np.allclose(t.grad.numpy(), g, rtol=1e-9, atol=1e-12)


def test_autograd_function(gpu):
    import torch

    from maboss.gpu_b200.autograd import window_probabilities

    u, d = 1.3, 0.7
    model = mb.Model(TWO_STATE, f"$u = {u}; $d = {d}; A.istate = 0.25; max_time = 2; time_tick = 0.5;")
    theta = torch.tensor([u, d], dtype=torch.float64, requires_grad=True)
    probs = window_probabilities(theta, gpu, model, ["$u", "$d"], 100_000, seed=5)
    loss = probs[:, 1].sum()
    loss.backward()
    cot = np.zeros(tuple(probs.shape))
    cot[:, 1] = 1.0
    g, fwd = mb.gradient(gpu, model, {"$u": u, "$d": d}, cot, 100_000, 5)
    assert np.allclose(probs.detach().numpy(), fwd.window_probs)
    assert np.allclose(theta.grad.numpy(), g)


def _sweep_batch(gpu, use_graph, autotune):
    b = mb.Batch(gpu)
    b.set_options(use_graph=use_graph, autotune=autotune)
    bases, variants = synth.c5_sweep(n_variants=12, seed=3)
    models = [mb.Model(*x) for x in bases]
    nets = [b.add_model(m) for m in models]
    for net, params, n in variants:
        b.add_variant(nets[net], min(n, 4_000), params)
    return b, len(variants)


def test_graph_replay_equals_direct_runs(gpu):
    """Runs replayed from the captured CUDA graph (seed updated in the kernel node) give the same
    statistics as runs enqueued directly, seed by seed; the autotuner picks one of the shapes it timed."""
    g, nv = _sweep_batch(gpu, use_graph=True, autotune=True)
    d, _ = _sweep_batch(gpu, use_graph=False, autotune=False)
    for seed in (5, 6, 5):
        g.run(seed)
        d.run(seed)
        for v in range(nv):
            _same(g.result(v), d.result(v))
    info = g.info
    assert info["graph_nodes"] > nv  # clears, kernel, extractions and copies of every variant
    assert len(info["tuning"]) >= 2
    assert (info["block"], info["blocks_per_sm"]) in {(t["block"], t["blocks_per_sm"]) for t in info["tuning"]}
    assert d.info["graph_nodes"] == 0


def test_changing_the_batch_rebuilds_the_plan(gpu):
    """add_variant after a run drops the captured graph: the new variant is simulated and the old
    ones are unchanged."""
    b, nv = _sweep_batch(gpu, use_graph=True, autotune=False)
    b.run(1)
    before = [b.result(v) for v in range(nv)]
    model = mb.Model(*model_text("metastasis"))
    extra = b.add_variant(b.add_model(model), 1_000)
    b.run(1)
    for v in range(nv):
        _same(b.result(v), before[v])
    _same(b.result(extra), gpu.compile(model).run(mode="fast", sample_count=1_000, seed=1))


def test_specialised_batch_kernels_equal_the_generic_ones(gpu):
    """A batch of one network runs the batched kernels compiled for that network (NVRTC,
    compile-time sizes and tables); the ahead-of-time kernels take any networks. Same algorithm,
    same random streams, same integer sums: the window sums, final states and fixed points of
    both are identical and the gradients equal up to the order of their f64 atomic sums, for two
    variants of the 50-node network and after set_variables."""
    model = mb.Model(*synth.c4())
    names = sorted(model.variables)
    theta = {k: model.variable(k) for k in names}
    other = {k: v * 1.1 for k, v in theta.items()}
    runs = []
    for spec in (True, False):
        b = mb.Batch(gpu)
        b.set_specialize(spec)
        net = b.add_model(model)
        v0 = b.add_variant(net, 20_000, theta, grad_params=names)
        v1 = b.add_variant(net, 15_000, other, grad_params=names)
        dims = None
        b.run(5)
        out = [b.result(v).raw() for v in (v0, v1)]
        dims = b.result(v0).dims
        cot = np.zeros((dims.windows, dims.bins))
        cot[:, 1::2] = 1.0
        b.run_gradient(7, {v0: cot, v1: cot})
        grads = [b.gradient(v) for v in (v0, v1)]
        b.set_variables(v1, theta)
        b.run(5)
        after = b.result(v1).raw()
        fins = [b.result(v).final_counts for v in (v0, v1)]
        runs.append((out, grads, after, fins))
    (oa, ga, aa, fa), (ob, gb, ab, fb) = runs
    for x, y in zip(oa, ob):
        assert np.array_equal(x["occ"], y["occ"]) and np.array_equal(x["h"], y["h"])
    # the gradient's per-parameter sums are f64 atomic adds, whose order changes from launch to launch
    for x, y in zip(ga, gb):
        assert np.allclose(x, y, rtol=1e-12, atol=1e-12 * np.abs(x).max())
    assert np.array_equal(aa["occ"], ab["occ"])
    for x, y in zip(fa, fb):
        assert np.array_equal(x, y)


@pytest.mark.parametrize("name,node,on", [("sizek", "PI3K", True), ("sizek", "PI3K", False),
                                          ("cellcycle", "CycE", True)])
def test_mutant_equals_the_edited_model(gpu, name, node, on):
    """Mutant analysis: a node forced on or off (mb_batch_add_mutant: initial state 1 / 0, both
    rates 0) equals, bit for bit, the fast mode of the model whose text forces that node; mutants of
    a sweep run in one launch with the wild type."""
    bnd, cfg = model_text(name)
    n = 20_000
    model = mb.Model(bnd, cfg)
    b = mb.Batch(gpu)
    b.set_specialize(False)
    net = b.add_model(model)
    wt = b.add_variant(net, n)
    mv = b.add_variant(net, n, mutants={node: on})
    b.run(11)
    edited = mb.Model(*force_node(bnd, cfg, node, on))
    ref = gpu.compile(edited).run(mode="fast", sample_count=n, seed=11)
    got = b.result(mv)
    assert got.transitions == ref.transitions
    ra, rb = got.raw(), ref.raw()
    assert np.array_equal(ra["occ"], rb["occ"]) and np.array_equal(ra["cnt"], rb["cnt"])
    assert np.array_equal(got.final_counts, ref.final_counts)
    assert [(tuple(s), c) for s, c in got.fixed] == [(tuple(s), c) for s, c in ref.fixed]
    # the forced node holds its value in every window
    idx = model.node_names.index(node)
    if idx in model.noninternal_nodes:
        k = model.noninternal_nodes.index(idx)
        probs = got.window_probs
        bins_with = np.array([(s >> k) & 1 for s in range(probs.shape[1])], bool)
        mass = probs[:, bins_with].sum(axis=1) if on else probs[:, ~bins_with].sum(axis=1)
        assert np.allclose(mass[probs.sum(axis=1) > 0], 1.0, atol=1e-6)
    rw = b.result(wt).raw()
    assert not (np.array_equal(rw["occ"], ra["occ"]) and np.array_equal(rw["cnt"], ra["cnt"]))


def test_mutant_sweep_runs_every_single_node_mutant(gpu):
    model = mb.Model(*model_text("cellcycle"))
    res = mb.mutant_sweep(gpu, model, 2_000, nodes=["CycD", "Rb"])
    assert set(res) == {("wt",), ("CycD", True), ("CycD", False), ("Rb", True), ("Rb", False)}
    assert all(r.transitions > 0 for r in res.values())
