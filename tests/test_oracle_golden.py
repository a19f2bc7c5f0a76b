"""Pins the CPU oracle against the reference's golden outputs (test/*.res of the reference).

The .res files are stdout dumps of the reference's `visualize` for its four example models, made
by an older build (state names joined with "-"). Window probabilities are compared bin by bin at
4 sigma (pooled binomial standard error; continuous-time window averages have less variance than
binomial, so the bound is conservative). Final states are compared for the continuous-time
models; cellcycle's dump records the final state one transition after the end of the run (the
older build flipped before stopping), so for it the final-state distribution is pinned against
the dump's last window, which the current reference semantics make identical to the final state.
"""
import json
import os
import re

import numpy as np
import pytest

from conftest import GOLDEN, model_text, pooled_z
from oracle.oracle import OracleModel

# (model, trajectories simulated by the oracle): sized for a CPU test suite of a few minutes
CASES = [("cellcycle", 100_000), ("sizek", 20_000), ("metastasis", 1_000), ("Montagud2022_Prostate_Cancer", 20_000)]


def _names(bnd: str) -> list[str]:
    return re.findall(r"(?im)^\s*node\s+(\w+)", bnd)


def _key(s: str) -> frozenset:
    return frozenset() if s == "<nil>" else frozenset(s.split("-"))


def _golden(name: str) -> dict:
    with open(os.path.join(GOLDEN, f"{name}.res.json")) as f:
        return json.load(f)


def _bins(m: OracleModel, names: list[str]) -> list[frozenset]:
    return [frozenset(names[m.noninternal[k]] for k in range(m.k) if (b >> k) & 1) for b in range(1 << m.k)]


@pytest.mark.parametrize("name,n", CASES)
def test_oracle_windows_match_golden(name, n):
    bnd, cfg = model_text(name)
    m = OracleModel(bnd, cfg)
    g = _golden(name)
    assert len(g["windows"]) == m.windows
    r = m.run(n=n, threads=0)
    bins = _bins(m, _names(bnd))
    ng = m.sample_count
    for w, win in enumerate(g["windows"]):
        assert win["begin"] == pytest.approx(w * m.tick, rel=1e-5, abs=1e-6)
        gp = {_key(k): v for k, v in win["probs"].items()}
        unknown = set(gp) - set(bins)
        assert not unknown, f"golden states not representable: {unknown}"
        q = np.array([gp.get(b, 0.0) for b in bins])
        z = pooled_z(r["probs"][w], n, q, ng)
        assert z.max() < 4.0, (name, w, z.argmax(), r["probs"][w][z.argmax()], q[z.argmax()])
        # probabilities of a window sum to one (up to the float window bounds (w+1)*tick) unless
        # trajectories stopped contributing (discrete-time fixed points, window_average_small.cu:123)
        if not m.discrete:
            tol = 2 * float(np.spacing(np.float32(m.max_time))) / m.tick + 1e-9
            assert r["probs"][w].sum() == pytest.approx(1.0, abs=tol)


@pytest.mark.parametrize("name,n", CASES)
def test_oracle_final_states_match_golden(name, n):
    bnd, cfg = model_text(name)
    m = OracleModel(bnd, cfg)
    g = _golden(name)
    r = m.run(n=n, threads=0)
    bins = _bins(m, _names(bnd))
    p = r["final"].astype(np.float64) / n
    assert r["final"].sum() == n
    if m.discrete:
        ref = {_key(k): v for k, v in g["windows"][-1]["probs"].items()}
    else:
        ref = {_key(k): v for k, v in g["final"].items()}
    q = np.array([ref.get(b, 0.0) for b in bins])
    z = pooled_z(p, n, q, m.sample_count)
    assert z.max() < 4.0, (name, z.argmax(), p[z.argmax()], q[z.argmax()])


@pytest.mark.parametrize("name,n", [("metastasis", 1_000), ("sizek", 20_000)])
def test_oracle_fixed_points_match_golden(name, n):
    bnd, cfg = model_text(name)
    m = OracleModel(bnd, cfg)
    g = _golden(name)
    r = m.run(n=n, threads=0)
    names = _names(bnd)
    ours = {}
    for st, c in zip(r["fixed_states"], r["fixed_counts"]):
        key = frozenset(names[i] for i in range(m.nodes) if (int(st[i // 32]) >> (i % 32)) & 1)
        ours[key] = c / n
    gold = {_key(k): v for k, v in g["fixed"].items()}
    for key in set(ours) | set(gold):
        p, q = ours.get(key, 0.0), gold.get(key, 0.0)
        z = pooled_z(np.array([p]), n, np.array([q]), m.sample_count)[0]
        assert z < 4.0, (name, sorted(key), p, q)


def test_oracle_is_deterministic_and_thread_independent():
    bnd, cfg = model_text("metastasis")
    m = OracleModel(bnd, cfg)
    a = m.run(n=300, threads=1)
    b = m.run(n=300, threads=4)
    assert np.array_equal(a["occ"], b["occ"]) and np.array_equal(a["h"], b["h"])
    assert np.array_equal(a["final"], b["final"]) and a["transitions"] == b["transitions"]
    assert np.array_equal(a["fixed_states"], b["fixed_states"])


def test_oracle_sharding_is_additive():
    """Trajectories [0, n) equal [0, k) + [k, n): each trajectory owns its random stream."""
    bnd, cfg = model_text("sizek")
    m = OracleModel(bnd, cfg)
    e = 40  # shared fixed-point exponent
    full = m.run(n=200, occ_exp=e, ent_exp=e)
    a = m.run(n=120, occ_exp=e, ent_exp=e)
    b = m.run(n=80, first=120, occ_exp=e, ent_exp=e)
    assert np.array_equal(full["occ"], a["occ"] + b["occ"])
    assert np.array_equal(full["final"], a["final"] + b["final"])
    assert full["transitions"] == a["transitions"] + b["transitions"]


@pytest.mark.parametrize("name,n", CASES)
def test_oracle_transition_entropy_matches_golden(name, n):
    """Per-window transition entropy (TH, window_average_small.cpp:222-223: the window's summed
    h * slice over the trajectories, divided by their number and, in continuous time, by the tick)
    against the `transition_entropy` of each window of the golden dump.

    TH is a mean over trajectories of X = (1/tick) * integral of h over the window (continuous) or
    the h of the window's step (discrete), with 0 <= X <= log2(k) for k non-internal nodes (h is the
    entropy of the normalised non-internal rates). So Var(X) <= E[X^2] <= log2(k) * E[X], which
    bounds the standard error of each estimate without assuming a distribution; late windows where
    only a few trajectories still move are covered by the same bound. Each window within 4.5 of
    those combined standard errors (plus the golden's 6-significant-digit printing)."""
    bnd, cfg = model_text(name)
    m = OracleModel(bnd, cfg)
    g = _golden(name)
    th = m.run(n=n, threads=0)["th"]
    gold = np.array([win["transition_entropy"] for win in g["windows"]])
    assert gold.shape == th.shape
    h_max = np.log2(max(m.k, 2))
    mean = np.maximum(th, gold)
    se = np.sqrt(h_max * mean * (1.0 / n + 1.0 / m.sample_count))
    tol = 4.5 * se + 5e-6 * np.abs(gold) + 1e-7
    bad = np.nonzero(np.abs(th - gold) > tol)[0]
    assert bad.size == 0, (name, bad[:5], th[bad[:5]], gold[bad[:5]], se[bad[:5]])
    # and the whole run's mean transition entropy (sum over windows) within the summed bound
    assert abs(th.sum() - gold.sum()) <= 4.5 * np.sqrt(h_max * mean.sum() * len(th) * (1.0 / n + 1.0 / m.sample_count))


@pytest.mark.parametrize("gen,kw,n", [("c1", {}, 3000), ("c3", dict(sample_count=200), 200),
                                      ("c4", {}, 2000), ("c2", dict(noninternal=20, discrete=True), 500)])
def test_oracle_incremental_fast_mode_equals_fast_mode(gen, kw, n):
    """Mode 2 (the fast process computed incrementally, as the engine's fast kernel does: unstable
    sets, word sums, dependents only) gives the same trajectories as mode 1 (every rate each step),
    integer for integer; it is the CPU baseline on the GPU kernel's own algorithm."""
    from maboss.gpu_b200 import synth

    bnd, cfg = getattr(synth, gen)(**kw)
    m = OracleModel(bnd, cfg)
    a, b = m.run(n=n, mode=1), m.run(n=n, mode=2)
    assert a["transitions"] == b["transitions"] > 0
    for k in ("occ", "cnt", "h", "final", "fixed_states", "fixed_counts"):
        assert np.array_equal(a[k], b[k]), k
