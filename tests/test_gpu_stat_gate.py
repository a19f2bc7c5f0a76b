"""Statistical gate of the fast mode (the benchmark's mode) against the exact mode, which is
bit-identical to the reference build (tests/test_gpu_ref_parity.py), on the benchmark networks at
>= 1e5 trajectories each.

The fast mode runs the same Markov process with other random streams (Philox) and integer rates
(every positive rate >= 2^20 units of the fixed point, relative rounding error <= 2^-21); it is
correct when its estimates and the exact mode's are two samples of the same distribution:
window probabilities, final-state distribution and fixed-point frequencies agree within a
family-wise binomial bound (conftest.assert_statistically_equal: 4 sigma or the Bonferroni
quantile over the populated bins at alpha = 1e-3, and mean z^2 < 1.2). Reference semantics:
simulation.cu:104-147 (waiting time, flip selection in proportion to the rates).

A network whose rates span 1e-3 ... 1e3 is too wide for the integer rates; its fast mode takes the
dense fp32 kernel and passes the same gate.
"""
import numpy as np
import pytest

import maboss.gpu_b200 as mb
from conftest import assert_statistically_equal
from maboss.gpu_b200 import synth
from test_codegen_host import wide_span_model

pytestmark = pytest.mark.gpu


def _fixed_freq(res, n):
    return {tuple(int(x) for x in st): c / n for st, c in res.fixed}


def _gate(gpu, bnd, cfg, n, fast_seed=1):
    model = mb.Model(bnd, cfg)
    mod = gpu.compile(model)
    exact = mod.run(mode="exact", sample_count=n)
    fast = mod.run(mode="fast", sample_count=n, seed=fast_seed)
    assert exact.fixed_overflow == 0 and fast.fixed_overflow == 0
    assert_statistically_equal(exact.window_probs, n, fast.window_probs, n)
    assert_statistically_equal(exact.final_counts / n, n, fast.final_counts / n, n)
    fa, fb = _fixed_freq(exact, n), _fixed_freq(fast, n)
    keys = sorted(set(fa) | set(fb))
    if keys:
        assert_statistically_equal(np.array([fa.get(k, 0.0) for k in keys]), n,
                                   np.array([fb.get(k, 0.0) for k in keys]), n)
    return exact, fast


@pytest.mark.parametrize("gen,kw,n", [(synth.c3, {}, 100_000), (synth.c2, dict(noninternal=20), 100_000),
                                      (synth.c2, dict(noninternal=20, discrete=True), 100_000),
                                      (synth.c4, {}, 200_000)],
                         ids=["c3", "c2b", "c2b_discrete", "c4"])
def test_fast_mode_statistically_equals_exact_mode(gpu, gen, kw, n):
    exact, fast = _gate(gpu, *gen(**kw), n)
    # the transition counts are sums of n independent trajectory lengths: their difference within
    # 6 standard errors, taking the per-trajectory standard deviation as at most 3x the mean length
    a, b = exact.transitions, fast.transitions
    assert abs(a - b) <= 6 * np.sqrt(2 * n) * 3 * (a / n), (a, b)


def test_fast_mode_on_a_wide_rate_span(gpu):
    """Rates from 1e-3 to 1e3: the fast mode's dense fp32 kernel against the exact mode."""
    _gate(gpu, *wide_span_model(), 200_000)
