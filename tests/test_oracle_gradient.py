"""Pins the oracle's score-function gradient (oracle.cpp: gradient_integer), the checker of the
engine's gradient kernel, against exact derivatives.

A single node switching on at rate u and off at rate d has window averages of P(on) in closed
form, and so do their derivatives. A 3-node network is small enough to solve exactly: its
8-state chain gives the expected cotangent-weighted window statistic (continuous time: window
integrals of the transient distribution, by the matrix exponential of the generator; discrete
time: the jump chain step by step, a fixed point counted once and then stopped, as the window
statistic does), and central differences of that exact value are exact derivatives up to
rounding. The oracle's estimate over its own fast-mode trajectories must agree within its spread.
"""
import itertools
import math

import numpy as np
import pytest
import scipy.linalg

from oracle.oracle import OracleModel

TWO_STATE = """
node A { logic = !A; rate_up = @logic ? $u : 0; rate_down = @logic ? 0 : $d; }
"""


def window_mean(u, d, p0, a, b):
    lam = u + d
    pi = u / lam
    return pi + (p0 - pi) * (math.exp(-lam * a) - math.exp(-lam * b)) / (lam * (b - a))


def two_state_derivatives():
    """d rate / d theta per (node, direction): node A's up rate is $u (parameter 0), down $d (1)."""
    return [[(0, 1.0)], [(1, 1.0)]]


def test_oracle_gradient_of_two_state_chain_matches_closed_form():
    u, d, p0, tick, tmax = 1.3, 0.7, 0.25, 0.5, 3.0
    o = OracleModel(TWO_STATE, f"$u = {u}; $d = {d}; A.istate = {p0}; max_time = {tmax}; time_tick = {tick};")
    T = int(round(tmax / tick))
    cot = np.zeros((T, 2))
    cot[:, 1] = 1.0
    est = np.array([o.gradient(250_000, cot, two_state_derivatives(), 2, seed=s) for s in range(4)])
    h = 1e-6

    def L(uu, dd):
        return sum(window_mean(uu, dd, p0, w * tick, (w + 1) * tick) for w in range(T))

    exact = np.array([(L(u + h, d) - L(u - h, d)) / (2 * h), (L(u, d + h) - L(u, d - h)) / (2 * h)])
    mean, sem = est.mean(axis=0), est.std(axis=0, ddof=1) / 2.0
    assert np.all(np.abs(mean - exact) < 4 * sem + 0.01 * np.abs(exact)), (mean, exact, sem)


def test_oracle_gradient_is_zero_for_a_deterministic_discrete_chain():
    o = OracleModel(TWO_STATE, "$u = 1.3; $d = 0.7; A.istate = 0.25; max_time = 3; time_tick = 0.5; "
                               "discrete_time = 1;")
    cot = np.ones((o.windows, 2))
    g = o.gradient(1000, cot, two_state_derivatives(), 2, seed=1)
    assert np.all(np.abs(g) < 1e-12), g


NET3 = """
node A { logic = !B | C; rate_up = @logic ? $ua : 0; rate_down = @logic ? 0 : $da; }
node B { logic = A; rate_up = @logic ? $ub : 0; rate_down = @logic ? 0 : $db; }
node C { logic = A & !B; rate_up = @logic ? $uc : 0; rate_down = @logic ? 0 : $dc; }
"""
NET3_NAMES = ["$ua", "$da", "$ub", "$db", "$uc", "$dc"]
NET3_THETA = dict(zip(NET3_NAMES, [1.3, 0.7, 2.1, 0.9, 0.6, 1.7]))
NET3_ISTATE = [0.3, 0.6, 0.5]
NET3_LOGIC = [lambda s: (not s[1]) or s[2], lambda s: s[0], lambda s: s[0] and not s[1]]
NET3_TMAX, NET3_TICK = 5.0, 0.5


def _net3_cfg(discrete: bool) -> str:
    c = "".join(f"{k} = {v};" for k, v in NET3_THETA.items())
    c += "".join(f"{n}.istate = {p};" for n, p in zip("ABC", NET3_ISTATE))
    c += f"max_time = {NET3_TMAX}; time_tick = {NET3_TICK}; C.is_internal = 1;"
    return c + (" discrete_time = 1;" if discrete else "")


def _net3_chain(th):
    """States (A, B, C), initial distribution and per-state rates of the 3-node network."""
    ru = [th["$ua"], th["$ub"], th["$uc"]]
    rd = [th["$da"], th["$db"], th["$dc"]]
    states = list(itertools.product([0, 1], repeat=3))
    p0 = np.array([np.prod([NET3_ISTATE[i] if s[i] else 1 - NET3_ISTATE[i] for i in range(3)]) for s in states])
    rates = [[(rd[i] if s[i] else ru[i]) if bool(NET3_LOGIC[i](s)) != bool(s[i]) else 0.0 for i in range(3)]
             for s in states]
    return states, p0, rates


def _net3_exact(th, cot, T, discrete):
    states, p0, rates = _net3_chain(th)
    index = {s: k for k, s in enumerate(states)}
    bins = np.array([s[0] | (s[1] << 1) for s in states])  # non-internal nodes A, B
    if discrete:
        L, p = 0.0, p0.copy()
        for w in range(T):
            L += float(p @ cot[w, bins])
            q = np.zeros_like(p)
            for k, s in enumerate(states):
                a0 = sum(rates[k])
                for i in range(3):
                    if rates[k][i] > 0:
                        t = list(s)
                        t[i] ^= 1
                        q[index[tuple(t)]] += p[k] * rates[k][i] / a0
            p = q  # fixed points (a0 = 0) drop out after being counted once
        return L
    Q = np.zeros((8, 8))
    for k, s in enumerate(states):
        for i in range(3):
            if rates[k][i] > 0:
                t = list(s)
                t[i] ^= 1
                Q[k, index[tuple(t)]] += rates[k][i]
                Q[k, k] -= rates[k][i]
    # [[Q, I], [0, 0]] exponentiated over a window gives the integral of exp(Q t) over it
    M = np.zeros((16, 16))
    M[:8, :8] = Q
    M[:8, 8:] = np.eye(8)
    E = scipy.linalg.expm(M * NET3_TICK)
    step, integral = E[:8, :8], E[:8, 8:]
    L, p = 0.0, p0.copy()
    for w in range(T):
        L += float((p @ integral) @ cot[w, bins]) / NET3_TICK
        p = p @ step
    return L


@pytest.mark.parametrize("discrete", [False, True], ids=["continuous", "discrete"])
def test_oracle_gradient_of_3_node_network_matches_exact_derivatives(discrete):
    o = OracleModel(NET3, _net3_cfg(discrete))
    T, S = o.windows, 1 << o.k
    assert (T, S, o.nodes) == (10, 4, 3)
    cot = np.random.default_rng(2).normal(size=(T, S))
    deriv = [[] for _ in range(6)]
    for p, k in enumerate(NET3_NAMES):
        deriv[2 * "abc".index(k[2]) + (0 if k[1] == "u" else 1)].append((p, 1.0))
    h = 1e-6
    exact = np.array([(_net3_exact(dict(NET3_THETA, **{k: NET3_THETA[k] + h}), cot, T, discrete) -
                       _net3_exact(dict(NET3_THETA, **{k: NET3_THETA[k] - h}), cot, T, discrete)) / (2 * h)
                      for k in NET3_NAMES])
    # the forward statistic itself first: the oracle's trajectories follow the exact chain
    fwd = (o.run(400_000, mode=1, seed=0)["probs"] * cot).sum()
    assert abs(fwd - _net3_exact(NET3_THETA, cot, T, discrete)) < 0.01
    est = np.array([o.gradient(500_000, cot, deriv, len(NET3_NAMES), seed=s) for s in range(4)])
    mean, sem = est.mean(axis=0), est.std(axis=0, ddof=1) / 2.0
    assert np.all(np.abs(mean - exact) <= 4 * sem + 1e-3 * np.abs(exact) + 1e-6), (mean, exact, sem)
