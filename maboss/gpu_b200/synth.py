"""Seeded synthetic Boolean networks in .bnd/.cfg form for the benchmark workloads.

Each generator returns (bnd_text, cfg_text). Rates are written with 6 significant digits so that
every consumer (the engine, the oracle, the reference) reads the same float values.

  c1  10 nodes, random 2-input AND/OR formulas, each literal negated with p=0.5, all rates 1,
      istate 0.5, continuous time, max_time 5, tick 0.2, 1e5 trajectories, all nodes non-internal
  c2  100 nodes (4 state words), 3 inputs per node in random AND/OR/NOT trees, rates
      lognormal(0,1), `internal_fraction` of the nodes internal, istate 0.3, max_time 100, tick 1,
      1e6 trajectories; continuous or discrete time
  c3  1000 nodes (32 state words), in-degree from a power law (exponent 2.5, max 8), threshold-style
      AND/OR formulas, rates uniform[0.1, 10], nodes 0-9 non-internal, max_time 50, tick 0.5,
      1e6 trajectories
  c4  50 nodes, 3 inputs, 20 nodes with named $u_i/$d_i rate parameters (40 parameters,
      lognormal(0, 0.5)), 8 output nodes non-internal, 1e6 trajectories
  c5  base networks of 20-500 nodes with 2-4 inputs (batched sweeps; network 0 has 20 nodes, network 7
      has 500)
"""
from __future__ import annotations

import numpy as np


def _g6(x: float) -> str:
    return f"{float(x):.6g}"


def _literal(rng: np.random.Generator, name: str, p_neg: float) -> str:
    return f"!{name}" if rng.random() < p_neg else name


def _tree(rng: np.random.Generator, names: list[str]) -> str:
    """Random AND/OR/NOT expression tree over the given input names (each used once)."""
    if len(names) == 1:
        return _literal(rng, names[0], 0.5)
    cut = int(rng.integers(1, len(names)))
    op = " & " if rng.random() < 0.5 else " | "
    expr = f"({_tree(rng, names[:cut])}{op}{_tree(rng, names[cut:])})"
    return f"!{expr}" if rng.random() < 0.25 else expr


def _node(name: str, logic: str, up: str, down: str) -> str:
    return (f"node {name}\n{{\n  logic = {logic};\n  rate_up = @logic ? {up} : 0;\n"
            f"  rate_down = @logic ? 0 : {down};\n}}\n\n")


def _cfg(names, internal, istate, sample_count, max_time, tick, discrete, seed, variables=None) -> str:
    lines = []
    for k, v in (variables or {}).items():
        lines.append(f"{k} = {_g6(v)};")
    for i, n in enumerate(names):
        lines.append(f"{n}.istate = {_g6(istate[i] if hasattr(istate, '__len__') else istate)};")
    for i, n in enumerate(names):
        if internal[i]:
            lines.append(f"{n}.is_internal = 1;")
    lines += [f"sample_count = {int(sample_count)};", f"max_time = {_g6(max_time)};",
              f"time_tick = {_g6(tick)};", f"discrete_time = {1 if discrete else 0};",
              f"seed_pseudorandom = {int(seed)};"]
    return "\n".join(lines) + "\n"


def c1(seed: int = 0, sample_count: int = 100_000, sim_seed: int = 0) -> tuple[str, str]:
    rng = np.random.default_rng(seed)
    n = 10
    names = [f"N{i}" for i in range(n)]
    bnd = ""
    for i in range(n):
        a, b = rng.choice(n, 2, replace=False)
        op = " & " if rng.random() < 0.5 else " | "
        logic = f"{_literal(rng, names[a], 0.5)}{op}{_literal(rng, names[b], 0.5)}"
        bnd += _node(names[i], logic, "1", "1")
    cfg = _cfg(names, [False] * n, 0.5, sample_count, 5, 0.2, False, sim_seed)
    return bnd, cfg


def c2(seed: int = 0, sample_count: int = 1_000_000, discrete: bool = False, internal_fraction: float = 0.2,
       noninternal: int | None = None, sim_seed: int = 0) -> tuple[str, str]:
    """`noninternal` overrides internal_fraction with an explicit count of output nodes (0..n-1)."""
    rng = np.random.default_rng(seed)
    n = 100
    names = [f"G{i}" for i in range(n)]
    bnd = ""
    for i in range(n):
        inputs = [names[j] for j in rng.choice(n, 3, replace=False)]
        up, down = np.exp(rng.normal(0.0, 1.0, 2))
        bnd += _node(names[i], _tree(rng, inputs), _g6(up), _g6(down))
    if noninternal is not None:
        internal = [i >= noninternal for i in range(n)]
    else:
        internal = list(rng.random(n) < internal_fraction)
    cfg = _cfg(names, internal, 0.3, sample_count, 100, 1, discrete, sim_seed)
    return bnd, cfg


def _power_law_degrees(rng: np.random.Generator, n: int, exponent: float, kmax: int) -> np.ndarray:
    k = np.arange(1, kmax + 1)
    p = k.astype(np.float64) ** (-exponent)
    p /= p.sum()
    return rng.choice(k, size=n, p=p)


def c3(seed: int = 0, sample_count: int = 1_000_000, n: int = 1000, n_out: int = 10, max_time: float = 50.0,
       tick: float = 0.5, sim_seed: int = 0) -> tuple[str, str]:
    rng = np.random.default_rng(seed)
    names = [f"X{i}" for i in range(n)]
    deg = _power_law_degrees(rng, n, 2.5, 8)
    bnd = ""
    for i in range(n):
        inputs = [names[j] for j in rng.choice(n, int(deg[i]), replace=False)]
        lits = [_literal(rng, x, 0.3) for x in inputs]
        if len(lits) <= 2:
            op = " & " if rng.random() < 0.5 else " | "
            logic = op.join(lits)
        else:
            # threshold-style: (at least one of the first half) AND/OR (all of the second half)
            h = len(lits) // 2
            first, second = " | ".join(lits[:h]), " & ".join(lits[h:])
            op = " & " if rng.random() < 0.5 else " | "
            logic = f"({first}){op}({second})"
        up, down = rng.uniform(0.1, 10.0, 2)
        bnd += _node(names[i], logic, _g6(up), _g6(down))
    internal = [i >= n_out for i in range(n)]
    cfg = _cfg(names, internal, 0.5, sample_count, max_time, tick, False, sim_seed)
    return bnd, cfg


def c4(seed: int = 0, sample_count: int = 1_000_000, sim_seed: int = 0) -> tuple[str, str]:
    rng = np.random.default_rng(seed)
    n, n_param_nodes, n_out = 50, 20, 8
    names = [f"P{i}" for i in range(n)]
    variables = {}
    bnd = ""
    for i in range(n):
        inputs = [names[j] for j in rng.choice(n, 3, replace=False)]
        logic = _tree(rng, inputs)
        if i < n_param_nodes:
            variables[f"$u_{i}"] = float(np.exp(rng.normal(0.0, 0.5)))
            variables[f"$d_{i}"] = float(np.exp(rng.normal(0.0, 0.5)))
            bnd += _node(names[i], logic, f"$u_{i}", f"$d_{i}")
        else:
            bnd += _node(names[i], logic, "1", "1")
    internal = [i >= n_out for i in range(n)]
    cfg = _cfg(names, internal, 0.5, sample_count, 20, 0.5, False, sim_seed, variables)
    return bnd, cfg


def c5_base(index: int, sample_count: int = 10_000, sim_seed: int = 0) -> tuple[str, str]:
    """Base network `index` (0..7) of the batched sweep: 20-500 nodes (network 0 has 20 and network 7
    has 500, so the sweep spans the whole range; the others are log-uniform in it), 2-4 inputs,
    8 outputs, node rates given by variables $u_i / $d_i (lognormal(0, 0.5)) so that variants can
    rescale them."""
    rng = np.random.default_rng(1000 + index)
    n = int(np.round(np.exp(rng.uniform(np.log(20), np.log(500)))))
    n = {0: 20, 7: 500}.get(index, n)
    kin = int(rng.integers(2, 5))
    names = [f"B{index}_{i}" for i in range(n)]
    variables = {}
    bnd = ""
    for i in range(n):
        inputs = [names[j] for j in rng.choice(n, kin, replace=False)]
        up, down = np.exp(rng.normal(0.0, 0.5, 2))
        variables[f"$u_{i}"], variables[f"$d_{i}"] = float(_g6(up)), float(_g6(down))
        bnd += _node(names[i], _tree(rng, inputs), f"$u_{i}", f"$d_{i}")
    max_time = float(rng.choice([20.0, 50.0, 100.0, 200.0]))
    internal = [i >= 8 for i in range(n)]
    cfg = _cfg(names, internal, 0.5, sample_count, max_time, max_time / 40, False, sim_seed, variables)
    return bnd, cfg


def c5_sweep(n_variants: int = 256, seed: int = 0):
    """The batched sweep: (base network index, variable overrides, trajectories) per variant, with
    lognormal(0, 0.3) multipliers on every rate and trajectories uniform in [1e3, 1e5]."""
    rng = np.random.default_rng(seed)
    bases = [c5_base(i) for i in range(8)]
    base_vars = []
    for bnd, cfg in bases:
        vals = {}
        for line in cfg.splitlines():
            if line.startswith("$"):
                k, v = line.rstrip(";").split(" = ")
                vals[k] = float(v)
        base_vars.append(vals)
    variants = []
    for v in range(n_variants):
        net = v % 8
        mult = np.exp(rng.normal(0.0, 0.3, len(base_vars[net])))
        params = {k: float(np.float32(x * m)) for (k, x), m in zip(base_vars[net].items(), mult)}
        variants.append((net, params, int(rng.integers(1_000, 100_001))))
    return bases, variants


WORKLOADS = {"c1": c1, "c2": c2, "c3": c3, "c4": c4}
