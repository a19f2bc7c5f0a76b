"""Python binding of the B200 trajectory engine (thin layer over the C ABI, no compute here)."""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass

import numpy as np

from ._lib import check, lib, read_string

MODES = {"exact": 0, "fast": 1, "epoch": 2, "epoch_dense": 3}


class RunConfig(C.Structure):
    """mb_run_config (include/maboss_b200.h)."""

    _fields_ = [
        ("mode", C.c_int),
        ("sample_count", C.c_longlong),
        ("seed", C.c_ulonglong),
        ("first_traj", C.c_ulonglong),
        ("traj_len", C.c_int),
        ("batch_limit", C.c_int),
        ("block", C.c_int),
        ("blocks_per_sm", C.c_int),
        ("fixed_capacity_log2", C.c_int),
        ("stats_trajectories", C.c_longlong),
        ("bin_capacity_log2", C.c_int),
        ("refill_reuse_rng", C.c_int),
    ]


class ResultDesc(C.Structure):
    """mb_result_desc (include/maboss_b200.h)."""

    _fields_ = [
        ("n_nodes", C.c_int),
        ("n_windows", C.c_int),
        ("discrete_time", C.c_int),
        ("time_tick", C.c_float),
        ("max_time", C.c_float),
        ("noninternal_nodes", C.c_void_p),
        ("n_noninternal", C.c_int),
        ("n_trajectories", C.c_longlong),
        ("occupancy_exponent", C.c_int),
        ("entropy_exponent", C.c_int),
        ("occupancy", C.c_void_p),
        ("counts", C.c_void_p),
        ("entropy", C.c_void_p),
        ("final_counts", C.c_void_p),
        ("n_fixed", C.c_int),
        ("fixed_states", C.c_void_p),
        ("fixed_counts", C.c_void_p),
        ("transitions", C.c_ulonglong),
    ]


class Model:
    """A parsed .bnd/.cfg model (the reference's `driver`)."""

    def __init__(self, bnd_text: str, cfg_text: str):
        h = C.c_void_p()
        check(lib().mb_model_parse_text(bnd_text.encode(), cfg_text.encode(), C.byref(h)))
        self._h = h

    @classmethod
    def from_files(cls, bnd_path: str, cfg_path: str) -> "Model":
        self = cls.__new__(cls)
        h = C.c_void_p()
        check(lib().mb_model_parse_files(bnd_path.encode(), cfg_path.encode(), C.byref(h)))
        self._h = h
        return self

    def __del__(self):
        h = getattr(self, "_h", None)
        if h:
            lib().mb_model_free(h)
            self._h = None

    @property
    def num_nodes(self) -> int:
        n = C.c_int()
        check(lib().mb_model_num_nodes(self._h, C.byref(n)))
        return n.value

    @property
    def node_names(self) -> list[str]:
        return [read_string(lib().mb_model_node_name, self._h, i) for i in range(self.num_nodes)]

    def node_info(self, i: int) -> tuple[float, bool]:
        istate, internal = C.c_float(), C.c_int()
        check(lib().mb_model_node_info(self._h, i, C.byref(istate), C.byref(internal)))
        return istate.value, bool(internal.value)

    @property
    def noninternal_nodes(self) -> list[int]:
        return [i for i in range(self.num_nodes) if not self.node_info(i)[1]]

    def set_istate(self, i: int, p: float) -> None:
        check(lib().mb_model_set_istate(self._h, i, p))

    def constant(self, name: str) -> float:
        v = C.c_float()
        check(lib().mb_model_get_constant(self._h, name.encode(), C.byref(v)))
        return v.value

    def set_constant(self, name: str, value: float) -> None:
        check(lib().mb_model_set_constant(self._h, name.encode(), value))

    def variable(self, name: str) -> float:
        v = C.c_float()
        check(lib().mb_model_get_variable(self._h, name.encode(), C.byref(v)))
        return v.value

    def set_variable(self, name: str, value: float) -> None:
        check(lib().mb_model_set_variable(self._h, name.encode(), value))

    @property
    def variables(self) -> dict[str, float]:
        n = C.c_int()
        check(lib().mb_model_num_variables(self._h, C.byref(n)))
        names = [read_string(lib().mb_model_variable_name, self._h, i) for i in range(n.value)]
        return {k: self.variable(k) for k in names}

    def apply_cfg_overrides(self) -> None:
        """mb_model_apply_cfg_overrides: node attributes defined again in the .cfg replace the .bnd's
        (opt-in; the reference keeps the first definition)."""
        check(lib().mb_model_apply_cfg_overrides(self._h))

    def generate_code(self) -> str:
        return read_string(lib().mb_model_generate_code, self._h)


class Context:
    """A CUDA device (primary context) and the engine's stream."""

    def __init__(self, device: int = 0):
        h = C.c_void_p()
        check(lib().mb_context_create(device, C.byref(h)))
        self._h = h
        self.device = device

    def __del__(self):
        h = getattr(self, "_h", None)
        if h:
            lib().mb_context_free(h)
            self._h = None

    @property
    def stream(self) -> int:
        s = C.c_void_p()
        check(lib().mb_context_stream(self._h, C.byref(s)))
        return s.value or 0

    @property
    def sm_count(self) -> int:
        n = C.c_int()
        check(lib().mb_context_sm_count(self._h, C.byref(n)))
        return n.value

    def compile(self, model: Model) -> "Module":
        h = C.c_void_p()
        check(lib().mb_module_compile_model(self._h, model._h, C.byref(h)))
        return Module(h, self, model)

    def compile_source(self, code: str) -> "Module":
        h = C.c_void_p()
        check(lib().mb_module_compile(self._h, code.encode(), C.byref(h)))
        return Module(h, self, None)


class Module:
    """Kernels of one model, NVRTC-compiled for sm_100a (the reference's kernel_compiler)."""

    def __init__(self, h, ctx: Context, model: Model | None):
        self._h = h
        self.ctx = ctx
        self.model = model

    def __del__(self):
        h = getattr(self, "_h", None)
        if h:
            lib().mb_module_free(h)
            self._h = None

    @property
    def state_size(self) -> tuple[int, int]:
        n, w = C.c_int(), C.c_int()
        check(lib().mb_module_state_size(self._h, C.byref(n), C.byref(w)))
        return n.value, w.value

    def config(self, mode: str = "exact", sample_count: int | None = None, seed: int | None = None,
               first_traj: int = 0, traj_len: int = 100, batch_limit: int = 1_000_000, block: int = 256,
               blocks_per_sm: int = 0, fixed_capacity_log2: int = 0, stats_trajectories: int = 0,
               bin_capacity_log2: int = 0, refill_reuse_rng: bool = False) -> RunConfig:
        cfg = RunConfig()
        check(lib().mb_run_config_default(self.model._h, C.byref(cfg)))
        cfg.mode = MODES[mode]
        if sample_count is not None:
            cfg.sample_count = sample_count
        if seed is not None:
            cfg.seed = seed
        cfg.first_traj = first_traj
        cfg.traj_len = traj_len
        cfg.batch_limit = batch_limit
        cfg.block = block
        cfg.blocks_per_sm = blocks_per_sm
        cfg.fixed_capacity_log2 = fixed_capacity_log2
        cfg.stats_trajectories = stats_trajectories
        cfg.bin_capacity_log2 = bin_capacity_log2
        cfg.refill_reuse_rng = 1 if refill_reuse_rng else 0
        return cfg

    def autotune(self, mode: str = "fast", sample_count: int | None = None, **kw) -> dict:
        """mb_autotune: the fastest launch shape for this run (pass the result to run() / runner())."""
        cfg = self.config(mode, sample_count, **kw)
        rate = C.c_float()
        shapes = (C.c_int * 48)()
        rates = (C.c_float * 16)()
        n = C.c_int()
        check(lib().mb_autotune(self._h, C.byref(cfg), C.byref(rate), shapes, rates, 16, C.byref(n)))
        cands = [dict(block=shapes[3 * i], blocks_per_sm=shapes[3 * i + 1], transitions_per_s=rates[i])
                 for i in range(min(n.value, 16))]
        return dict(block=cfg.block, blocks_per_sm=cfg.blocks_per_sm, transitions_per_s=rate.value,
                    candidates=cands)

    def run(self, mode: str = "exact", sample_count: int | None = None, **kw) -> "Result":
        """simulation_runner::run_simulation with the built-in statistics (synchronous)."""
        cfg = self.config(mode, sample_count, **kw)
        h = C.c_void_p()
        check(lib().mb_run(self._h, C.byref(cfg), C.byref(h)))
        return Result(h)

    def runner(self, mode: str = "exact", sample_count: int | None = None, **kw) -> "Runner":
        """Buffers allocated once; launch() is asynchronous on the context's stream."""
        cfg = self.config(mode, sample_count, **kw)
        h = C.c_void_p()
        check(lib().mb_runner_create(self._h, C.byref(cfg), C.byref(h)))
        return Runner(h, self, cfg)

    # -- kernel entry points on caller-owned device buffers (integer device addresses)
    def launch_initialize_random(self, n: int, seed: int, first: int, rands: int, stream: int = 0) -> None:
        check(lib().mb_launch_initialize_random(self._h, stream or None, n, seed, first, rands))

    def launch_initialize_initial_state(self, n: int, stride: int, istate: int, last_states: int,
                                        last_times: int, rands: int, stream: int = 0) -> None:
        check(lib().mb_launch_initialize_initial_state(self._h, stream or None, n, stride, istate, last_states,
                                                        last_times, rands))

    def launch_simulate(self, n: int, stride: int, traj_len: int, last_states: int, last_times: int, rands: int,
                        traj_states: int, traj_times: int, traj_h: int, statuses: int, transitions: int,
                        stream: int = 0) -> None:
        check(lib().mb_launch_simulate(self._h, stream or None, n, stride, traj_len, last_states, last_times, rands,
                                       traj_states, traj_times, traj_h, statuses, transitions))

    def stats(self, time_tick: float, max_time: float, discrete: bool, noninternal: list[int],
              sample_count: int) -> "Stats":
        arr = (C.c_int * max(1, len(noninternal)))(*noninternal)
        h = C.c_void_p()
        check(lib().mb_stats_create(self._h, time_tick, max_time, int(discrete), arr, len(noninternal),
                                    sample_count, C.byref(h)))
        return Stats(h, self)


class Runner:
    def __init__(self, h, mod: Module, cfg: RunConfig):
        self._h = h
        self.mod = mod
        self.cfg = cfg

    def __del__(self):
        h = getattr(self, "_h", None)
        if h:
            lib().mb_runner_free(h)
            self._h = None

    def launch(self, stream: int = 0) -> None:
        check(lib().mb_runner_launch(self._h, stream or None))

    def result(self, stream: int = 0) -> "Result":
        h = C.c_void_p()
        check(lib().mb_runner_result(self._h, stream or None, C.byref(h)))
        return Result(h)

    @property
    def kernel_launches(self) -> int:
        n = C.c_uint()
        check(lib().mb_runner_kernel_launches(self._h, C.byref(n)))
        return n.value


def _names_values(params: dict[str, float] | None):
    params = params or {}
    names = (C.c_char_p * max(1, len(params)))(*[k.encode() for k in params])
    values = (C.c_float * max(1, len(params)))(*[float(v) for v in params.values()])
    return names, values, len(params)


class Batch:
    """Parameter variants of one or more networks in one persistent launch (fast-mode algorithm)."""

    def __init__(self, ctx: Context):
        h = C.c_void_p()
        check(lib().mb_batch_create(ctx._h, C.byref(h)))
        self._h = h
        self.ctx = ctx
        self._models = []

    def __del__(self):
        h = getattr(self, "_h", None)
        if h:
            lib().mb_batch_free(h)
            self._h = None

    def add_model(self, model: Model) -> int:
        n = C.c_int()
        check(lib().mb_batch_add_model(self._h, model._h, C.byref(n)))
        self._models.append(model)
        return n.value

    def add_variant(self, net: int, n_traj: int, params: dict[str, float] | None = None,
                    first_traj: int = 0, grad_params: list[str] | None = None,
                    mutants: dict[str, bool] | None = None) -> int:
        """A variant of network `net` (`params`: its $variable values); with `grad_params`, the
        $variables whose gradient run_gradient computes for it; with `mutants` ({node: True for
        forced on, False for forced off}), a mutant (mb_batch_add_mutant)."""
        names, values, k = _names_values(params)
        v = C.c_int()
        if mutants:
            if grad_params:
                raise ValueError("a mutant variant has no gradient parameters")
            nodes = (C.c_char_p * len(mutants))(*[n.encode() for n in mutants])
            on = (C.c_int * len(mutants))(*[1 if x else 0 for x in mutants.values()])
            check(lib().mb_batch_add_mutant(self._h, net, names, values, k, n_traj, first_traj, nodes, on,
                                            len(mutants), C.byref(v)))
        elif grad_params:
            gp = (C.c_char_p * len(grad_params))(*[g.encode() for g in grad_params])
            check(lib().mb_batch_add_variant_grad(self._h, net, names, values, k, n_traj, first_traj, gp,
                                                  len(grad_params), C.byref(v)))
        else:
            check(lib().mb_batch_add_variant(self._h, net, names, values, k, n_traj, first_traj, C.byref(v)))
        self._n_variants = getattr(self, "_n_variants", 0) + 1
        return v.value

    def set_variables(self, variant: int, params: dict[str, float]) -> None:
        """mb_batch_set_variables: new values of some of a variant's $variables, in place."""
        names, values, k = _names_values(params)
        check(lib().mb_batch_set_variables(self._h, variant, names, values, k))

    def run(self, seed: int = 0) -> float:
        ms = C.c_float()
        check(lib().mb_batch_run(self._h, seed, C.byref(ms)))
        return ms.value

    def run_gradient(self, seed: int, cotangents: dict[int, np.ndarray]) -> float:
        """mb_batch_run_gradient: one run with a cotangent per variant (`cotangents[v]`, shape
        [windows, 2^k]; missing variants take zeros). Returns the kernel time in ms."""
        n = getattr(self, "_n_variants", 0)
        arrays = {v: np.ascontiguousarray(c, dtype=np.float64).ravel() for v, c in cotangents.items()}
        ptrs = (C.c_void_p * max(1, n))(*[arrays[v].ctypes.data if v in arrays else None for v in range(n)])
        ms = C.c_float()
        check(lib().mb_batch_run_gradient(self._h, seed, ptrs, n, C.byref(ms)))
        return ms.value

    def gradient(self, variant: int) -> np.ndarray:
        """mb_batch_gradient: d sum(cotangent * window_probs) / d grad_params of the last gradient run."""
        n = C.c_int()
        check(lib().mb_batch_gradient(self._h, variant, None, 0, C.byref(n)))
        out = np.zeros(max(1, n.value), np.float64)
        check(lib().mb_batch_gradient(self._h, variant, out.ctypes.data_as(C.POINTER(C.c_double)), n.value,
                                      C.byref(n)))
        return out[: n.value]

    def result(self, variant: int) -> "Result":
        h = C.c_void_p()
        check(lib().mb_batch_result(self._h, variant, C.byref(h)))
        return Result(h)

    def set_specialize(self, on: bool = True) -> None:
        """mb_batch_set_specialize: a batch of one network runs kernels compiled for it (default) or
        the ahead-of-time kernels that take any networks; both give the same results."""
        check(lib().mb_batch_set_specialize(self._h, 1 if on else 0))

    def set_options(self, use_graph: bool = True, autotune: bool = True) -> None:
        """mb_batch_set_options: CUDA-graph replay of runs and launch-shape autotuning."""
        check(lib().mb_batch_set_options(self._h, 1 if use_graph else 0, 1 if autotune else 0))

    @property
    def info(self) -> dict:
        """Launch shape of the last run, node count of its CUDA graph, autotuner timings."""
        b, ps, t = C.c_int(), C.c_int(), C.c_int()
        g, n = C.c_uint(), C.c_uint()
        check(lib().mb_batch_info(self._h, C.byref(b), C.byref(ps), C.byref(g), C.byref(n), C.byref(t)))
        tuning = []
        for i in range(t.value):
            gr, bl, bp, ms = C.c_int(), C.c_int(), C.c_int(), C.c_float()
            check(lib().mb_batch_tuning(self._h, i, C.byref(gr), C.byref(bl), C.byref(bp), C.byref(ms)))
            tuning.append(dict(gradient=bool(gr.value), block=bl.value, blocks_per_sm=bp.value, kernel_ms=ms.value))
        return dict(block=b.value, blocks_per_sm=ps.value, grid=g.value, graph_nodes=n.value, tuning=tuning)


def gradient(ctx: Context, model: Model, params: dict[str, float], cotangent: np.ndarray, n_traj: int,
             seed: int = 0) -> tuple[np.ndarray, "Result"]:
    """d/dparams of sum(cotangent * window_probs) by the score-function estimator (same trajectories
    as the forward statistics, which are returned too)."""
    names, values, k = _names_values(params)
    cot = np.ascontiguousarray(cotangent, dtype=np.float64).ravel()
    grad = np.zeros(max(1, k), np.float64)
    h = C.c_void_p()
    check(lib().mb_gradient(ctx._h, model._h, names, values, k, n_traj, seed, cot.ctypes.data, grad.ctypes.data,
                            C.byref(h)))
    return grad[:k], Result(h)


def mutant_sweep(ctx: Context, model: Model, n_traj: int, nodes: list[str] | None = None, seed: int = 0,
                 params: dict[str, float] | None = None) -> dict:
    """Mutant analysis in one launch: the wild type and, for every listed node (default: all), the
    node forced on and forced off (mb_batch_add_mutant). Returns {("wt",): Result,
    (node, True): Result, (node, False): Result}."""
    b = Batch(ctx)
    net = b.add_model(model)
    nodes = model.node_names if nodes is None else nodes
    keys = [("wt",)] + [(n, on) for n in nodes for on in (True, False)]
    ids = [b.add_variant(net, n_traj, params)] + [b.add_variant(net, n_traj, params, mutants={n: on})
                                                  for n in nodes for on in (True, False)]
    b.run(seed)
    return {k: b.result(v) for k, v in zip(keys, ids)}


def merge_results(results: list["Result"]) -> "Result":
    """mb_result_merge: the statistics of the union of disjoint trajectory shards of one job."""
    hs = (C.c_void_p * len(results))(*[r._h for r in results])
    out = C.c_void_p()
    check(lib().mb_result_merge(hs, len(results), C.byref(out)))
    return Result(out)


def rand_state_size() -> int:
    return int(lib().mb_rand_state_size())


class Stats:
    """Device accumulators of the window / final / fixed statistics plugins."""

    def __init__(self, h, mod: Module):
        self._h = h
        self.mod = mod

    def __del__(self):
        h = getattr(self, "_h", None)
        if h:
            lib().mb_stats_free(h)
            self._h = None

    def window(self, n, stride, traj_len, traj_states, traj_times, traj_h, stream: int = 0):
        check(lib().mb_launch_window_average_stats(self._h, stream or None, n, stride, traj_len, traj_states,
                                                   traj_times, traj_h))

    def final(self, n, stride, last_states, statuses, stream: int = 0):
        check(lib().mb_launch_final_states_stats(self._h, stream or None, n, stride, last_states, statuses))

    def fixed(self, n, stride, last_states, statuses, stream: int = 0):
        check(lib().mb_launch_fixed_states_stats(self._h, stream or None, n, stride, last_states, statuses))

    def finalize(self, n_trajectories: int) -> "Result":
        h = C.c_void_p()
        check(lib().mb_stats_finalize(self._h, n_trajectories, C.byref(h)))
        return Result(h)


@dataclass
class Dims:
    windows: int
    bins: int
    noninternal: int
    state_words: int
    nodes: int


class Result:
    """Statistics of one run (window probabilities, entropies, final states, fixed points)."""

    def __init__(self, h):
        self._h = h
        w, b, k, sw, n = (C.c_int() for _ in range(5))
        check(lib().mb_result_dims(h, C.byref(w), C.byref(b), C.byref(k), C.byref(sw), C.byref(n)))
        self.dims = Dims(w.value, b.value, k.value, sw.value, n.value)

    def __del__(self):
        h = getattr(self, "_h", None)
        if h:
            lib().mb_result_free(h)
            self._h = None

    @property
    def transitions(self) -> int:
        t = C.c_ulonglong()
        check(lib().mb_result_transitions(self._h, C.byref(t)))
        return t.value

    @property
    def timing(self) -> tuple[float, float, int]:
        k, t, e = C.c_float(), C.c_float(), C.c_int()
        check(lib().mb_result_timing(self._h, C.byref(k), C.byref(t), C.byref(e)))
        return k.value, t.value, e.value

    @property
    def window_probs(self) -> np.ndarray:
        out = np.zeros((self.dims.windows, self.dims.bins), np.float64)
        check(lib().mb_result_window_probs(self._h, out.ctypes.data))
        return out

    @property
    def window_entropy(self) -> np.ndarray:
        out = np.zeros(self.dims.windows, np.float64)
        check(lib().mb_result_window_entropy(self._h, out.ctypes.data))
        return out

    def raw(self) -> dict:
        T, S = self.dims.windows, self.dims.bins
        occ = np.zeros(T * S, np.int64)
        cnt = np.zeros(T * S, np.uint32)
        h = np.zeros(T, np.int64)
        eo, eh = C.c_int(), C.c_int()
        check(lib().mb_result_window_raw(self._h, occ.ctypes.data, cnt.ctypes.data, h.ctypes.data,
                                         C.byref(eo), C.byref(eh)))
        return dict(occ=occ.reshape(T, S), cnt=cnt.reshape(T, S), h=h, occ_exp=eo.value, ent_exp=eh.value)

    @property
    def final_counts(self) -> np.ndarray:
        out = np.zeros(self.dims.bins, np.uint32)
        check(lib().mb_result_final_counts(self._h, out.ctypes.data))
        return out

    @property
    def fixed_overflow(self) -> int:
        n, o = C.c_int(), C.c_uint()
        check(lib().mb_result_num_fixed(self._h, C.byref(n), C.byref(o)))
        return o.value

    @property
    def fixed(self) -> list[tuple[np.ndarray, int]]:
        n, o = C.c_int(), C.c_uint()
        check(lib().mb_result_num_fixed(self._h, C.byref(n), C.byref(o)))
        out = []
        for i in range(n.value):
            st = np.zeros(self.dims.state_words, np.uint32)
            c = C.c_uint()
            check(lib().mb_result_fixed(self._h, i, st.ctypes.data, C.byref(c)))
            out.append((st, c.value))
        return out

    def info(self) -> dict:
        """mb_result_info: trajectory count, time constants and non-internal nodes."""
        n, d, t, m = C.c_longlong(), C.c_int(), C.c_float(), C.c_float()
        ni = np.zeros(max(1, self.dims.noninternal), np.int32)
        check(lib().mb_result_info(self._h, C.byref(n), C.byref(d), C.byref(t), C.byref(m), ni.ctypes.data))
        return dict(n_trajectories=n.value, discrete=bool(d.value), time_tick=t.value, max_time=m.value,
                    noninternal=[int(x) for x in ni[: self.dims.noninternal]])

    @classmethod
    def from_raw(cls, *, n_nodes: int, n_windows: int, discrete: bool, time_tick: float, max_time: float,
                 noninternal: list[int], n_trajectories: int, occ_exp: int, ent_exp: int, occ=None, cnt=None,
                 h=None, final=None, fixed_states=None, fixed_counts=None, transitions: int = 0) -> "Result":
        """mb_result_create: a result from raw accumulators (window sums in fixed point)."""
        S = 1 << len(noninternal)
        keep = []

        def arr(a, dtype, size):
            x = np.ascontiguousarray(np.asarray(a, dtype).reshape(-1))
            if x.size != size:
                raise ValueError(f"expected {size} values, got {x.size}")
            keep.append(x)
            return x.ctypes.data

        words = (n_nodes + 31) // 32
        fs = np.zeros((0, words), np.uint32) if fixed_states is None else np.asarray(fixed_states, np.uint32)
        fc = np.zeros(0, np.uint32) if fixed_counts is None else np.asarray(fixed_counts, np.uint32)
        d = ResultDesc()
        d.n_nodes, d.n_windows, d.discrete_time = n_nodes, n_windows, 1 if discrete else 0
        d.time_tick, d.max_time = time_tick, max_time
        d.noninternal_nodes = arr(noninternal, np.int32, len(noninternal)) if noninternal else None
        d.n_noninternal = len(noninternal)
        d.n_trajectories = n_trajectories
        d.occupancy_exponent, d.entropy_exponent = occ_exp, ent_exp
        if discrete:
            d.counts = arr(cnt, np.uint32, n_windows * S)
        else:
            d.occupancy = arr(occ, np.int64, n_windows * S)
        d.entropy = arr(h, np.int64, n_windows)
        d.final_counts = arr(final, np.uint32, S)
        d.n_fixed = len(fc)
        if len(fc):
            d.fixed_states = arr(fs, np.uint32, len(fc) * words)
            d.fixed_counts = arr(fc, np.uint32, len(fc))
        d.transitions = transitions
        h_out = C.c_void_p()
        check(lib().mb_result_create(C.byref(d), C.byref(h_out)))
        return cls(h_out)

    @property
    def is_sparse(self) -> bool:
        """More than 20 non-internal nodes: windows and final states as sparse entries."""
        return self.dims.bins == 0 and self.dims.noninternal > 20

    @property
    def windows_sparse(self) -> bool:
        """mb_result_windows_sparse: the windows are stored as sparse entries (more than 20 non-internal
        nodes, or a large dense histogram of which only the non-zero cells were copied back);
        sparse() gives them, window_probs / raw() still give the dense arrays."""
        v = C.c_int()
        check(lib().mb_result_windows_sparse(self._h, C.byref(v)))
        return bool(v.value)

    def sparse(self) -> dict:
        """mb_result_sparse_*: window entries (window, state, raw sum, probability) sorted by window then
        state, final states and counts, and the number of bin additions lost to a full table. States are
        non-internal indices as (bits 0-63, bits 64-127) uint64 pairs."""
        nw, nf, ovf = C.c_longlong(), C.c_longlong(), C.c_uint()
        check(lib().mb_result_sparse_size(self._h, C.byref(nw), C.byref(nf), C.byref(ovf)))
        # every entry is written by the C ABI: no zero fill (the arrays reach gigabytes)
        w = np.empty(max(1, nw.value), np.int32)
        st = np.empty((max(1, nw.value), 2), np.uint64)
        raw = np.empty(max(1, nw.value), np.int64)
        pr = np.empty(max(1, nw.value), np.float64)
        check(lib().mb_result_sparse_windows(self._h, w.ctypes.data, st.ctypes.data, raw.ctypes.data, pr.ctypes.data))
        fs = np.empty((max(1, nf.value), 2), np.uint64)
        fc = np.empty(max(1, nf.value), np.uint32)
        check(lib().mb_result_sparse_final(self._h, fs.ctypes.data, fc.ctypes.data))
        n, m = nw.value, nf.value
        return dict(windows=w[:n], states=st[:n], raw=raw[:n], probs=pr[:n], final_states=fs[:m],
                    final_counts=fc[:m], overflow=ovf.value)

    def write_csv(self, model: Model, prefix: str) -> None:
        check(lib().mb_result_write_csv(self._h, model._h, prefix.encode()))

    def write_final_csv(self, model: Model, prefix: str) -> None:
        """mb_result_write_final_csv: <prefix>_finalprob.csv (opt-in; the reference writes no such file)."""
        check(lib().mb_result_write_final_csv(self._h, model._h, prefix.encode()))

    def visualize(self, model: Model) -> str:
        return read_string(lib().mb_result_visualize, self._h, model._h)
