"""CPU ORACLE (test infrastructure) -- ctypes wrapper of liboracle.so.

Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg use this module; the
engine never does. See oracle.cpp for what it restates and how it is pinned.
"""
from __future__ import annotations

import ctypes as C
import math
import os
import subprocess

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB = None


def build() -> str:
    """Compile liboracle.so in place (needs g++ with OpenMP)."""
    subprocess.run(["make", "-s", "-C", _HERE], check=True)
    return os.path.join(_HERE, "liboracle.so")


def lib() -> C.CDLL:
    global _LIB
    if _LIB is None:
        path = os.path.join(_HERE, "liboracle.so")
        if not os.path.exists(path):
            build()
        L = C.CDLL(path)
        L.oracle_model_load.restype = C.c_void_p
        L.oracle_model_load.argtypes = [C.c_char_p, C.c_char_p, C.c_char_p, C.c_size_t]
        L.oracle_model_free.argtypes = [C.c_void_p]
        L.oracle_model_dims.argtypes = [C.c_void_p] + [C.POINTER(C.c_int)] * 5 + [
            C.POINTER(C.c_longlong), C.POINTER(C.c_ulonglong), C.POINTER(C.c_float), C.POINTER(C.c_float)]
        L.oracle_model_noninternal.argtypes = [C.c_void_p, C.POINTER(C.c_int)]
        L.oracle_model_rate.restype = C.c_float
        L.oracle_model_rate.argtypes = [C.c_void_p, C.c_int, C.POINTER(C.c_uint32)]
        L.oracle_run.restype = C.c_void_p
        L.oracle_run.argtypes = [C.c_void_p, C.c_int, C.c_longlong, C.c_ulonglong, C.c_ulonglong, C.c_int,
                                 C.c_int, C.c_int, C.c_int]
        L.oracle_run_ex.restype = C.c_void_p
        L.oracle_run_ex.argtypes = [C.c_void_p, C.c_int, C.c_longlong, C.c_ulonglong, C.c_ulonglong, C.c_int,
                                    C.c_int, C.c_int, C.c_int, C.c_int]
        L.oracle_result_sparse_size.argtypes = [C.c_void_p, C.POINTER(C.c_longlong), C.POINTER(C.c_longlong)]
        L.oracle_result_sparse.argtypes = [C.c_void_p] + [C.c_void_p] * 5
        L.oracle_result_free.argtypes = [C.c_void_p]
        L.oracle_result_get.argtypes = [C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p,
                                        C.POINTER(C.c_ulonglong), C.POINTER(C.c_double)]
        L.oracle_result_num_fixed.argtypes = [C.c_void_p]
        L.oracle_result_fixed.argtypes = [C.c_void_p, C.c_void_p, C.c_void_p]
        L.oracle_model_set_variables.restype = C.c_int
        L.oracle_model_set_variables.argtypes = [C.c_void_p, C.POINTER(C.c_char_p), C.POINTER(C.c_float), C.c_int]
        L.oracle_trace.argtypes = [C.c_void_p, C.c_int, C.c_ulonglong, C.c_ulonglong, C.c_int,
                                   C.POINTER(C.c_int), C.POINTER(C.c_float), C.c_int]
        L.oracle_gradient.restype = C.c_int
        L.oracle_gradient.argtypes = [C.c_void_p, C.c_ulonglong, C.c_ulonglong, C.c_longlong, C.c_void_p, C.c_int,
                                      C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p]
        _LIB = L
    return _LIB


def occupancy_exponent(n: int, tick: float, discrete: bool) -> int:
    """Fixed-point exponent of window occupancy sums (same rule as the engine)."""
    if discrete:
        return 0
    bound = max(1.0, float(max(1, n)) * float(max(np.float32(tick), np.float32(1e-30))))
    return min(max(int(math.floor(61.0 - math.log2(bound))), 0), 100)


def entropy_exponent(n: int, tick: float, discrete: bool) -> int:
    per = 8.0 if discrete else 8.0 * float(max(np.float32(tick), np.float32(1e-30)))
    bound = max(1.0, float(max(1, n)) * per)
    return min(max(int(math.floor(61.0 - math.log2(bound))), 0), 100)


class OracleModel:
    def __init__(self, bnd_text: str, cfg_text: str):
        err = C.create_string_buffer(4096)
        self._h = lib().oracle_model_load(bnd_text.encode(), cfg_text.encode(), err, 4096)
        if not self._h:
            raise ValueError(err.value.decode())
        n, w, k, T, d = (C.c_int() for _ in range(5))
        sc, seed = C.c_longlong(), C.c_ulonglong()
        tick, mt = C.c_float(), C.c_float()
        lib().oracle_model_dims(self._h, C.byref(n), C.byref(w), C.byref(k), C.byref(T), C.byref(d),
                                C.byref(sc), C.byref(seed), C.byref(tick), C.byref(mt))
        self.nodes, self.words, self.k, self.windows = n.value, w.value, k.value, T.value
        self.discrete = bool(d.value)
        self.sample_count, self.seed = sc.value, seed.value
        self.tick, self.max_time = tick.value, mt.value
        ni = (C.c_int * max(1, self.k))()
        lib().oracle_model_noninternal(self._h, ni)
        self.noninternal = list(ni)[: self.k]

    @classmethod
    def from_files(cls, bnd: str, cfg: str) -> "OracleModel":
        with open(bnd) as f, open(cfg) as g:
            return cls(f.read(), g.read())

    def __del__(self):
        if getattr(self, "_h", None):
            lib().oracle_model_free(self._h)
            self._h = None

    def set_variables(self, params: dict) -> None:
        """Set $variables; rates of @logic-form nodes become exact floats (as in batched runs)."""
        names = (C.c_char_p * max(1, len(params)))(*[k.encode() for k in params])
        values = (C.c_float * max(1, len(params)))(*[float(v) for v in params.values()])
        if lib().oracle_model_set_variables(self._h, names, values, len(params)) != 0:
            raise KeyError("unknown variable")

    def rate(self, node: int, state_words) -> float:
        arr = (C.c_uint32 * self.words)(*state_words)
        return lib().oracle_model_rate(self._h, node, arr)

    def run(self, n: int | None = None, mode: int = 0, seed: int | None = None, first: int = 0,
            traj_len: int = 100, occ_exp: int | None = None, ent_exp: int | None = None,
            threads: int = 0, sparse: bool = False) -> dict:
        """Simulate trajectories [first, first+n) on the CPU. mode 0 = exact, 1 = fast, 2 = fast computed
        incrementally like the engine's fast kernel (same results as mode 1). With more than 20
        non-internal nodes (or sparse=True) the windows and final states come back as sparse entries
        under the key "sparse" (the dense arrays are then empty; states as (bits 0-63, bits 64-127) pairs)."""
        n = self.sample_count if n is None else n
        seed = self.seed if seed is None else seed
        if occ_exp is None:
            occ_exp = occupancy_exponent(n, self.tick, self.discrete)
        if ent_exp is None:
            ent_exp = entropy_exponent(n, self.tick, self.discrete)
        r = lib().oracle_run_ex(self._h, mode, n, seed, first, traj_len, occ_exp, ent_exp, threads,
                                1 if sparse else 0)
        if not r:
            raise ValueError("oracle: unsupported model (more than 112 non-internal nodes)")
        try:
            nw, nf = C.c_longlong(), C.c_longlong()
            is_sparse = lib().oracle_result_sparse_size(r, C.byref(nw), C.byref(nf)) == 1
            sp = None
            if is_sparse:
                w = np.zeros(max(1, nw.value), np.int32)
                ix = np.zeros((max(1, nw.value), 2), np.uint64)
                val = np.zeros(max(1, nw.value), np.int64)
                fi = np.zeros((max(1, nf.value), 2), np.uint64)
                fc = np.zeros(max(1, nf.value), np.uint64)
                lib().oracle_result_sparse(r, w.ctypes.data, ix.ctypes.data, val.ctypes.data, fi.ctypes.data,
                                           fc.ctypes.data)
                sp = dict(windows=w[:nw.value], states=ix[:nw.value], raw=val[:nw.value],
                          final_states=fi[:nf.value], final_counts=fc[:nf.value])
            S = 0 if is_sparse else 1 << self.k
            T = self.windows
            occ = np.zeros(T * S, np.int64)
            cnt = np.zeros(T * S, np.uint32)
            h = np.zeros(T, np.int64)
            fin = np.zeros(S, np.uint32)
            tr, secs = C.c_ulonglong(), C.c_double()
            lib().oracle_result_get(r, occ.ctypes.data, cnt.ctypes.data, h.ctypes.data, fin.ctypes.data,
                                    C.byref(tr), C.byref(secs))
            nfx = lib().oracle_result_num_fixed(r)
            fs = np.zeros(max(1, nfx) * self.words, np.uint32)
            fcx = np.zeros(max(1, nfx), np.uint32)
            lib().oracle_result_fixed(r, fs.ctypes.data, fcx.ctypes.data)
        finally:
            lib().oracle_result_free(r)
        out = dict(n=n, windows=T, bins=S, discrete=self.discrete, tick=self.tick,
                   occ=occ.reshape(T, S), cnt=cnt.reshape(T, S), h=h, final=fin,
                   fixed_states=fs[: nfx * self.words].reshape(nfx, self.words), fixed_counts=fcx[:nfx],
                   transitions=tr.value, seconds=secs.value, occ_exp=occ_exp, ent_exp=ent_exp, sparse=sp)
        out["probs"] = window_probs(out)
        out["th"] = window_th(out)
        if sp is not None:
            raw = sp["raw"].astype(np.float64)
            sp["probs"] = raw / n if self.discrete else (raw / 2.0 ** occ_exp) / (n * float(np.float32(self.tick)))
        return out

    def gradient(self, n: int, cotangent: np.ndarray, derivatives: list[list[tuple[int, float]]],
                 n_params: int, seed: int | None = None, first: int = 0) -> np.ndarray:
        """Score-function gradient of sum(cotangent * window probabilities) over the fast-mode
        (integer-rate) trajectories first .. first + n - 1, by the direct definition
        (oracle.cpp: gradient_integer). derivatives[2 i] / [2 i + 1] list the (parameter, d rate /
        d parameter) pairs of node i's up / down rate. Scaled like the probabilities."""
        seed = self.seed if seed is None else seed
        cot = np.ascontiguousarray(cotangent, dtype=np.float64).ravel()
        assert cot.size == self.windows << self.k and len(derivatives) == 2 * self.nodes
        gptr = np.zeros(2 * self.nodes + 1, np.int32)
        gp, gd = [], []
        for e, lst in enumerate(derivatives):
            for p, d in lst:
                gp.append(p)
                gd.append(d)
            gptr[e + 1] = len(gp)
        gp = np.ascontiguousarray(gp if gp else [0], dtype=np.int32)
        gd = np.ascontiguousarray(gd if gd else [0.0], dtype=np.float32)
        out = np.zeros(max(1, n_params), np.float64)
        if lib().oracle_gradient(self._h, seed, first, n, cot.ctypes.data, n_params, gptr.ctypes.data,
                                 gp.ctypes.data, gd.ctypes.data, out.ctypes.data) != 0:
            raise ValueError("the gradient needs integer rates and at most 20 non-internal nodes")
        scale = 1.0 / (n * (1.0 if self.discrete else float(np.float32(self.tick))))
        return out[:n_params] * scale

    def trace(self, traj: int, mode: int = 0, seed: int | None = None, traj_len: int = 100, cap: int = 1 << 16):
        seed = self.seed if seed is None else seed
        flips = (C.c_int * cap)()
        times = (C.c_float * cap)()
        k = lib().oracle_trace(self._h, mode, seed, traj, traj_len, flips, times, cap)
        k = min(k, cap)
        return list(flips)[:k], list(times)[:k]


def window_probs(r: dict) -> np.ndarray:
    """Probability per (window, bin) (window_average_small.cpp:126-140), float64."""
    n = r["n"]
    if r["discrete"]:
        return r["cnt"].astype(np.float64) / n
    return (r["occ"].astype(np.float64) / 2.0 ** r["occ_exp"]) / (n * float(np.float32(r["tick"])))


def window_th(r: dict) -> np.ndarray:
    v = (r["h"].astype(np.float64) / 2.0 ** r["ent_exp"]) / r["n"]
    return v if r["discrete"] else v / float(np.float32(r["tick"]))
