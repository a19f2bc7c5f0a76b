"""The generated model code compiled for the host with g++ (it is plain C++ apart from CUDA
qualifiers), checked on random states:

* every `<node>_rate` (through `compute_transition_rates`, generator.cpp:84-144) equals the oracle's
  independent evaluation of the same model text, bit for bit;
* the straight-line helpers the exact kernels use instead of the reference's `rates[N]` array equal
  the reference-form computations on the same rates: `mbg_total_rate` the sum of
  `compute_transition_rates`, `mbg_entropy` `compute_transition_entropy` (generator.cpp:146-175),
  `mbg_select_flip(r)` the reference's prefix count (simulation.cu:9-21);
* `get_non_internal_index` (generator.cpp:207-235) packs the non-internal bits in node order;
* the incremental kernels' tables encode exactly what the rate functions compute: each node's own
  record (truth table and inputs) gives its logic, so its rate is its up/down rate when it
  differs from the logic and 0 otherwise; the fixed-point rates round the float rates; and a flip of
  node j changes no rate outside j's dependent records.

Models: the reference's four example models, the synthetic networks of the benchmarks and random
models whose rates mix the @logic form with general expressions (ternaries on node states, integer
and 6-digit literals, integer division, $variables).
"""
import ctypes as C
import os
import subprocess

import numpy as np
import pytest

import maboss.gpu_b200 as mb
from conftest import ROOT, model_text
from maboss.gpu_b200 import synth
from oracle.oracle import OracleModel

PRELUDE = r"""
#include <cstdint>
#include <cmath>
#define __device__
#define __forceinline__ inline
#define __constant__
struct uint2 { unsigned x, y; };
struct uint4 { unsigned x, y, z, w; };
template <class T> T __ldg(const T* p) { return *p; }
"""

WRAPPER = r"""
extern "C" float host_rates(float* r, const uint32_t* s) { return compute_transition_rates(r, s); }
extern "C" float host_entropy_ref(const float* r) { return compute_transition_entropy(r); }
extern "C" float host_total(const uint32_t* s) { return mbg_total_rate(s); }
extern "C" int host_select(const uint32_t* s, float r) { return mbg_select_flip(s, r); }
extern "C" float host_entropy(const uint32_t* s) { return mbg_entropy(s); }
extern "C" uint32_t host_ni_index(const uint32_t* s) { return get_non_internal_index(s); }
extern "C" int host_nonnegative() { return mbg_rates_nonnegative ? 1 : 0; }
#ifdef MBG_INCREMENTAL
extern "C" int host_has_tables() { return 1; }
extern "C" int host_rate_shift() { return mbg_inc_rate_shift; }
#ifdef MBG_INTEGER_RATES
extern "C" int host_integer_rates() { return 1; }
#else
extern "C" int host_integer_rates() { return 0; }
#endif
extern "C" unsigned host_q(int e) { return mbg_inc_q[e]; }
extern "C" float host_inc_rate(int e) { return mbg_inc_rate[e]; }
// logic of record r's node in state s: the truth table indexed by the input pattern
extern "C" int host_record_logic(int r, const uint32_t* s)
{
    const uint4 rec = mbg_inc_crec[r], ext = mbg_inc_cext[r];
    const int m = (rec.x >> 16) & 31;
    const unsigned ins[6] = { rec.z, rec.w, ext.x, ext.y, ext.z, ext.w };
    unsigned p = 0;
    for (int t = 0; t < m; t++)
    {
        const unsigned node = (ins[t >> 1] >> ((t & 1) * 16)) & 0xffffu;
        p |= ((s[node >> 5] >> (node & 31)) & 1u) << t;
    }
    const unsigned w = m <= 5 ? rec.y : mbg_inc_tt[rec.y + (p >> 5)];
    return (w >> (p & 31)) & 1u;
}
extern "C" int host_record_node(int r) { return (int)(mbg_inc_crec[r].x & 0xffffu); }
extern "C" int host_record_inputs(int r) { return (int)((mbg_inc_crec[r].x >> 16) & 31u); }
extern "C" int host_record_input(int r, int t)
{
    const uint4 rec = mbg_inc_crec[r], ext = mbg_inc_cext[r];
    const unsigned ins[6] = { rec.z, rec.w, ext.x, ext.y, ext.z, ext.w };
    return (int)((ins[t >> 1] >> ((t & 1) * 16)) & 0xffffu);
}
extern "C" int host_record_ni(int r) { return (int)((mbg_inc_crec[r].x >> 21) & 127u) - 1; }
extern "C" int host_self(int i) { return mbg_inc_self[i]; }
extern "C" int host_dep_first(int j) { return (int)mbg_inc_dep[2 * j]; }
extern "C" int host_dep_count(int j) { return (int)(mbg_inc_dep[2 * j + 1] & 0xffffu); }
struct host_view { const uint32_t *s, *u; uint32_t S(int w) const { return s[w]; } uint32_t U(int w) const { return u[w]; } };
// the generated straight-line entropy sums, and the same sums by the loop over the tables
extern "C" void host_ni_sums(const uint32_t* s, const uint32_t* u, float* out)
{
    float t = 0.f, tl = 0.f;
    mbg_ni_rate_sums(host_view{ s, u }, t, tl);
    float t2 = 0.f, tl2 = 0.f;
    for (int k = 0; k < mbg_noninternal_count; k++)
    {
        const int i = mbg_inc_ni_node[k];
        const uint32_t bit = 1u << (i & 31);
        if (u[i >> 5] & bit)
        {
            const bool up = (s[i >> 5] & bit) != 0;
            t2 += up ? mbg_inc_ni_down[k] : mbg_inc_ni_up[k];
            tl2 += up ? mbg_inc_ni_dl[k] : mbg_inc_ni_ul[k];
        }
    }
    out[0] = t; out[1] = tl; out[2] = t2; out[3] = tl2;
}
extern "C" int host_dep_ni(int j) { return (int)(mbg_inc_dep[2 * j + 1] >> 16) - 1; }
#else
extern "C" int host_has_tables() { return 0; }
#endif
"""


def _compile(code: str, tmp_path, tag: str) -> C.CDLL:
    src = tmp_path / f"{tag}.cpp"
    so = tmp_path / f"{tag}.so"
    src.write_text(PRELUDE + code + WRAPPER)
    subprocess.run(["g++", "-std=c++17", "-O1", "-shared", "-fPIC", "-o", str(so), str(src)], check=True,
                   capture_output=True, timeout=600)
    L = C.CDLL(str(so))
    u32p, f32p = C.POINTER(C.c_uint32), C.POINTER(C.c_float)
    for name, res, args in [("host_rates", C.c_float, [f32p, u32p]), ("host_entropy_ref", C.c_float, [f32p]),
                            ("host_total", C.c_float, [u32p]), ("host_select", C.c_int, [u32p, C.c_float]),
                            ("host_entropy", C.c_float, [u32p]), ("host_ni_index", C.c_uint32, [u32p]),
                            ("host_nonnegative", C.c_int, []), ("host_has_tables", C.c_int, [])]:
        getattr(L, name).restype = res
        getattr(L, name).argtypes = args
    if L.host_has_tables():
        for name, res, args in [("host_rate_shift", C.c_int, []), ("host_integer_rates", C.c_int, []),
                                ("host_q", C.c_uint, [C.c_int]),
                                ("host_inc_rate", C.c_float, [C.c_int]),
                                ("host_record_logic", C.c_int, [C.c_int, u32p]),
                                ("host_record_node", C.c_int, [C.c_int]), ("host_record_ni", C.c_int, [C.c_int]),
                                ("host_record_inputs", C.c_int, [C.c_int]),
                                ("host_record_input", C.c_int, [C.c_int, C.c_int]),
                                ("host_self", C.c_int, [C.c_int]), ("host_dep_first", C.c_int, [C.c_int]),
                                ("host_dep_count", C.c_int, [C.c_int]), ("host_dep_ni", C.c_int, [C.c_int]),
                                ("host_ni_sums", None, [C.c_void_p, C.c_void_p, C.c_void_p])]:
            getattr(L, name).restype = res
            getattr(L, name).argtypes = args
    return L


def _random_state(rng, n, words):
    bits = rng.random(n) < rng.uniform(0.2, 0.8)
    st = np.zeros(words, np.uint32)
    for i in np.nonzero(bits)[0]:
        st[i >> 5] |= np.uint32(1 << (i & 31))
    return st


def _ptr(a, t):
    return a.ctypes.data_as(C.POINTER(t))


def _check_model(bnd, cfg, tmp_path, tag, n_states=200, n_flip_states=20):
    model = mb.Model(bnd, cfg)
    o = OracleModel(bnd, cfg)
    N, W = o.nodes, o.words
    L = _compile(model.generate_code(), tmp_path, tag)
    rng = np.random.default_rng(abs(hash(tag)) % (1 << 32))
    rates = np.zeros(N, np.float32)
    nonneg = bool(L.host_nonnegative())
    tables = bool(L.host_has_tables())
    if tables:
        shift = L.host_rate_shift()
        for e in range(2 * N):
            r = np.float64(L.host_inc_rate(e))
            assert L.host_q(e) == int(np.rint(r * 2.0 ** shift)), (tag, e)
        # the fixed point: the largest shift <= 31 keeping every word's largest rate sum below
        # 2^32; the fast kernel's integer rates only when every positive rate gets >= 2^20 units
        hi = [max(float(L.host_inc_rate(2 * i)), float(L.host_inc_rate(2 * i + 1))) for i in range(N)]
        worst = max(sum(hi[32 * w:32 * w + 32]) for w in range(W))
        assert worst * 2.0 ** shift < 2.0 ** 32 and (shift == 31 or worst * 2.0 ** (shift + 1) >= 2.0 ** 32)
        fine = all(L.host_q(e) >= 2 ** 20 for e in range(2 * N) if L.host_inc_rate(e) > 0)
        assert bool(L.host_integer_rates()) == fine, tag
        ni_pos = {node: k for k, node in enumerate(o.noninternal)}
        deps = []
        for j in range(N):
            assert L.host_record_node(L.host_self(j)) == j
            f, c = L.host_dep_first(j), L.host_dep_count(j)
            assert f <= L.host_self(j) < f + c
            assert L.host_dep_ni(j) == ni_pos.get(j, -1)
            deps.append({L.host_record_node(d) for d in range(f, f + c)})
            for d in range(f, f + c):
                k = L.host_record_node(d)
                assert L.host_record_ni(d) == ni_pos.get(k, -1)
                # every record of node k carries k's own logic
                assert L.host_record_inputs(d) == L.host_record_inputs(L.host_self(k))
        # every node is re-evaluated after a flip of any of its logic's inputs
        for k in range(N):
            r = L.host_self(k)
            for t in range(L.host_record_inputs(r)):
                x = L.host_record_input(r, t)
                assert k in deps[x], (tag, k, x)
    for s in range(n_states):
        st = _random_state(rng, N, W)
        total = L.host_rates(_ptr(rates, C.c_float), _ptr(st, C.c_uint32))
        ref = np.array([o.rate(i, st.tolist()) for i in range(N)], np.float32)
        assert np.array_equal(rates, ref), (tag, s, np.nonzero(rates != ref)[0][:5])
        # reference order: sequential fp32 sum in node order
        acc = np.float32(0)
        prefix = np.zeros(N, np.float32)
        for i in range(N):
            acc = np.float32(acc + rates[i])
            prefix[i] = acc
        assert np.float32(total) == acc and np.float32(L.host_total(_ptr(st, C.c_uint32))) == acc
        h_ref = L.host_entropy_ref(_ptr(rates, C.c_float))
        h = L.host_entropy(_ptr(st, C.c_uint32))
        assert np.float32(h) == np.float32(h_ref) or (np.isnan(h) and np.isnan(h_ref))
        idx = 0
        for k, node in enumerate(o.noninternal):
            idx |= int((st[node >> 5] >> np.uint32(node & 31)) & 1) << k
        assert L.host_ni_index(_ptr(st, C.c_uint32)) == idx
        if nonneg and acc > 0:
            for u in rng.random(3):
                r = np.float32(np.float32(u) * acc)
                expect = min(int(np.count_nonzero(prefix < r)), N - 1)
                assert L.host_select(_ptr(st, C.c_uint32), C.c_float(r)) == expect
        if tables:
            for i in range(N):
                on = bool((st[i >> 5] >> np.uint32(i & 31)) & 1)
                logic = bool(L.host_record_logic(L.host_self(i), _ptr(st, C.c_uint32)))
                want = np.float32(L.host_inc_rate(2 * i + (1 if on else 0))) if on != logic else np.float32(0)
                assert rates[i] == want, (tag, s, i)
            if s < n_flip_states:
                for j in range(N):
                    st2 = st.copy()
                    st2[j >> 5] ^= np.uint32(1 << (j & 31))
                    r2 = np.zeros(N, np.float32)
                    L.host_rates(_ptr(r2, C.c_float), _ptr(st2, C.c_uint32))
                    changed = set(np.nonzero(r2 != rates)[0].tolist())
                    assert changed <= deps[j], (tag, j, changed - deps[j])
            # the straight-line entropy sums equal the table loop bit for bit (random unstable masks)
            un = _random_state(rng, N, W)
            sums = np.zeros(4, np.float32)
            L.host_ni_sums(st.ctypes.data, un.ctypes.data, sums.ctypes.data)
            assert sums[0] == sums[2] and sums[1] == sums[3], (tag, sums)
    return tables


@pytest.mark.parametrize("name", ["cellcycle", "sizek", "metastasis", "Montagud2022_Prostate_Cancer"])
def test_generated_code_of_example_models(name, tmp_path):
    _check_model(*model_text(name), tmp_path, name, n_states=100)


@pytest.mark.parametrize("gen,kw", [(synth.c1, {}), (synth.c2, dict(noninternal=20)), (synth.c4, {}),
                                    (synth.c5_base, dict(index=3))], ids=["c1", "c2", "c4", "c5_base3"])
def test_generated_code_of_synthetic_networks(gen, kw, tmp_path):
    assert _check_model(*gen(**kw), tmp_path, gen.__name__, n_states=100)


def test_generated_code_of_the_1000_node_network(tmp_path):
    assert _check_model(*synth.c3(), tmp_path, "c3", n_states=6, n_flip_states=1)


def _random_logic(rng, names, depth=0):
    if depth > 2 or rng.random() < 0.35:
        x = names[rng.integers(len(names))]
        return f"!{x}" if rng.random() < 0.3 else x
    op = rng.choice([" & ", " | ", " ^ "], p=[0.45, 0.45, 0.1])
    return f"({_random_logic(rng, names, depth + 1)}{op}{_random_logic(rng, names, depth + 1)})"


def _random_number(rng):
    k = rng.integers(4)
    if k == 0:
        return str(int(rng.integers(0, 6)))  # integer literal
    if k == 1:
        return f"{rng.uniform(0.01, 9.0):.6g}"
    if k == 2:
        return f"$v{rng.integers(4)}"
    return f"{rng.uniform(0.1, 3.0):.3f}"


def _random_rate(rng, names, depth=0):
    if depth > 1 or rng.random() < 0.4:
        return _random_number(rng)
    k = rng.integers(4)
    a, b = _random_rate(rng, names, depth + 1), _random_rate(rng, names, depth + 1)
    if k == 0:
        return f"({a} + {b})"
    if k == 1:
        return f"({a} * {b})"
    if k == 2:
        return f"({a} / {int(rng.integers(1, 5))})"  # integer division when a is an integer
    return f"({_random_logic(rng, names, 2)} ? {a} : {b})"


def _random_model(seed):
    rng = np.random.default_rng(seed)
    n = int(rng.integers(4, 14))
    names = [f"N{i}" for i in range(n)]
    bnd = ""
    tables = seed % 2 == 0  # all rates of the @logic form with constant U, D: the incremental tables
    for i, nm in enumerate(names):
        logic = _random_logic(rng, names)
        kind = 0 if tables else rng.integers(3)
        if kind == 0:  # the @logic form (incremental-kernel eligible)
            up, down = f"@logic ? {_random_number(rng)} : 0", f"@logic ? 0 : {_random_number(rng)}"
        elif kind == 1:
            up, down = f"@logic ? {_random_rate(rng, names)} : 0", f"@logic ? 0 : {_random_rate(rng, names)}"
        else:
            up, down = _random_rate(rng, names), _random_rate(rng, names)
        bnd += f"node {nm} {{ logic = {logic}; rate_up = {up}; rate_down = {down}; }}\n"
    cfg = "".join(f"$v{k} = {rng.uniform(0.05, 5.0):.7g};\n" for k in range(4))
    cfg += "".join(f"{nm}.is_internal = {int(rng.random() < 0.4)};\n" for nm in names)
    cfg += "max_time = 5; time_tick = 0.5; sample_count = 100;\n"
    return bnd, cfg


@pytest.mark.parametrize("seed", range(16))
def test_generated_code_of_random_models(seed, tmp_path):
    """Even seeds: every rate of the @logic form (the tables are checked too); odd seeds: general
    expressions, which leave the model to the dense kernels."""
    assert _check_model(*_random_model(seed), tmp_path, f"rand{seed}", n_states=60) == (seed % 2 == 0)


def wide_span_model(n=40, seed=7):
    """A @logic-form network whose rates span 1e-3 ... 1e3 (log-uniform): too wide for 2^20 units of
    the integer fixed point, so fast mode takes the dense fp32 kernel; exact mode keeps the
    incremental kernel."""
    rng = np.random.default_rng(seed)
    names = [f"S{i}" for i in range(n)]
    bnd = ""
    for i in range(n):
        a, b = rng.choice(n, 2, replace=False)
        op = " & " if rng.random() < 0.5 else " | "
        logic = f"{'!' if rng.random() < 0.5 else ''}{names[a]}{op}{'!' if rng.random() < 0.5 else ''}{names[b]}"
        up, down = 10.0 ** rng.uniform(-3, 3, 2)
        bnd += (f"node {names[i]} {{ logic = {logic}; rate_up = @logic ? {up:.6g} : 0; "
                f"rate_down = @logic ? 0 : {down:.6g}; }}\n")
    cfg = "".join(f"{names[i]}.is_internal = 1;\n" for i in range(6, n))
    cfg += "max_time = 10; time_tick = 0.5; sample_count = 1000;\n"
    return bnd, cfg


def test_generated_code_of_a_wide_rate_span_model(tmp_path):
    assert _check_model(*wide_span_model(), tmp_path, "wide", n_states=100)
    L = _compile(mb.Model(*wide_span_model()).generate_code(), tmp_path, "wide2")
    assert L.host_integer_rates() == 0


@pytest.mark.parametrize("family", ["EXACT", "FAST", "EPOCH"])
def test_wide_rate_span_model_compiles_for_sm100a(family, tmp_path):
    """The generated code of a model whose rates are too wide for the integer rates (fast mode: dense
    kernel; exact and epoch modes: incremental kernels) compiles in every kernel family with nvcc
    for sm_100a, as NVRTC compiles it at run time."""
    csrc = os.path.join(ROOT, "maboss", "gpu_b200", "csrc", "kernels")
    src = mb.Model(*wide_span_model()).generate_code() + f"\n#define MB_FAMILY_{family} 1\n"
    for f in ("params.cuh", "common.cuh", "engine.cuh"):
        src += open(os.path.join(csrc, f)).read() + "\n"
    (tmp_path / "m.cu").write_text(src)
    p = subprocess.run(["nvcc", "-std=c++17", "-gencode", "arch=compute_100a,code=sm_100a", "-O1", "-cubin",
                        "-o", str(tmp_path / "m.cubin"), str(tmp_path / "m.cu")], capture_output=True, text=True,
                       timeout=600)
    assert p.returncode == 0, p.stderr[-3000:]

