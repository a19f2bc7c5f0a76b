"""The allocation-free fixed-point statistics entry point, mb_fixed_states_noalloc.

Some callers cannot allocate device memory: their framework's caching allocator owns the whole
device, or the process runs under a fixed memory budget, or a cudaMalloc would stall a device that
is busy with other work. For them the library offers one entry point whose work table is a static
device array. These tests check, through the C ABI, that it returns exactly what the regular
(allocating) fixed-point statistics return on the same device buffers, on two calls in a row (the
static table keeps the previous call's contents, so the second call also checks that it is
cleared), and that sizes beyond its stated limits are refused with a clear error.
"""
import ctypes as C

import numpy as np
import pytest

import maboss.gpu_b200 as mb

pytestmark = pytest.mark.gpu


def _model(n_nodes: int) -> "mb.Model":
    names = [f"F{i}" for i in range(n_nodes)]
    bnd = "".join(f"node {names[i]} {{ logic = {names[(i + 1) % n_nodes]}; rate_up = @logic ? 1 : 0; "
                  f"rate_down = @logic ? 0 : 1; }}\n" for i in range(n_nodes))
    cfg = "".join(f"{names[i]}.is_internal = 1;\n" for i in range(4, n_nodes)) + "max_time = 1; time_tick = 0.5;"
    return mb.Model(bnd, cfg)


def _inputs(torch, n: int, stride: int, words: int, pool: int, seed: int):
    g = np.random.default_rng(seed)
    states = g.integers(0, 2**32, size=(pool, words), dtype=np.uint64).astype(np.uint32)
    pick = g.integers(0, pool, size=n)
    soa = np.zeros((words, stride), np.uint32)
    soa[:, :n] = states[pick].T
    status = np.zeros(stride, np.uint8)
    status[:n] = g.integers(0, 3, size=n)  # CONTINUE / FINISHED / FIXED_POINT
    dev = torch.device("cuda", 0)
    return (torch.from_numpy(soa.view(np.int32).ravel()).to(dev), torch.from_numpy(status).to(dev))


def _reference_order(records):
    # std::map<static_state_t> order: compare from the highest word down
    return sorted(records, key=lambda r: tuple(reversed(r[0])))


def _noalloc(torch, n, stride, words, last, stat, cap):
    out_states = torch.zeros(cap * words, dtype=torch.int32, device="cuda")
    out_counts = torch.zeros(cap, dtype=torch.int32, device="cuda")
    out_n = C.c_int(-1)
    torch.cuda.synchronize()
    st = mb.lib().mb_fixed_states_noalloc(None, n, stride, words, C.c_void_p(last.data_ptr()),
                                          C.c_void_p(stat.data_ptr()), C.c_void_p(out_states.data_ptr()),
                                          C.c_void_p(out_counts.data_ptr()), cap, C.byref(out_n))
    return st, out_n.value, out_states, out_counts


def _declare():
    f = mb.lib().mb_fixed_states_noalloc
    f.restype = C.c_int
    f.argtypes = [C.c_void_p, C.c_int, C.c_int, C.c_int, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_int,
                  C.POINTER(C.c_int)]


@pytest.mark.parametrize("n_nodes", [96, 200])  # 3 words (exact keys) and 7 words (hashed keys)
def test_noalloc_matches_allocating_fixed_point_statistics(n_nodes):
    import torch

    _declare()
    ctx = mb.Context(0)
    model = _model(n_nodes)
    mod = ctx.compile(model)
    _, words = mod.state_size
    n, stride, cap = 50_000, 50_123, 4096
    for call, (pool, seed) in enumerate([(300, 1), (700, 2)]):  # two calls in a row
        last, stat = _inputs(torch, n, stride, words, pool, seed)
        torch.cuda.synchronize()
        stats = mod.stats(0.5, 1.0, False, model.noninternal_nodes, n)
        stats.fixed(n, stride, last.data_ptr(), stat.data_ptr())
        expected = [(tuple(int(x) for x in s), c) for s, c in stats.finalize(n).fixed]
        st, got_n, out_states, out_counts = _noalloc(torch, n, stride, words, last, stat, cap)
        assert st == 0, mb.lib().mb_last_error()
        assert got_n == len(expected), (call, got_n, len(expected))
        s = out_states[: got_n * words].cpu().numpy().view(np.uint32).reshape(got_n, words)
        c = out_counts[:got_n].cpu().numpy()
        got = _reference_order([(tuple(int(x) for x in s[i]), int(c[i])) for i in range(got_n)])
        assert got == expected, call
        assert sum(cnt for _, cnt in got) == int((stat[:n] == 2).sum())


def test_noalloc_rejects_sizes_beyond_its_limits():
    import torch

    _declare()
    mb.Context(0)
    words = 32
    # more distinct fixed points than the static table holds for 32-word states (16384)
    n = 40_000
    last, stat = _inputs(torch, n, n, words, pool=n, seed=3)
    stat.fill_(2)
    st, got_n, _, _ = _noalloc(torch, n, n, words, last, stat, 64)
    assert st == 5 and b"static table" in mb.lib().mb_last_error()  # MB_ERR_LIMIT
    assert got_n == -1  # the number of distinct fixed points is unknown after an overflow
    # state words beyond the maximum
    st, _, _, _ = _noalloc(torch, 10, 10, 65, last, stat, 64)
    assert st == 5 and b"state_words" in mb.lib().mb_last_error()
    # outputs too small for the result
    last, stat = _inputs(torch, 5_000, 5_000, 2, pool=100, seed=4)
    stat.fill_(2)
    st, got_n, _, _ = _noalloc(torch, 5_000, 5_000, 2, last, stat, 10)
    assert st == 5 and got_n == 100 and b"out_cap" in mb.lib().mb_last_error()
