"""The host decode of the sparse window bins (csrc/sparse_bins.cpp), compiled for the test with g++:
sorted (key, value) pairs of the device bin table -> per-window entries, window offsets and final
states, against a sequential restatement; single-threaded (small inputs) and split over threads
(large inputs), with runs of equal keys across the nominal chunk boundaries."""
import ctypes as C
import os
import subprocess

import numpy as np
import pytest

from conftest import ROOT

SHIM = r"""
#include "sparse_bins.h"
#include <cstring>
#include <stdexcept>
extern "C" int decode(const uint64_t* keys, const long long* vals, size_t n, int n_windows, int threads,
                      int* sp_w, uint64_t* sp_idx, long long* sp_val, size_t* sp_begin, uint64_t* fin_idx,
                      unsigned* fin_cnt, size_t* counts)
{
    mb::bulk_vector<int> w; mb::bulk_vector<unsigned __int128> idx; mb::bulk_vector<long long> val;
    std::vector<size_t> begin;
    std::vector<unsigned __int128> fi; std::vector<unsigned> fc;
    mb::decode_sorted_bins(keys, vals, n, n_windows, threads, w, idx, val, begin, fi, fc);
    counts[0] = w.size(); counts[1] = fi.size();
    for (size_t i = 0; i < w.size(); i++) { sp_w[i] = w[i]; sp_idx[2 * i] = (uint64_t)idx[i];
        sp_idx[2 * i + 1] = (uint64_t)(idx[i] >> 64); sp_val[i] = val[i]; }
    for (size_t i = 0; i < begin.size(); i++) sp_begin[i] = begin[i];
    for (size_t i = 0; i < fi.size(); i++) { fin_idx[2 * i] = (uint64_t)fi[i]; fin_idx[2 * i + 1] = (uint64_t)(fi[i] >> 64);
        fin_cnt[i] = fc[i]; }
    return 0;
}
extern "C" int throwing(int T, int bad, unsigned* hits)
{
    // every chunk records that it ran; chunk `bad` then throws (bad == 0: the calling thread's chunk)
    try
    {
        mb::parallel_for(T, [&](int t) {
            __atomic_fetch_add(&hits[t], 1u, __ATOMIC_RELAXED);
            if (t == bad)
                throw std::runtime_error("chunk failed");
        });
    }
    catch (const std::runtime_error& e)
    {
        return std::strcmp(e.what(), "chunk failed") == 0 ? 1 : 2;
    }
    return 0;
}
extern "C" void ranges(size_t n, int threads, unsigned* hits)
{
    mb::parallel_ranges(n, threads, [&](size_t a, size_t b) { for (size_t i = a; i < b; i++) hits[i]++; });
}
"""


@pytest.fixture(scope="module")
def decoder(tmp_path_factory):
    d = tmp_path_factory.mktemp("sparse_bins")
    csrc = os.path.join(ROOT, "maboss", "gpu_b200", "csrc")
    (d / "shim.cpp").write_text(SHIM)
    so = d / "decode.so"
    subprocess.run(["g++", "-std=c++17", "-O2", "-shared", "-fPIC", "-pthread", f"-I{csrc}", "-o", str(so),
                    str(d / "shim.cpp"), os.path.join(csrc, "sparse_bins.cpp")], check=True, timeout=300)
    L = C.CDLL(str(so))
    L.decode.argtypes = [C.c_void_p, C.c_void_p, C.c_size_t, C.c_int, C.c_int] + [C.c_void_p] * 7
    L.ranges.argtypes = [C.c_size_t, C.c_int, C.c_void_p]
    L.throwing.argtypes = [C.c_int, C.c_int, C.c_void_p]
    return L


def _random_bins(rng, n, n_windows, dup_fraction):
    """Sorted keys {lo, hi = idx_hi | (w + 1) << 48}, some repeated, windows 0..n_windows (the last: finals)."""
    w = rng.integers(0, n_windows + 1, n).astype(np.uint64)
    lo = rng.integers(0, 1 << 63, n, dtype=np.uint64) * np.uint64(2) + rng.integers(0, 2, n, dtype=np.uint64)
    hi_idx = rng.integers(0, 1 << 48, n, dtype=np.uint64)
    hi = hi_idx | ((w + np.uint64(1)) << np.uint64(48))
    # repeat some keys (adjacent after sorting), in runs of 2 to 40
    reps = np.where(rng.random(n) < dup_fraction, rng.integers(2, 41, n), 1)
    lo, hi = np.repeat(lo, reps), np.repeat(hi, reps)
    order = np.lexsort((lo, hi))
    keys = np.empty((len(order), 2), np.uint64)
    keys[:, 0], keys[:, 1] = lo[order], hi[order]
    vals = rng.integers(1, 1 << 40, len(order)).astype(np.int64)
    return keys, vals


def _reference(keys, vals, n_windows):
    sp_w, sp_idx, sp_val, fin_idx, fin_cnt = [], [], [], [], []
    i, n = 0, len(keys)
    while i < n:
        j, v = i, 0
        while j < n and keys[j, 0] == keys[i, 0] and keys[j, 1] == keys[i, 1]:
            v += int(vals[j])
            j += 1
        w = int(keys[i, 1] >> np.uint64(48)) - 1
        idx = (int(keys[i, 0]), int(keys[i, 1] & np.uint64((1 << 48) - 1)))
        if w < n_windows:
            sp_w.append(w), sp_idx.append(idx), sp_val.append(v)
        else:
            fin_idx.append(idx), fin_cnt.append(v & 0xffffffff)
        i = j
    begin = [int(np.searchsorted(np.array(sp_w, np.int64), w, "left")) for w in range(n_windows + 1)]
    return sp_w, sp_idx, sp_val, begin, fin_idx, fin_cnt


def _decode(L, keys, vals, n_windows, threads):
    n = len(keys)
    m = max(1, n)
    sp_w, sp_idx, sp_val = np.empty(m, np.int32), np.empty((m, 2), np.uint64), np.empty(m, np.int64)
    begin = np.empty(n_windows + 1, np.uint64)
    fin_idx, fin_cnt, counts = np.empty((m, 2), np.uint64), np.empty(m, np.uint32), np.zeros(2, np.uint64)
    keys = np.ascontiguousarray(keys) if n else np.zeros((1, 2), np.uint64)
    vals = np.ascontiguousarray(vals) if n else np.zeros(1, np.int64)
    L.decode(keys.ctypes.data, vals.ctypes.data, n, n_windows, threads, sp_w.ctypes.data, sp_idx.ctypes.data,
             sp_val.ctypes.data, begin.ctypes.data, fin_idx.ctypes.data, fin_cnt.ctypes.data, counts.ctypes.data)
    a, b = int(counts[0]), int(counts[1])
    return sp_w[:a], sp_idx[:a], sp_val[:a], begin, fin_idx[:b], fin_cnt[:b]


@pytest.mark.parametrize("n,threads,dup", [(0, 8, 0.0), (1, 8, 0.0), (500, 8, 0.3), (70_000, 1, 0.2),
                                           (200_000, 8, 0.2), (200_000, 64, 0.5), (300_000, 3, 0.0)])
def test_decode_sorted_bins_equals_sequential_restatement(decoder, n, threads, dup):
    rng = np.random.default_rng(n + threads)
    n_windows = 37
    keys, vals = _random_bins(rng, n, n_windows, dup)
    w, idx, val, begin, fi, fc = _decode(decoder, keys, vals, n_windows, threads)
    rw, ridx, rval, rbegin, rfi, rfc = _reference(keys, vals, n_windows)
    assert w.tolist() == rw
    assert [tuple(x) for x in idx.tolist()] == ridx
    assert val.tolist() == rval
    assert begin.tolist() == rbegin
    assert [tuple(x) for x in fi.tolist()] == rfi
    assert fc.tolist() == rfc


@pytest.mark.parametrize("n,threads", [(0, 8), (5, 8), (65_535, 8), (65_536, 7), (1_000_003, 16), (200_000, 0)])
def test_parallel_ranges_cover_every_index_once(decoder, n, threads):
    hits = np.zeros(max(1, n), np.uint32)
    decoder.ranges(n, threads, hits.ctypes.data)
    assert np.all(hits[:n] == 1)


@pytest.mark.parametrize("T,bad", [(1, 0), (4, 0), (4, 3), (8, 5), (64, 63)])
def test_parallel_for_rethrows_after_joining(decoder, T, bad):
    """A chunk that throws (a failed allocation, say) neither terminates the process nor leaves
    threads unjoined: every chunk still runs once and the exception reaches the caller."""
    hits = np.zeros(T, np.uint32)
    assert decoder.throwing(T, bad, hits.ctypes.data) == 1
    assert np.array_equal(hits, np.ones(T, np.uint32))
