"""More than 20 non-internal nodes (the reference stops at 20, src/main.cpp:142-146): 128-bit
non-internal indices and sparse window bins in a device hash table, against the oracle's sparse
path, which is itself pinned against its dense path on the reference models."""
import numpy as np
import pytest

import maboss.gpu_b200 as mb
from conftest import model_text
from maboss.gpu_b200 import synth
from oracle.oracle import OracleModel

P_ABS, P_REL, H_REL = 1e-5, 1e-4, 1e-4


def _c2_literal(**kw):
    """The 100-node network with 20 % internal nodes (~80 non-internal)."""
    return synth.c2(**kw)


def _index(pairs):
    pairs = np.asarray(pairs, np.uint64).reshape(-1, 2)
    return [int(a) | (int(b) << 64) for a, b in pairs]


@pytest.mark.parametrize("name", ["sizek", "cellcycle"])
def test_oracle_sparse_path_equals_its_dense_path(name):
    o = OracleModel(*model_text(name))
    d, s = o.run(n=400), o.run(n=400, sparse=True)
    sp = s["sparse"]
    dense = d["cnt"] if o.discrete else d["occ"]
    rebuilt = np.zeros_like(dense, dtype=np.int64)
    rebuilt[sp["windows"], np.array(_index(sp["states"]), np.int64)] = sp["raw"]
    assert np.array_equal(rebuilt, dense)
    fin = np.zeros_like(d["final"], dtype=np.int64)
    fin[np.array(_index(sp["final_states"]), np.int64)] = sp["final_counts"]
    assert np.array_equal(fin, d["final"])
    assert np.array_equal(s["h"], d["h"]) and s["transitions"] == d["transitions"]


def test_oracle_wide_model_probabilities_add_up():
    o = OracleModel(*_c2_literal())
    assert o.k > 64
    r = o.run(n=60)
    sp = r["sparse"]
    assert max(_index(sp["states"])) >= 1 << 64 or o.k <= 64
    sums = np.bincount(sp["windows"], weights=sp["probs"], minlength=o.windows)
    assert np.allclose(sums, 1.0, atol=1e-6)
    assert int(np.sum(sp["final_counts"])) == 60


def test_generated_code_uses_a_wide_index():
    code = mb.Model(*_c2_literal()).generate_code()
    assert "#define MBG_WIDE_INDEX 1" in code and "unsigned __int128 get_non_internal_index" in code
    narrow = mb.Model(*synth.c2(noninternal=20)).generate_code()
    assert "MBG_WIDE_INDEX" not in narrow


def test_jit_of_a_wide_model_compiles_every_family():
    import ctypes as C
    code = mb.Model(*_c2_literal()).generate_code().encode()
    size, log = C.c_size_t(), C.create_string_buffer(1 << 16)
    status = mb.lib().mb_jit_check(code, C.byref(size), log, 1 << 16)
    assert status == 0, log.value.decode()[-2000:]
    assert size.value > 0


def _compare_sparse(res, ref, exact_values):
    a, b = res.sparse(), ref["sparse"]
    assert a["overflow"] == 0
    assert np.array_equal(a["windows"], b["windows"])
    assert _index(a["states"]) == _index(b["states"])
    if exact_values:
        assert np.array_equal(a["raw"], b["raw"])
    else:
        assert np.all(np.abs(a["probs"] - b["probs"]) <= P_ABS + P_REL * b["probs"])
    assert _index(a["final_states"]) == _index(b["final_states"])
    assert np.array_equal(a["final_counts"].astype(np.int64), b["final_counts"].astype(np.int64))
    th, th2 = res.window_entropy, ref["th"]
    assert np.all(np.abs(th - th2) <= 1e-6 + H_REL * np.abs(th2))


@pytest.mark.gpu
@pytest.mark.parametrize("kw,n,mode", [({}, 300, "exact"), ({}, 300, "fast"),
                                       (dict(noninternal=30, discrete=True), 1_000, "exact"),
                                       (dict(noninternal=24), 1_000, "exact")])
def test_wide_model_matches_oracle(gpu, kw, n, mode):
    bnd, cfg = _c2_literal(**kw)
    model = mb.Model(bnd, cfg)
    res = gpu.compile(model).run(mode=mode, sample_count=n)
    assert res.is_sparse
    raw = res.raw()
    o = OracleModel(bnd, cfg)
    ref = o.run(n=n, mode=0 if mode == "exact" else 1, occ_exp=raw["occ_exp"], ent_exp=raw["ent_exp"])
    assert res.transitions == ref["transitions"]
    _compare_sparse(res, ref, exact_values=o.discrete)
    assert [(s.tolist(), c) for s, c in res.fixed] == \
        [(s.tolist(), int(c)) for s, c in zip(ref["fixed_states"], ref["fixed_counts"])]


@pytest.mark.gpu
def test_wide_epoch_modes_equal_fused_exact(gpu, tmp_path):
    bnd, cfg = _c2_literal()
    model = mb.Model(bnd, cfg)
    mod = gpu.compile(model)
    a = mod.run(mode="exact", sample_count=500)
    for mode in ("epoch", "epoch_dense"):
        b = mod.run(mode=mode, sample_count=500, batch_limit=200)
        sa, sb = a.sparse(), b.sparse()
        for k in ("windows", "raw", "final_counts"):
            assert np.array_equal(sa[k], sb[k]), (mode, k)
        assert _index(sa["states"]) == _index(sb["states"]) and a.transitions == b.transitions
        assert np.array_equal(a.raw()["h"], b.raw()["h"])
    # output files and the merge of shards
    a.write_csv(model, str(tmp_path / "w"))
    lines = open(str(tmp_path / "w_probtraj.csv")).read().splitlines()
    assert len(lines) == a.dims.windows + 1 and "State" in lines[0]
    parts = [mod.run(mode="exact", sample_count=c, first_traj=f, stats_trajectories=500)
             for f, c in ((0, 200), (200, 300))]
    m = mb.merge_results(parts)
    sm, sa = m.sparse(), a.sparse()
    assert np.array_equal(sm["raw"], sa["raw"]) and _index(sm["states"]) == _index(sa["states"])
    assert m.visualize(model) == a.visualize(model)


@pytest.mark.gpu
def test_full_bin_table_is_reported_not_fatal(gpu):
    mod = gpu.compile(mb.Model(*_c2_literal()))
    res = mod.run(mode="fast", sample_count=200, bin_capacity_log2=5)
    assert res.sparse()["overflow"] > 0
    assert res.transitions > 0
