"""The reference build (oracle/_ref/ref_run, built from the reference's own sources by
oracle/refbuild/Makefile) on the CPU: its generator, fed by the parser of this build's reference
recipe, and this engine's generator emit the same model code; its harness refuses the inputs for
which the reference's own arithmetic leaves its buffers; its dump reader.

The reference generator (generator.cpp:84-235, expressions.cpp:83-230) prints every `<node>_rate`
function, `compute_transition_rates`, `compute_transition_entropy` and `get_non_internal_index`
from the parsed expression trees; this engine's code generator reproduces that text so that the
compiled rate arithmetic is identical. Equal text for the four example models, the synthetic
benchmark networks and random models pins (a) the engine's parser and code generator against the
reference's, and (b) the recipe's parser stand-in (oracle/refbuild/parser_shim.cpp) against the
engine's independent parser. No GPU is used: `--emit-code` exits, and refused inputs stop, before
any CUDA call.
"""
import os
import re
import subprocess

import numpy as np
import pytest

from conftest import ROOT, model_files
from maboss.gpu_b200 import synth
from test_codegen_host import _random_model

REF_RUN = os.path.join(ROOT, "oracle", "_ref", "ref_run")
STUBS = os.path.join(ROOT, "oracle", "_ref", "stubs")
OURS = os.path.join(ROOT, "maboss", "gpu_b200", "MaBoSS.GPU")

pytestmark = pytest.mark.skipif(not os.path.exists(REF_RUN),
                                reason="reference build absent (oracle/refbuild needs the reference sources)")


def _run_ref_cpu(args):
    env = dict(os.environ)
    env["LD_LIBRARY_PATH"] = STUBS + (":" + env["LD_LIBRARY_PATH"] if env.get("LD_LIBRARY_PATH") else "")
    return subprocess.run([REF_RUN] + args, capture_output=True, text=True, env=env)


def _emit_ref(bnd, cfg):
    return _run_ref_cpu(["--emit-code", bnd, cfg])


def _emit_ours(bnd, cfg):
    return subprocess.run([OURS, "--emit-code", bnd, cfg], capture_output=True, text=True)


_FUNC = re.compile(r"^__device__ (?:float|uint32_t) (\w+)\([^)]*\)\s*\n\{\n.*?^\}\n", re.S | re.M)
_CONST = re.compile(r"^constexpr \w+ (?:state_size|state_words|discrete_time|max_time|time_tick) = [^;]*;$", re.M)


def _blocks(code: str) -> dict:
    out = {m.group(1): m.group(0) for m in _FUNC.finditer(code)}
    out["constexpr"] = "\n".join(_CONST.findall(code))
    return out


def _compare(bnd_path, cfg_path):
    ref, ours = _emit_ref(bnd_path, cfg_path), _emit_ours(bnd_path, cfg_path)
    assert ref.returncode == 0, ref.stderr
    assert ours.returncode == 0, ours.stderr
    a, b = _blocks(ref.stdout), _blocks(ours.stdout)
    rates = [k for k in a if k.endswith("_rate")]
    assert rates and "compute_transition_rates" in a and "get_non_internal_index" in a
    for k in rates + ["compute_transition_rates", "compute_transition_entropy", "get_non_internal_index",
                      "constexpr"]:
        assert k in b, k
        assert a[k] == b[k], (k, a[k], b[k])
    return len(rates)


def _write(tmp_path, bnd, cfg):
    (tmp_path / "m.bnd").write_text(bnd)
    (tmp_path / "m.cfg").write_text(cfg)
    return str(tmp_path / "m.bnd"), str(tmp_path / "m.cfg")


@pytest.mark.parametrize("name", ["cellcycle", "sizek", "metastasis", "Montagud2022_Prostate_Cancer"])
def test_reference_generator_example_models(name):
    assert _compare(*model_files(name)) > 0


@pytest.mark.parametrize("gen,kw", [(synth.c1, {}), (synth.c2, dict(noninternal=20)), (synth.c3, {}),
                                    (synth.c4, {}), (synth.c5_base, dict(index=3))],
                         ids=["c1", "c2b", "c3", "c4", "c5_base3"])
def test_reference_generator_synthetic_networks(gen, kw, tmp_path):
    assert _compare(*_write(tmp_path, *gen(**kw))) > 0


@pytest.mark.parametrize("seed", range(16))
def test_reference_generator_random_models(seed, tmp_path):
    """Random models (ternaries on node states, integer and 6-digit literals, integer division,
    $variables). The reference generator has no XOR case (expressions.cpp:83-149) and throws when
    it has to print one; a model it refuses must use XOR."""
    bnd, cfg = _random_model(seed)
    paths = _write(tmp_path, bnd, cfg)
    if _emit_ref(*paths).returncode != 0:
        assert "^" in bnd
        return
    assert _compare(*paths) > 0


def test_reference_parser_errors(tmp_path):
    """Syntax errors are reported and fail the parse (return 1), as the bison parser does; an
    unknown node in the .cfg makes the reference's driver throw."""
    good_bnd = "Node A { logic = A; rate_up = @logic ? 1 : 0; rate_down = @logic ? 0 : 1; }\n"
    cases = {
        "bad_char": (good_bnd, "max_time = 5 # 3;\n"),
        "missing_semicolon": (good_bnd, "max_time = 5\n"),
        "not_node": ("Nod A { logic = A; rate_up = 1; rate_down = 1; }\n", "max_time = 5;\n"),
        "istate_brackets": (good_bnd, "[A].istate = 0.3[1], 0.7[0];\n"),
    }
    for name, (bnd, cfg) in cases.items():
        (tmp_path / f"{name}.bnd").write_text(bnd)
        (tmp_path / f"{name}.cfg").write_text(cfg)
        r = _emit_ref(str(tmp_path / f"{name}.bnd"), str(tmp_path / f"{name}.cfg"))
        assert r.returncode == 1 and r.stderr, (name, r.returncode, r.stderr)
    (tmp_path / "u.bnd").write_text(good_bnd)
    (tmp_path / "u.cfg").write_text("B.istate = 1;\n")
    assert _emit_ref(str(tmp_path / "u.bnd"), str(tmp_path / "u.cfg")).returncode != 0


@pytest.mark.parametrize("case", ["c3_1e6", "window_walk", "noninternal_21"])
def test_reference_harness_refuses_out_of_bounds_inputs(case, tmp_path):
    """ref_run checks, before any CUDA call, the sizes for which the reference's own arithmetic
    stays inside its buffers, and exits with code 3 otherwise (harness.cu: check_inputs):
    * 1000 nodes (32 words) x 1e6 trajectories: batch * 100 * words = 3.2e9 overflows the int
      sizes and indices of simulation_runner.cu:68 and window_average_small.cu:71;
    * max_time 1, tick 0.01: 100 * 0.01f rounds below 1.0f, so the window walk of
      window_average_small.cu:75-92 would reach window 100 of 100;
    * 21 non-internal nodes (main.cpp:142)."""
    if case == "c3_1e6":
        bnd, cfg = synth.c3()
    elif case == "window_walk":
        bnd, cfg = synth.c1()
        cfg = cfg.replace("max_time = 5;", "max_time = 1;").replace("time_tick = 0.2;", "time_tick = 0.01;")
    else:
        bnd, cfg = synth.c2(noninternal=21)
    r = _run_ref_cpu(list(_write(tmp_path, bnd, cfg)))
    assert r.returncode == 3, (r.returncode, r.stdout, r.stderr)
    assert "refused" in r.stdout


def test_reference_dump_reader(tmp_path):
    """oracle/reference.read_dump against a dump written by hand in harness.cu's format."""
    from oracle.reference import read_dump

    T, S, W = 3, 4, 2
    win = np.arange(T * S, dtype=np.float32)
    h = np.array([1.0, 2.0, 3.0], np.float32)
    fin = np.array([5, 0, 7, 8], np.int32)
    fst = np.array([[1, 2], [3, 4]], np.uint32)
    fc = np.array([9, 10], np.int32)
    with open(tmp_path / "d.bin", "wb") as f:
        f.write(b"MBREF001")
        f.write(np.array([20, 40, W, 2, T, S, 0, 1234, 2], np.int64).tobytes())
        f.write(np.array([1.5, 0.5], np.float32).tobytes())
        for a in (win, h, fin, fst, fc):
            f.write(a.tobytes())
    d = read_dump(str(tmp_path / "d.bin"))
    assert d["transitions"] == 1234 and d["windows"] == T and d["bins"] == S and not d["discrete"]
    assert np.array_equal(d["window"].ravel(), win) and np.array_equal(d["final"], fin)
    assert np.array_equal(d["fixed_states"], fst) and np.array_equal(d["fixed_counts"], fc)
    assert np.allclose(d["probs"].ravel(), win / np.float32(20 * 0.5))
    assert np.allclose(d["th"], h / 20 / 0.5)
