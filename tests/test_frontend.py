"""CPU tests of the engine's host side: parser, code generator, C ABI surface, CLI, generators."""
import ctypes as C
import os
import re
import subprocess

import numpy as np
import pytest

import maboss.gpu_b200 as mb
from conftest import ROOT, model_files, model_text
from maboss.gpu_b200 import synth
from oracle.oracle import OracleModel

HEADER = os.path.join(ROOT, "include", "maboss_b200.h")
CLI = os.path.join(ROOT, "maboss", "gpu_b200", "MaBoSS.GPU")


def test_library_exports_every_declared_symbol():
    decl = open(HEADER).read()
    names = set(re.findall(r"^\s*(?:mb_status|const char\*|size_t)\s+(mb_\w+)\s*\(", decl, re.M))
    assert len(names) > 40
    L = C.CDLL(mb._lib.LIB_PATH)
    missing = [n for n in sorted(names) if not hasattr(L, n)]
    assert not missing, missing
    nm = subprocess.run(["nm", "-D", "--defined-only", mb._lib.LIB_PATH], capture_output=True, text=True).stdout
    exported = set(re.findall(r" T (mb_\w+)", nm))
    assert names <= exported


def test_no_device_is_an_error_not_a_crash():
    if os.path.exists("/dev/nvidia0"):
        pytest.skip("a GPU is present")
    with pytest.raises(mb.EngineError) as e:
        mb.Context(0)
    assert e.value.status == 6  # MB_ERR_NO_DEVICE


@pytest.mark.parametrize("name", ["cellcycle", "sizek", "metastasis", "Montagud2022_Prostate_Cancer"])
def test_parser_agrees_with_oracle_parser(name):
    bnd, cfg = model_files(name)
    m = mb.Model.from_files(bnd, cfg)
    o = OracleModel.from_files(bnd, cfg)
    assert m.num_nodes == o.nodes
    assert m.noninternal_nodes == o.noninternal
    assert m.constant("sample_count") == o.sample_count
    assert m.constant("max_time") == np.float32(o.max_time)
    assert m.constant("time_tick") == np.float32(o.tick)
    assert bool(m.constant("discrete_time")) == o.discrete


def test_generated_code_matches_reference_form():
    """Emitted text for cellcycle equals the reference generator's (README example of the reference)."""
    m = mb.Model(*model_text("cellcycle"))
    code = m.generate_code()
    assert "constexpr int state_size = 10;\nconstexpr int state_words = 1;\nconstexpr bool discrete_time = 1;\n" \
           "constexpr float max_time = 5;\nconstexpr float time_tick = 0.2;\n" in code
    assert ("__device__ float CycD_rate(const state_word_t* __restrict__ state) \n{\n"
            "    const bool is_up = ((state[0] & 1u) != 0);\n    const bool logic = ((state[0] & 1u) != 0);\n"
            "    return is_up == logic ? 0 : 10;\n}\n") in code
    assert ("__device__ float CycE_rate(const state_word_t* __restrict__ state) \n{\n"
            "    const bool is_up = ((state[0] & 2u) != 0);\n"
            "    const bool logic = !((state[0] & 16u) != 0) & ((state[0] & 32u) != 0);\n"
            "    return is_up == logic ? 0 : (is_up ? 10 : 1);\n}\n") in code
    assert "    tmp = CycD_rate(state);\n    transition_rates[0] = tmp;\n    sum += tmp;\n" in code
    assert "((state[0] & 1u)) | ((state[0] & 2u)) | ((state[0] & 4u)) | ((state[0] & 8u))" in code


BND = """
node A { logic = B; rate_up = @logic ? $k : 0; rate_down = @logic ? 0 : 2.5; }
Node B { logic = A XOR C; rate_up = @logic ? 1 : 0; rate_down = @logic ? 0 : 1; }
NODE C { logic = !A and B; rate_up = A ? 3 : 1; rate_down = 0.5 * $k; }
"""
CFG = """
$k = 1.25;
A.istate = 0.25;
[B].istate = 1 [1], 3 [0];
C.is_internal = TRUE;
C.is_internal = FALSE; // first attribute wins
max_time = 2 * 3; time_tick = .5; sample_count = 1e3;
"""


def test_parser_semantics():
    m = mb.Model(BND, CFG)
    assert m.node_names == ["A", "B", "C"]
    assert m.node_info(0) == (0.25, False)
    assert m.node_info(1)[0] == pytest.approx(0.25)  # 1 / (1 + 3)
    assert m.node_info(2) == (0.5, True)
    assert m.noninternal_nodes == [0, 1]
    assert m.constant("max_time") == 6 and m.constant("time_tick") == 0.5
    assert m.constant("sample_count") == 1000
    assert m.constant("discrete_time") == 0 and m.constant("seed_pseudorandom") == 0  # defaults
    assert m.constant("not_there") == 0
    assert m.variables == {"$k": 1.25}
    code = m.generate_code()
    assert "((state[0] & 1u) != 0) ^ ((state[0] & 4u) != 0)" in code  # XOR
    assert "return ((state[0] & 4u) != 0) ?\n          (0.5 * 1.25)\n        : (((state[0] & 1u) != 0) ? 3 : 1);" in code


def test_variable_override_rebakes_literals():
    m = mb.Model(BND, CFG)
    m.set_variable("$k", 3.0)
    assert "return is_up == logic ? 0 : (is_up ? 2.5 : 3);" in m.generate_code()


def test_oracle_rates_follow_generated_semantics():
    o = OracleModel(BND, CFG)
    # state A=0, B=1, C=0: A unstable (logic=B=1) up rate $k
    assert o.rate(0, [0b010]) == pytest.approx(1.25)
    # C (general form) with C=0 and A=0 -> rate_up = A ? 3 : 1 = 1; with C=1 -> 0.5 * 1.25
    assert o.rate(2, [0b000]) == 1.0
    assert o.rate(2, [0b100]) == pytest.approx(0.625)


@pytest.mark.parametrize("bnd,cfg,needle", [
    ("node A { logic = A; rate_down = 1; }", "", "rate_up"),
    ("node A { logic = A; rate_up = 1; rate_down = 1; } node A { logic = A; rate_up = 1; rate_down = 1; }", "",
     "already exists"),
    ("node A { logic = A; rate_up = 1; rate_down = 1; }", "B.istate = 1;", "Unknown node B"),
    ("node A { logic = A # B; rate_up = 1; rate_down = 1; }", "", "invalid character"),
    ("nod A { logic = A; rate_up = 1; rate_down = 1; }", "", "expected 'node'"),
    ("node A { logic = A; rate_up = 1; rate_down = 1 }", "", "syntax error"),
    ("node A { logic = A; rate_up = 1; rate_down = 1; }", "max_time = $undefined;", "unknown variable"),
])
def test_parse_errors_are_reported(bnd, cfg, needle):
    with pytest.raises(mb.EngineError) as e:
        mb.Model(bnd, cfg)
    assert e.value.status == 2  # MB_ERR_PARSE
    assert needle in str(e.value)


def test_jit_compiles_for_sm100a_without_a_device():
    code = mb.Model(*model_text("cellcycle")).generate_code()
    n = C.c_size_t()
    log = C.create_string_buffer(1 << 16)
    st = mb.lib().mb_jit_check(code.encode(), C.byref(n), log, 1 << 16)
    assert st == 0, mb.lib().mb_last_error()
    assert n.value > 10_000


def test_jit_reports_compile_errors():
    n = C.c_size_t()
    st = mb.lib().mb_jit_check(b"constexpr int state_size = 1;\nconstexpr int state_words = 1;\nsyntax error here",
                               C.byref(n), None, 0)
    assert st == 3  # MB_ERR_COMPILE
    assert b"error" in mb.lib().mb_last_error()


def test_cli_emits_code_and_rejects_bad_usage():
    b, c = model_files("cellcycle")
    out = subprocess.run([CLI, "--emit-code", b, c], capture_output=True, text=True)
    assert out.returncode == 0 and "CycD_rate" in out.stdout
    bad = subprocess.run([CLI, b], capture_output=True, text=True)
    assert bad.returncode == 1 and "Usage" in bad.stdout


@pytest.mark.parametrize("gen,kw,nodes,k", [
    (synth.c1, {}, 10, 10), (synth.c2, dict(noninternal=20), 100, 20), (synth.c3, {}, 1000, 10),
    (synth.c4, {}, 50, 8), (synth.c5_base, dict(index=3), None, 8)])
def test_synthetic_generators_are_seeded_and_parse(gen, kw, nodes, k):
    a = gen(**kw)
    assert a == gen(**kw)
    m = mb.Model(*a)
    o = OracleModel(*a)
    if nodes is not None:
        assert m.num_nodes == nodes
    assert len(m.noninternal_nodes) == k == o.k
    assert m.noninternal_nodes == o.noninternal


def test_cfg_overrides_are_opt_in():
    """A node attribute given again in the .cfg: the reference keeps the .bnd's first definition
    (driver.cpp:65-77, parse_types.cpp:6-13), so by default the generated rate is the .bnd's;
    mb_model_apply_cfg_overrides (CLI --cfg-overrides) makes the .cfg's win."""
    bnd = ("node A { logic = !B; rate_up = @logic ? 2 : 0; rate_down = @logic ? 0 : 3; }\n"
           "node B { logic = A; rate_up = @logic ? 1 : 0; rate_down = @logic ? 0 : 1; }\n")
    cfg = "A.rate_up = @logic ? 7.5 : 0; B.is_internal = 1; B.is_internal = 0; max_time = 1; time_tick = 0.5;\n"
    m = mb.Model(bnd, cfg)
    code = m.generate_code()
    assert "(is_up ? 3 : 2)" in code and "7.5" not in code
    assert m.node_info(1)[1]  # B internal by its first definition
    assert m.noninternal_nodes == [0]
    m.apply_cfg_overrides()
    code = m.generate_code()
    assert "(is_up ? 3 : 7.5)" in code
    assert m.noninternal_nodes == [0, 1]


def test_cfg_overrides_on_the_command_line(tmp_path):
    bnd = "node A { logic = !A; rate_up = @logic ? 2 : 0; rate_down = @logic ? 0 : 3; }\n"
    (tmp_path / "m.bnd").write_text(bnd)
    (tmp_path / "m.cfg").write_text("A.rate_down = @logic ? 0 : 9; max_time = 1; time_tick = 0.5;\n")
    cli = os.path.join(ROOT, "maboss", "gpu_b200", "MaBoSS.GPU")
    a = subprocess.run([cli, "--emit-code", str(tmp_path / "m.bnd"), str(tmp_path / "m.cfg")],
                       capture_output=True, text=True, check=True).stdout
    b = subprocess.run([cli, "--cfg-overrides", "--emit-code", str(tmp_path / "m.bnd"), str(tmp_path / "m.cfg")],
                       capture_output=True, text=True, check=True).stdout
    assert "(is_up ? 3 : 2)" in a and "(is_up ? 9 : 2)" in b


def test_final_states_csv_is_opt_in(tmp_path):
    """mb_result_write_final_csv (CLI --final-csv): the final-state distribution, which the
    reference only prints (final_states.cpp:53-70), as <prefix>_finalprob.csv."""
    names = ["A", "B", "C"]
    res = mb.Result.from_raw(n_nodes=3, n_windows=2, discrete=True, time_tick=1.0, max_time=2.0,
                             noninternal=[0, 2], n_trajectories=10, occ_exp=0, ent_exp=0,
                             cnt=np.zeros(8, np.uint32), h=np.zeros(2, np.int64),
                             final=np.array([4, 0, 1, 5], np.uint32))
    bnd = "".join(f"node {n} {{ logic = {n}; rate_up = @logic ? 1 : 0; rate_down = @logic ? 0 : 1; }}\n"
                  for n in names)
    model = mb.Model(bnd, "B.is_internal = 1; max_time = 2; time_tick = 1; discrete_time = 1;")
    res.write_final_csv(model, str(tmp_path / "out"))
    text = (tmp_path / "out_finalprob.csv").read_text().splitlines()
    assert text == ["Final States (3)", "Proba\tState", "0.4\t<nil>", "0.1\tC", "0.5\tA -- C"]
