"""The C++ mirror of the reference's host classes (maboss/gpu_b200/host: driver, generator,
kernel_compiler, simulation_runner, stats_composite and the three statistics plugins), exercised
by tests/cpp/mirror_test.cpp and by the MaBoSS.GPU command line built on it."""
import os
import subprocess

import pytest

import maboss.gpu_b200 as mb
from conftest import ROOT, model_files, model_text

PKG = os.path.join(ROOT, "maboss", "gpu_b200")
CLI = os.path.join(PKG, "MaBoSS.GPU")


@pytest.fixture(scope="module")
def mirror_test(tmp_path_factory):
    exe = str(tmp_path_factory.mktemp("mirror") / "mirror_test")
    subprocess.run(["g++", "-O1", "-std=c++17", "-Wall", "-I" + os.path.join(ROOT, "include"),
                    "-I" + os.path.join(PKG, "host"), os.path.join(ROOT, "tests", "cpp", "mirror_test.cpp"),
                    "-L" + PKG, "-lmaboss_host", "-lmaboss_b200", "-Wl,-rpath," + PKG, "-o", exe], check=True)
    return exe


@pytest.mark.parametrize("name", ["sizek", "Montagud2022_Prostate_Cancer"])
def test_driver_members_and_generator_edits(mirror_test, tmp_path, name):
    """driver exposes nodes/constants/variables like src/parser/driver.h:41-43, and edits of those
    members reach generator::generate_code (the reference generates from the same members)."""
    bnd, cfg = model_files(name)
    out = tmp_path / "gen.cu"
    p = subprocess.run([mirror_test, "frontend", bnd, cfg, str(out)], capture_output=True, text=True, check=True)
    lines = p.stdout.splitlines()
    m = mb.Model(*model_text(name))
    assert lines[0] == f"nodes {m.num_nodes}"
    nodes = [l.split() for l in lines if l.startswith("node ")]
    assert [n[1] for n in nodes] == m.node_names
    for (_, _, ist, internal), i in zip(nodes, range(m.num_nodes)):
        p_i, int_i = m.node_info(i)
        assert float(ist) == pytest.approx(p_i, rel=1e-5) and bool(int(internal)) == int_i
    variables = {l.split()[1]: float(l.split()[2]) for l in lines if l.startswith("variable ")}
    assert variables.keys() == m.variables.keys()
    constants = {l.split()[1] for l in lines if l.startswith("constant ")}
    assert {"max_time", "time_tick", "sample_count", "discrete_time", "seed_pseudorandom"} <= constants
    # the same edits through the C ABI give the same code
    if variables:
        first = sorted(m.variables)[0]
        m.set_variable(first, m.variable(first) * 2.0)
    m.set_constant("max_time", 7.5)
    m.set_istate(0, 0.25)
    assert out.read_text() == m.generate_code()


def test_driver_parse_error_returns_one(mirror_test, tmp_path):
    bnd = tmp_path / "bad.bnd"
    bnd.write_text("node A { logic = ; rate_up = 1; rate_down = 1; }\n")
    cfg = tmp_path / "bad.cfg"
    cfg.write_text("")
    p = subprocess.run([mirror_test, "frontend", str(bnd), str(cfg), str(tmp_path / "x")], capture_output=True,
                       text=True)
    assert p.returncode == 2 and p.stderr.strip()


def test_cli_usage_and_limits(tmp_path):
    assert subprocess.run([CLI], capture_output=True).returncode == 1
    names = [f"N{i}" for i in range(21)]
    bnd = "".join(f"node {n} {{ logic = {n}; rate_up = 1; rate_down = 1; }}\n" for n in names)
    (tmp_path / "m.bnd").write_text(bnd)
    (tmp_path / "m.cfg").write_text("max_time = 1;\n")
    p = subprocess.run([CLI, str(tmp_path / "m.bnd"), str(tmp_path / "m.cfg")], capture_output=True, text=True)
    assert p.returncode == 1 and "maximum of 20 non-internal nodes" in p.stderr
    code = subprocess.run([CLI, "--max-noninternal", "64", "--emit-code", str(tmp_path / "m.bnd"),
                           str(tmp_path / "m.cfg")], capture_output=True, text=True)
    assert code.returncode == 0 and "MBG_WIDE_INDEX" in code.stdout


def test_cli_emits_the_generated_code():
    for name in ("cellcycle", "sizek"):
        bnd, cfg = model_files(name)
        out = subprocess.run([CLI, "--emit-code", bnd, cfg], capture_output=True, text=True, check=True).stdout
        assert out == mb.Model(*model_text(name)).generate_code()


def _small_cfg(tmp_path, name, n):
    bnd, cfg = model_files(name)
    text = open(cfg).read() + f"\nsample_count = {n};\n"
    path = tmp_path / f"{name}.cfg"
    path.write_text(text)
    return bnd, str(path)


@pytest.mark.gpu
@pytest.mark.parametrize("name,n", [("metastasis", 1_000), ("cellcycle", 3_000), ("sizek", 1_000)])
def test_user_plugin_buffered_run_equals_fused_run(mirror_test, tmp_path, name, n):
    """A user stats plugin forces the reference's buffered epoch loop (SoA views, partition and
    refill with batches of n/3); it counts exactly the runner's transitions, and the built-in
    statistics of that run equal the fused exact run's byte for byte."""
    bnd, cfg = _small_cfg(tmp_path, name, n)
    prefix = str(tmp_path / "out")
    p = subprocess.run([mirror_test, "plugin", bnd, cfg, str(n), prefix], capture_output=True, text=True)
    assert p.returncode == 0, p.stderr
    f = p.stdout.split()
    trans, counted, fused, epochs_b, epochs_f = int(f[1]), int(f[3]), int(f[5]), int(f[7]), int(f[8])
    assert trans == counted == fused > 0
    assert epochs_f == 1 and epochs_b >= 3
    for suffix in ("_probtraj.csv", "_fp.csv"):
        a = open(prefix + "_buffered" + suffix).read()
        b = open(prefix + "_fused" + suffix).read()
        assert a == b, suffix


@pytest.mark.gpu
@pytest.mark.parametrize("mode", ["exact", "epoch"])
def test_cli_matches_python_binding(tmp_path, gpu, mode):
    """MaBoSS.GPU (mirror classes) writes the same CSV files as a run through the C ABI."""
    n = 2_000
    bnd, cfg = _small_cfg(tmp_path, "sizek", n)
    prefix = str(tmp_path / "cli")
    subprocess.run([CLI, "--mode", mode, "-o", prefix, bnd, cfg], check=True)
    model = mb.Model(*model_text("sizek"))
    res = gpu.compile(model).run(mode="exact", sample_count=n)
    res.write_csv(model, str(tmp_path / "py"))
    for suffix in ("_probtraj.csv", "_fp.csv"):
        assert open(prefix + suffix).read() == open(str(tmp_path / "py") + suffix).read(), suffix
    out = subprocess.run([CLI, "--mode", mode, bnd, cfg], capture_output=True, text=True, check=True).stdout
    assert out == res.visualize(model)
