import os
import subprocess
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)

GOLDEN = os.path.join(ROOT, "tests", "golden")
MODELS = os.path.join(GOLDEN, "models")


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a B200 (sm_100) GPU")


def model_files(name: str) -> tuple[str, str]:
    return os.path.join(MODELS, f"{name}.bnd"), os.path.join(MODELS, f"{name}.cfg")


def model_text(name: str) -> tuple[str, str]:
    b, c = model_files(name)
    with open(b) as f, open(c) as g:
        return f.read(), g.read()


@pytest.fixture(scope="session", autouse=True)
def _built():
    """Build the engine library and the oracle in place once per session."""
    subprocess.run(["make", "-s", "-j8", "-C", os.path.join(ROOT, "maboss", "gpu_b200", "csrc")], check=True)
    subprocess.run(["make", "-s", "-C", os.path.join(ROOT, "oracle")], check=True)


@pytest.fixture(scope="session")
def gpu():
    import maboss.gpu_b200 as mb
    return mb.Context(0)


def pooled_z(p: np.ndarray, n1: int, q: np.ndarray, n2: int) -> np.ndarray:
    """|p - q| in units of the pooled binomial standard error of two independent estimates."""
    pooled = (p * n1 + q * n2) / (n1 + n2)
    var = pooled * (1.0 - pooled) * (1.0 / n1 + 1.0 / n2)
    z = np.zeros_like(p)
    nz = var > 0
    z[nz] = np.abs(p[nz] - q[nz]) / np.sqrt(var[nz])
    return z


def assert_statistically_equal(p: np.ndarray, n1: int, q: np.ndarray, n2: int, alpha: float = 1e-3) -> None:
    """Two Monte-Carlo estimates of the same probabilities (per window and state) agree.

    Each compared bin is a 4-sigma-style binomial test with the pooled standard error; over M bins
    the family-wise threshold is Bonferroni: P(max |z| > z_crit) <= alpha. The sum of z^2 over
    the populated bins must not exceed the chi-square(M) quantile 1 - alpha (time-averaged
    window probabilities have at most binomial variance, so the test is conservative; a systematic
    difference inflates every bin's z)."""
    from statistics import NormalDist

    from scipy.stats import chi2

    z = pooled_z(np.asarray(p, np.float64).ravel(), n1, np.asarray(q, np.float64).ravel(), n2)
    populated = (np.asarray(p).ravel() > 0) | (np.asarray(q).ravel() > 0)
    m = max(1, int(populated.sum()))
    z_crit = max(4.0, NormalDist().inv_cdf(1.0 - alpha / (2.0 * m)))
    assert z.max() < z_crit, (z.max(), z_crit, int(z.argmax()))
    s2 = float((z[populated] ** 2).sum())
    assert chi2.sf(s2, m) > alpha, (s2 / m, m)


def force_node(bnd: str, cfg: str, node: str, on: bool) -> tuple[str, str]:
    """The model text with `node` forced, as a mutant: both rates 0 and initial state 1 (on) or 0 (off)."""
    import re

    pat = re.compile(r"(node\s+" + node + r"\s*\{)(.*?)(\})", re.S | re.I)
    m = pat.search(bnd)
    body = re.sub(r"rate_up\s*=[^;]*;", "rate_up = @logic ? 0 : 0;", m.group(2))
    body = re.sub(r"rate_down\s*=[^;]*;", "rate_down = @logic ? 0 : 0;", body)
    return bnd[:m.start(2)] + body + bnd[m.end(2):], cfg + f"\n{node}.istate = {1 if on else 0};\n"
