"""Mutant semantics on the CPU: a node forced on or off (both rates 0, initial state 1 or 0) keeps
its value in every window and final state of the oracle's simulation, and the forced model stays on
the incremental kernels' table-driven path. The GPU tests (tests/test_gpu_batch.py) check that
mb_batch_add_mutant equals the fast mode of exactly this edited model text."""
import numpy as np
import pytest

import maboss.gpu_b200 as mb
from conftest import force_node, model_text
from oracle.oracle import OracleModel


@pytest.mark.parametrize("name,node,on", [("cellcycle", "CycE", True), ("cellcycle", "CycE", False),
                                          ("cellcycle", "CycA", True)])
def test_forced_node_holds_its_value(name, node, on):
    bnd, cfg = force_node(*model_text(name), node, on)
    model = mb.Model(bnd, cfg)
    code = model.generate_code()
    assert "#define MBG_INCREMENTAL 1" in code
    i = model.node_names.index(node)
    assert model.node_info(i)[0] == (1.0 if on else 0.0)
    o = OracleModel(bnd, cfg)
    assert i in o.noninternal
    k = o.noninternal.index(i)
    n = 2000
    r = o.run(n=n, mode=1, seed=5)
    probs = r["probs"]
    states = np.arange(probs.shape[1])
    with_node = ((states >> k) & 1).astype(bool)
    mass = probs.sum(axis=1)
    held = probs[:, with_node if on else ~with_node].sum(axis=1)
    assert np.allclose(held[mass > 0], mass[mass > 0], atol=1e-9)
    final = np.asarray(r["final"])
    other = final[~with_node if on else with_node]
    assert other.sum() == 0 and final.sum() == n
