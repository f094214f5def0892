"""The time loop of SWESim_run_simulation captured in a CUDA graph (src/swe.cpp:183-223 as one graph
launch): the replayed graph gives the bits of the directly launched sequence (HHG_GRAPH=0), across
runs that continue the state, resets, restarts and a changed setup."""
import os

import numpy as np
import pytest

from conftest import load_golden

pytestmark = pytest.mark.gpu


def runs(param, precision, graph: bool):
    from pySWE import pyswe

    if graph:
        os.environ.pop("HHG_GRAPH", None)
    else:
        os.environ["HHG_GRAPH"] = "0"
    try:
        s = pyswe.SWE(pyswe.Settings(dict(param)), precision=precision, solver=param.get("solver", "rspace"))
        out = []
        s.run_simulation()                      # first run: captures the graph
        out.append(np.stack(s.get_current()[1:]))
        s.run_simulation()                      # continues from the propagated state: replays it
        out.append(np.array(s.get_rho_k()))
        s.reset()
        s.run_simulation()
        out.append(np.stack(s.get_current()[1:]))
        s.restart()                             # a new setup: the graph is captured again
        s.run_simulation()
        out.append(np.stack(s.get_current()[1:]))
        launches = s.last_launches()
        s.delete()
    finally:
        os.environ.pop("HHG_GRAPH", None)
    return out, launches


@pytest.mark.parametrize("name,precision", [("haldane_12_pol", "fp64"), ("c1", "fp64"), ("tmd11_10", "mixed"),
                                            ("tmd11_10", "fp64"), ("ks_tmd11_10", "mixed")])
def test_graph_replay_is_bitwise_the_direct_launch(name, precision):
    _, param, _, _ = load_golden(name)
    if name == "c1":
        param = dict(param, tmax=4.4)  # 200 steps of the 200 x 200 grid (column-tile kernel)
    g, n_g = runs(param, precision, True)
    d, n_d = runs(param, precision, False)
    assert n_g == n_d
    for a, b in zip(g, d):
        assert np.array_equal(a, b)
