"""The product's Min-Fill (sparse adjacency, fill counts updated from each
elimination's new edges) against the oracle's restatement of the reference's
loop, which recounts every remaining vertex at every step
(treewidth_analyzer.cpp:72-128), on seeded random netlists: resistor graphs of
random density with parallel duplicates, MOSFET four-terminal cliques,
diodes, capacitors and voltage sources (whose branch ids can collide with the
node count). Orderings, treewidths and filled patterns must be equal. CPU
only."""
import numpy as np
import pytest

from karam_b200 import _abi as A
from karam_b200 import circuits


def random_netlist(seed):
    rng = np.random.default_rng(seed)
    n = int(rng.integers(6, 90))
    nl = circuits.Netlist()
    nmod = nl.model("NMOS", A.MODEL_NMOS, 1.1e-4, 0.7, 0.04)
    nl.vsource(1, 0, 1.8)
    for _ in range(int(rng.integers(0, 3))):
        a = int(rng.integers(1, n + 1))
        nl.vsource(a, 0 if rng.random() < 0.7 else int(rng.integers(1, n + 1)), 0.5)
    p_edge = float(rng.uniform(1.2, 4.0)) / n
    for a in range(1, n + 1):
        for b in range(a + 1, n + 1):
            if rng.random() < p_edge:
                nl.resistor(a, b, float(rng.uniform(10.0, 1e4)))
                if rng.random() < 0.05:
                    nl.resistor(a, b, 1e3)  # a parallel duplicate
        if rng.random() < 0.3:
            nl.resistor(a, 0, 1e5)
        if rng.random() < 0.2:
            nl.capacitor(a, 0 if rng.random() < 0.5 else int(rng.integers(1, n + 1)), 1e-12)
    for _ in range(int(rng.integers(0, n // 4 + 1))):
        d, g, s = (int(x) for x in rng.integers(0, n + 1, size=3))
        nl.mosfet(max(d, 1), g, s, 0, nmod, 2e-6, 1.8e-7)
    for _ in range(int(rng.integers(0, 4))):
        nl.diode(int(rng.integers(1, n + 1)), int(rng.integers(0, n + 1)))
    for a in range(1, nl.n_nodes + 1):  # no node left without an element
        nl.resistor(a, 0, 1e6)
    return nl


@pytest.mark.parametrize("seed", range(40))
def test_min_fill_equals_rescanning_restatement(product, port, seed):
    nl = random_netlist(1000 + seed)
    prob = product.Problem(None, nl)
    raw, perm, tw = prob.ordering()
    raw_o, perm_o, tw_o = port.ordering(nl)
    assert np.array_equal(raw, raw_o) and np.array_equal(perm, perm_o) and tw == tw_o
    sym = port.symbolic(nl)
    frp, fcol = prob.filled_pattern()
    assert np.array_equal(frp, sym["row_ptr"]) and np.array_equal(fcol, sym["col"])
    prob.close()
