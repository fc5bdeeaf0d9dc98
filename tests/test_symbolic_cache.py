"""The symbolic-analysis cache of karam_problem_create: an identical netlist
reuses the analysis (same tables, one build), any change of content builds a
new one, and the fingerprint follows the content."""
import numpy as np

from karam_b200 import circuits


def test_identical_netlist_reuses_the_analysis(product):
    product.symbolic_cache_clear()
    a = product.Problem(None, circuits.grid_circuit(12))
    assert product.symbolic_cache_info() == (1, 0, 1)
    b = product.Problem(None, circuits.grid_circuit(12))
    assert product.symbolic_cache_info() == (1, 1, 1)
    for q in ("pattern", "filled_pattern", "stamp_map"):
        x, y = getattr(a, q)(), getattr(b, q)()
        x, y = (x, y) if isinstance(x, tuple) else ((x,), (y,))
        for xi, yi in zip(x, y):
            assert np.array_equal(xi, yi), q
    assert a.info == b.info


def test_changed_content_is_a_new_analysis(product):
    product.symbolic_cache_clear()
    base = circuits.grid_circuit(10)
    other = circuits.grid_circuit(10)
    other.res[0] = (other.res[0][0], other.res[0][1], other.res[0][2] * 1.0000001)
    other._struct = None
    assert product.netlist_hash(base) == product.netlist_hash(circuits.grid_circuit(10))
    assert product.netlist_hash(base) != product.netlist_hash(other)
    product.Problem(None, base)
    product.Problem(None, other)
    assert product.symbolic_cache_info() == (2, 0, 2)


def test_spice_and_builder_share_an_analysis(product):
    """A SPICE text equal to a builder's netlist, content for content, hits the
    builder's cached analysis."""
    product.symbolic_cache_clear()
    text = "\n".join(["divider", "V1 a 0 1", "R1 a b 1e3", "R2 b 0 2e3", ".end"])
    nl = circuits.Netlist()
    nl.vsource(1, 0, 1.0)
    nl.resistor(1, 2, 1e3)
    nl.resistor(2, 0, 2e3)
    sp = product.parse_spice(text)
    assert product.netlist_hash(sp) == product.netlist_hash(nl)
    product.Problem(None, nl)
    product.Problem(None, sp)
    assert product.symbolic_cache_info() == (1, 1, 1)
