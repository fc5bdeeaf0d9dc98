"""Host-side behaviour of the C ABI that needs no GPU: calls that need a
device fail with a message on a symbolic-only problem, malformed input is an
error, and the symbolic queries of the level schedule and the tail tables are
consistent."""
import numpy as np
import pytest

from karam_b200 import circuits


def test_device_calls_on_a_symbolic_problem_fail(product):
    prob = product.Problem(None, circuits.grid_circuit(8))
    with pytest.raises(product.KaramError):
        prob.tune_schedule()
    with pytest.raises(product.KaramError):
        prob.solve_dc()


def test_empty_and_degenerate_netlists_are_errors(product):
    with pytest.raises(product.KaramError, match="empty netlist"):
        product.parse_spice("")
    sp = product.parse_spice("title only\n.end\n")
    assert sp.n_nodes == 0
    with pytest.raises(product.KaramError):
        product.Problem(None, sp)


@pytest.mark.parametrize("N", [8, 12, 20])
def test_grid_level_schedule_is_well_formed(product, N):
    """Every pivot in exactly one level, every level's pivots independent, and
    the back substitution reading only columns solved in later levels."""
    prob = product.Problem(None, circuits.grid_circuit(N))
    sch = prob.lu_schedule()
    assert sch is not None
    n = prob.n
    piv = sch["lv_piv"]
    assert sorted(piv.tolist()) == list(range(n))
    level = np.zeros(n, int)
    for lv in range(sch["levels"]):
        level[piv[sch["lv_piv_ptr"][lv]:sch["lv_piv_ptr"][lv + 1]]] = lv
    owner = np.repeat(np.arange(n), np.diff(sch["bs_off"]))
    assert (level[sch["bs_c"]] > level[owner]).all()
    # each L entry belongs to a pivot of its own level
    lp = sch["lv_l_ptr"]
    for lv in range(sch["levels"]):
        assert (level[sch["l_piv"][lp[lv]:lp[lv + 1]]] == lv).all()
