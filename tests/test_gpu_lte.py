"""Transient step control by local truncation error (opts.lte_reltol /
lte_abstol) on the GPU against the oracle, which runs the same documented
rule: a converged sub-step whose accepted point leaves the linear
extrapolation from the two previous accepted points by more than
lte_reltol * max(|x|, |v1|) + lte_abstol at some node is redone with half
the step. The reference's own arbiter (physics/circuitsim.h:57-368) is not a
parity target (it fails its second step as written); the oracle's
restatement of this rule is.

The grids' gate ramp makes the rule reject sub-steps; the decisions (the
number of LTE rejections and of halvings), the NR iteration counts and the
voltages must match the oracle's, and the persistent kernel must give the
per-round graph's results bit for bit."""
import numpy as np
import pytest

from karam_b200 import _abi as A
from karam_b200 import circuits

pytestmark = pytest.mark.gpu

POLISH = dict(polish_max=8)
LTE = dict(lte_rel=1e-3, lte_abs=1e-4)
DT, STEPS, HALV = 40e-12, 20, 6


def scaled_err(v, v_ref):
    return float(np.max(np.abs(v - v_ref) / (1e-9 * np.abs(v_ref) + 1e-12)))


def product_opts(product, prec, **kw):
    return product.options(precision=prec, max_halvings=HALV, lte_reltol=LTE["lte_rel"],
                           lte_abstol=LTE["lte_abs"], **POLISH, **kw)


@pytest.mark.parametrize("N", [8, 12])
def test_lte_step_control_matches_oracle(product, ctx, port, N):
    nl = circuits.grid_circuit(N)
    ni = 2
    inst = circuits.mc_instances(nl, ni)
    prob = product.Problem(ctx, nl, max_instances=ni)
    prob.set_instances(inst)
    opts = product_opts(product, A.PREC_FP64)
    vdc, _ = prob.solve_dc(opts)
    nodes = [2, 3, 10, 30]
    v, st, wave = prob.step_transient(DT, STEPS, A.TRAN_TRAP, opts, wave_nodes=nodes)
    for i in range(ni):
        v_ref, st_ref, w_ref = port.transient(nl, vdc[i], DT, STEPS, A.TRAN_TRAP, inst, i,
                                              wave_nodes=nodes, linear_solver=1,
                                              max_halvings=HALV, **POLISH, **LTE)
        assert st_ref["converged"] == 1 and st[i]["status"] == A.ST_CONVERGED
        assert st_ref["lte_rejects"] > 0
        assert st[i]["lte_rejects"] == st_ref["lte_rejects"]
        assert st[i]["halvings"] == st_ref["halvings"]
        assert scaled_err(v[i], v_ref) <= 1.0
        assert np.max(np.abs(wave[i] - w_ref)) <= 1e-9 * np.max(np.abs(w_ref)) + 1e-12
    # the same job without the rule takes no halvings and fewer iterations
    prob.solve_dc(opts)
    _, st0, _ = prob.step_transient(DT, STEPS, A.TRAN_TRAP,
                                    product.options(precision=A.PREC_FP64, max_halvings=HALV,
                                                    **POLISH), wave_nodes=nodes)
    assert all(s["lte_rejects"] == 0 and s["halvings"] == 0 for s in st0)
    prob.close()


@pytest.mark.parametrize("prec", [A.PREC_FP64, A.PREC_MIXED])
def test_lte_persistent_equals_round_graph(product, ctx, prec):
    nl = circuits.grid_circuit(8)
    ni = 3
    inst = circuits.mc_instances(nl, ni)
    prob = product.Problem(ctx, nl, max_instances=ni)
    prob.set_instances(inst)
    out = []
    for schedule in (-4, -3):
        prob.run_mc_device(DT, STEPS, A.TRAN_TRAP, product_opts(product, prec, schedule=schedule))
        v, st = prob.read_results()
        out.append((v, [(s["status"], s["iterations"], s["halvings"], s["lte_rejects"]) for s in st]))
    assert np.array_equal(out[0][0], out[1][0]) and out[0][1] == out[1][1]
    assert all(k[3] > 0 for k in out[0][1])
    prob.close()
