"""The persistent per-instance kernel (opts.schedule -4: one CTA runs every NR
round of its instance in one launch, rescues included) runs the code of the
per-round block-per-instance kernels (-3: k_es_one + k_lu_big with the packed
program + k_rescue, a launch each per round), so its voltages, iteration
counts and statuses equal theirs bit for bit; and it is what small batches
(no more instances than SMs) get by default."""
import numpy as np
import pytest

from karam_b200 import _abi as A
from karam_b200 import circuits

pytestmark = pytest.mark.gpu

POLISH = dict(polish_max=8)


def stats_key(st):
    return [(s["status"], s["iterations"], s["polish_iters"], s["damped"], s["rescued"],
             s["halvings"]) for s in st]


@pytest.mark.parametrize("prec", [A.PREC_FP64, A.PREC_MIXED])
def test_config1_persistent_equals_round_graph_and_oracle(product, ctx, port, prec):
    nl = circuits.config1()
    prob = product.Problem(ctx, nl, max_instances=1)
    prob.set_instances(None)
    v4, st4 = prob.solve_dc(product.options(precision=prec, schedule=-4, **POLISH))
    t4 = prob.timing()
    v3, st3 = prob.solve_dc(product.options(precision=prec, schedule=-3, **POLISH))
    v0, st0 = prob.solve_dc(product.options(precision=prec, **POLISH))
    t0 = prob.timing()
    assert t4["level_schedule"] == 5 and t4["persistent_rounds"] == t4["rounds"] > 0
    assert t0["level_schedule"] == 5  # the default for one instance
    assert np.array_equal(v4, v3) and np.array_equal(v4, v0)
    assert stats_key(st4) == stats_key(st3) == stats_key(st0)
    v_ref, st_ref = port.solve_dc(nl, **POLISH)
    assert st4[0]["status"] == A.ST_CONVERGED
    assert np.max(np.abs(v4[0] - v_ref) / (1e-9 * np.abs(v_ref) + 1e-12)) <= 1.0


@pytest.mark.parametrize("prec", [A.PREC_MIXED, A.PREC_FP64])
def test_config2_batch_persistent_equals_round_graph(product, ctx, prec):
    """DC + 20 BE steps of a 40-instance config-2 batch (unseeded: GMIN-step
    rescues happen), in one persistent launch vs the per-round graph."""
    nl = circuits.config2()
    ni = 40
    inst = circuits.mc_instances(nl, ni)
    prob = product.Problem(ctx, nl, max_instances=ni)
    prob.set_instances(inst)
    out = []
    for schedule in (-4, -3):
        prob.run_mc_device(1e-12, 20, A.TRAN_BE, product.options(precision=prec, schedule=schedule,
                                                                 **POLISH))
        t = prob.timing()
        v, st = prob.read_results()
        out.append((t, v, st))
    (t4, v4, s4), (t3, v3, s3) = out
    assert t4["level_schedule"] == 5 and t3["level_schedule"] == 4
    assert np.array_equal(v4, v3)
    assert stats_key(s4) == stats_key(s3)
    assert t4["rescues"] == t3["rescues"]
    assert sum(s["status"] == A.ST_CONVERGED for s in s4) >= ni - 2


def test_round_budget_stops_persistent_kernel(product, ctx):
    nl = circuits.config1()
    prob = product.Problem(ctx, nl, max_instances=1)
    prob.set_instances(None)
    _, st = prob.solve_dc(product.options(precision=A.PREC_FP64, schedule=-4, max_rounds=10))
    assert st[0]["status"] == A.ST_TIMEOUT and prob.timing()["rounds"] == 10


@pytest.mark.parametrize("prec", [A.PREC_MIXED, A.PREC_FP64])
def test_uneven_batch_in_one_launch_equals_per_problem_runs(product, ctx, prec):
    """Grids of three sizes (8 x 8 and 16 x 16 fit the packed program in shared
    memory, 40 x 40 keeps its slots in global memory) and a config-2 batch:
    DC + 10 trapezoidal steps of all four problems in ONE k_persist_multi
    launch equal each problem's own per-round run bit for bit."""
    specs = [(circuits.grid_circuit(8), 3), (circuits.grid_circuit(16), 2),
             (circuits.grid_circuit(40), 2), (circuits.config2(), 4)]
    dt, steps = 20e-12, 10
    opts = product.options(precision=prec, **POLISH)
    probs = []
    for nl, ni in specs:
        p = product.Problem(ctx, nl, max_instances=ni)
        p.set_instances(circuits.mc_instances(nl, ni))
        probs.append(p)
    product.run_mc_multi(probs, dt, steps, A.TRAN_TRAP, opts)
    multi = [p.read_results() for p in probs]
    t = probs[0].timing()
    assert t["level_schedule"] == 5 and t["persistent_rounds"] == t["rounds"] > 0
    for p, (v_m, st_m) in zip(probs, multi):
        p.run_mc_device(dt, steps, A.TRAN_TRAP,
                        product.options(precision=prec, schedule=-2, **POLISH))
        v, st = p.read_results()
        assert np.array_equal(v_m, v)
        assert stats_key(st_m) == stats_key(st)
        assert sum(s["status"] == A.ST_CONVERGED for s in st) >= len(st) - 1
    for p in probs:
        p.close()


def test_multi_launch_argument_errors(product, ctx):
    nl = circuits.config1()
    p = product.Problem(ctx, nl, max_instances=1)
    p.set_instances(None)
    with pytest.raises(product.KaramError) as e:
        product.run_mc_multi([p, p], 0.0, 0, A.TRAN_BE, product.options())
    assert e.value.code == A.KARAM_E_INVALID
    ctx2 = product.Context(0)
    q = product.Problem(ctx2, nl, max_instances=1)
    q.set_instances(None)
    with pytest.raises(product.KaramError) as e:
        product.run_mc_multi([p, q], 0.0, 0, A.TRAN_BE, product.options())
    assert e.value.code == A.KARAM_E_INVALID
    # one problem alone in the multi launch equals its own persistent solve
    product.run_mc_multi([p], 0.0, 0, A.TRAN_BE, product.options(precision=A.PREC_FP64))
    v1, s1 = p.read_results()
    v2, s2 = p.solve_dc(product.options(precision=A.PREC_FP64, schedule=-4))
    assert np.array_equal(v1, v2) and stats_key(s1) == stats_key(s2)
    q.close()
    ctx2.close()
    p.close()
