"""The batch statistical seeder (KARAM_SEED_EMA) on the GPU.

NeuralSeeder::predictSeed (solvers/neural_seeder.h:100-137) seeds the batch
from the plain-NR DC solutions of its first KARAM_SEED_HISTORY instances; the
seeded instances start at the final GMIN step and fall back to full GMIN
stepping after seed_max_iter iterations. Plain NR decides the result: the
seeded solutions must meet the same tolerances against the oracle (node
voltages |dv| <= 1e-9 |v| + 1e-12 V, Norton branch currents within 1e-12 A).
"""
import numpy as np
import pytest

from karam_b200 import _abi as A
from karam_b200 import circuits

from test_gpu_parity import POLISH, branch_currents, scaled_err

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("prec", [A.PREC_FP64, A.PREC_MIXED])
def test_ema_seeded_dc_matches_oracle(product, ctx, port, prec):
    nl = circuits.config2()
    ni = A.SEED_HISTORY + 4
    inst = circuits.mc_instances(nl, ni)
    prob = product.Problem(ctx, nl, max_instances=ni)
    prob.set_instances(inst)
    v_plain, st_plain = prob.solve_dc(product.options(precision=prec, **POLISH))
    v, st = prob.solve_dc(product.options(precision=prec, seeded=A.SEED_EMA, **POLISH))
    for i in range(ni):
        assert st[i]["status"] == A.ST_CONVERGED, st[i]
        # every instance of the batch job starts from the seed and needs no fallback
        assert st[i]["seeded_ok"] == 1, (i, st[i])
        assert st[i]["iterations"] < st_plain[i]["iterations"], (i, st[i], st_plain[i])
    for i in (0, A.SEED_HISTORY, ni - 1):
        v_ref, st_ref = port.solve_dc(nl, inst, i, linear_solver=1, **POLISH)
        assert st_ref["converged"] == 1
        assert scaled_err(v[i], v_ref) <= 1.0, (i, scaled_err(v[i], v_ref))
        dI = np.abs(branch_currents(nl, v[i]) - branch_currents(nl, v_ref))
        assert dI.max() <= 1e-12, (i, dI)
    assert scaled_err(v, v_plain) <= 1.0


def test_ema_seeded_mc_matches_plain(product, ctx):
    nl = circuits.config2()
    ni = 40
    inst = circuits.mc_instances(nl, ni)
    prob = product.Problem(ctx, nl, max_instances=ni)
    plain = product.options(precision=A.PREC_MIXED, **POLISH)
    seeded = product.options(precision=A.PREC_MIXED, seeded=A.SEED_EMA, **POLISH)
    v0, st0 = prob.run_mc(inst, 1e-12, 20, A.TRAN_BE, plain)
    r0 = prob.timing()["rounds"]
    v1, st1 = prob.run_mc(inst, 1e-12, 20, A.TRAN_BE, seeded)
    t1 = prob.timing()
    assert all(s["status"] == A.ST_CONVERGED for s in st0 + st1)
    assert all(s["seeded_ok"] == 1 for s in st1)
    assert scaled_err(v1, v0) <= 1.0
    # the seeded job skips the GMIN stepping of all but the history instances
    assert t1["rounds"] < r0, (t1["rounds"], r0)


def test_ema_seeder_small_batch_runs_plain(product, ctx):
    nl = circuits.config1()
    ni = A.SEED_HISTORY
    inst = circuits.mc_instances(nl, ni)
    prob = product.Problem(ctx, nl, max_instances=ni)
    prob.set_instances(inst)
    v0, st0 = prob.solve_dc(product.options(precision=A.PREC_FP64, **POLISH))
    v1, st1 = prob.solve_dc(product.options(precision=A.PREC_FP64, seeded=A.SEED_EMA, **POLISH))
    assert [s["iterations"] for s in st1] == [s["iterations"] for s in st0]
    assert all(s["seeded_ok"] == 0 for s in st1)
    assert np.array_equal(v0, v1)
