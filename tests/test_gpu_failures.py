"""Failure statuses and convergence diagnostics on the GPU, every failure made
on the host (no GPU fault is involved):

- KARAM_ST_SINGULAR: two floating nodes joined by a 1e-15 ohm resistor, so the
  second pivot of their block cancels to exactly zero (|pivot| < 1e-25, the
  reference's singular test, math/linalg.h:782-797);
- KARAM_ST_NAN: an instance whose MOSFET KP is NaN (the KCL residual turns
  non-finite; circuitsim_solver.cpp:381 sanitises only the update);
- KARAM_ST_TIMEOUT: a round budget (opts.max_rounds) that ends before the solve;
- KARAM_ST_NOCONV: a one-iteration NR budget per GMIN step.

The DC convergence diagnostics (ConvergenceEngine::classifyFailure, the
stagnation / divergence flags, the history length) are compared with the
oracle's, which keeps the whole history; the device keeps running counts and a
ring of the last KARAM_HISTORY_MAX iterations."""
import math

import numpy as np
import pytest

from karam_b200 import _abi as A
from karam_b200 import circuits

pytestmark = pytest.mark.gpu

DIAG = ("failure_type", "stagnation", "divergence", "history_len")


def singular_netlist():
    nl = circuits.Netlist()
    nl.vsource(1, 0, 1.0)
    nl.resistor(1, 0, 1e3)
    nl.resistor(1, 2, 1e3)
    nl.resistor(3, 4, 1e-15)  # nodes 3 and 4 float together
    nl.resistor(4, 5, 1e-15)
    return nl


@pytest.mark.parametrize("prec", [A.PREC_FP64, A.PREC_MIXED])
def test_singular_status(product, ctx, port, prec):
    nl = singular_netlist()
    _, st_ref = port.solve_dc(nl)
    assert st_ref["singular"] == 1 and st_ref["converged"] == 0
    prob = product.Problem(ctx, nl, max_instances=1)
    prob.set_instances(None)
    _, st = prob.solve_dc(product.options(precision=prec))
    assert st[0]["status"] == A.ST_SINGULAR
    assert st[0]["failure_type"] == A.FAIL_SINGULAR_MATRIX == st_ref["failure_type"]


@pytest.mark.parametrize("prec", [A.PREC_FP64, A.PREC_MIXED])
def test_nan_parameter_status(product, ctx, prec):
    nl = circuits.config1()
    ni = 3
    inst = circuits.mc_instances(nl, ni)
    inst.mos_kp = inst.mos_kp.copy()
    inst.mos_kp[1, 5] = np.float32(math.nan)
    prob = product.Problem(ctx, nl, max_instances=ni)
    prob.set_instances(inst)
    v, st = prob.solve_dc(product.options(precision=prec, polish_max=6))
    assert [s["status"] for s in st] == [A.ST_CONVERGED, A.ST_NAN, A.ST_CONVERGED]
    assert np.all(np.isfinite(v[0])) and np.all(np.isfinite(v[2]))


def test_round_budget_timeout(product, ctx):
    nl = circuits.config1()
    prob = product.Problem(ctx, nl, max_instances=1)
    prob.set_instances(None)
    _, st = prob.solve_dc(product.options(precision=A.PREC_FP64, max_rounds=16))
    assert st[0]["status"] == A.ST_TIMEOUT
    # the same problem solves to the end without the budget
    _, st = prob.solve_dc(product.options(precision=A.PREC_FP64))
    assert st[0]["status"] == A.ST_CONVERGED


@pytest.mark.parametrize("max_nr_iter", [1, 3])
def test_iteration_budget_noconv_matches_oracle(product, ctx, port, max_nr_iter):
    nl = circuits.config1()
    _, st_ref = port.solve_dc(nl, max_nr_iter=max_nr_iter)
    assert st_ref["converged"] == 0
    prob = product.Problem(ctx, nl, max_instances=1)
    prob.set_instances(None)
    _, st = prob.solve_dc(product.options(precision=A.PREC_FP64, max_nr_iter=max_nr_iter))
    assert st[0]["status"] == A.ST_NOCONV
    assert st[0]["iterations"] == st_ref["iterations"]
    assert {k: st[0][k] for k in DIAG} == {k: st_ref[k] for k in DIAG}
    f, dv = prob.history(0)
    assert len(f) == min(st_ref["history_len"], A.HISTORY_MAX)


def test_converged_diagnostics_match_oracle(product, ctx, port):
    """config 1 in FP64 takes the oracle's NR path (84 iterations); the
    classification of the full history (the reference classifies converged
    solves too: its first step from the seed moves nodes by > 100 V) and the
    flags agree, and the ring holds the last iterations with the final
    residual below the last GMIN step's tolerance."""
    nl = circuits.config1()
    _, st_ref = port.solve_dc(nl)
    prob = product.Problem(ctx, nl, max_instances=1)
    prob.set_instances(None)
    _, st = prob.solve_dc(product.options(precision=A.PREC_FP64))
    assert st[0]["status"] == A.ST_CONVERGED and st[0]["iterations"] == st_ref["iterations"]
    assert {k: st[0][k] for k in DIAG} == {k: st_ref[k] for k in DIAG}
    f, dv = prob.history(0)
    assert len(f) == A.HISTORY_MAX and f[-1] < 1e-9 and np.all(dv >= 0)
