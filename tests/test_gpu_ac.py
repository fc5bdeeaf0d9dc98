"""Small-signal AC sweeps on the GPU (karam_ac_sweep) against the oracle.

Each instance's sweep runs at the product's own DC point: Y(jw) = the FP64 NR
Jacobian there + jwC + 1e-12 on every diagonal, the input node driven through
1e6 S, factored on the problem's static pivots in complex FP64. The oracle
(pinned bit for bit to the reference build's sweep of the same rule by the
CPU tests) runs the same sweep at the same DC point with a dense LU and
partial pivoting; the two agree within |dv| / (1e-9 |v| + 1e-12 V) <= 1 on
every complex node voltage. The error cases come from the host: a problem
with no DC point, and a grid whose level program does not fit one CTA."""
import os
import sys

import numpy as np
import pytest

from karam_b200 import _abi as A
from karam_b200 import circuits

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(HERE, "golden"))
import cases  # noqa: E402

pytestmark = pytest.mark.gpu

POLISH = dict(polish_max=8)


def scaled(x, ref):
    return float(np.max(np.abs(x - ref) / (1e-9 * np.abs(ref) + 1e-12)))


def frequencies(f0, f1, npts):
    lo, hi = np.log10(max(f0, 1e-3)), np.log10(max(f1, f0 + 1.0))
    return np.array([10.0 ** (lo + (hi - lo) * i / max(npts - 1, 1)) for i in range(npts)])


@pytest.mark.parametrize("prec", [A.PREC_FP64, A.PREC_MIXED])
@pytest.mark.parametrize("name", sorted(cases.AC_CASES))
def test_ac_sweep_matches_oracle(product, ctx, port, name, prec):
    make, node, f0, f1, npts = cases.AC_CASES[name]
    nl = make()
    ni = 3 if nl.n_mos else 1
    inst = circuits.mc_instances(nl, ni) if nl.n_mos else None
    prob = product.Problem(ctx, nl, max_instances=ni)
    prob.set_instances(inst)
    v, st = prob.solve_dc(product.options(precision=prec, **POLISH))
    f, x, status = prob.ac_sweep(f0, f1, npts, node)
    assert np.allclose(f, frequencies(f0, f1, npts), rtol=1e-15, atol=0)
    assert x.shape == (ni, npts, nl.n_nodes)
    for i in range(ni):
        assert st[i]["status"] == A.ST_CONVERGED
        assert np.all(status[i] == A.ST_CONVERGED)
        x_ref, singular = port.ac(nl, v[i], f0, f1, npts, node, inst=inst, idx=i)
        assert singular == 0
        assert scaled(x[i], x_ref) <= 1.0, (name, i, scaled(x[i], x_ref))
    prob.close()


def test_ac_sweep_error_cases(product, ctx):
    nl = cases.rc_ladder_diodes()
    prob = product.Problem(ctx, nl, max_instances=1)
    prob.set_instances(None)
    with pytest.raises(product.KaramError) as e:
        prob.ac_sweep(1e3, 1e9, 4, 1)  # no DC point yet
    assert e.value.code == A.KARAM_E_STATE
    prob.solve_dc(product.options(precision=A.PREC_FP64))
    prob.ac_sweep(1e3, 1e9, 4, 1)
    prob.run_mc_device(1e-12, 2, A.TRAN_BE, product.options(precision=A.PREC_FP64))
    with pytest.raises(product.KaramError) as e:
        prob.ac_sweep(1e3, 1e9, 4, 1)  # the last job ran a transient
    assert e.value.code == A.KARAM_E_STATE
    prob.close()
    nl = circuits.grid_circuit(24)  # no packed level program
    prob = product.Problem(ctx, nl, max_instances=1)
    prob.set_instances(None)
    prob.solve_dc(product.options(precision=A.PREC_MIXED, **POLISH))
    with pytest.raises(product.KaramError) as e:
        prob.ac_sweep(1e3, 1e9, 4, 1)
    assert e.value.code == A.KARAM_E_UNSUPPORTED
    prob.close()
