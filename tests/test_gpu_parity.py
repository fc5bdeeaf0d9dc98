"""Parity of the CUDA path (through the C ABI) with the CPU oracle.

Tolerances (FP64 oracle as truth, both sides polished to the FP64 fixed point):
node voltages |dv| <= 1e-9 |v| + 1e-12 V; Norton branch currents
I = 1e3 (V - (v+ - v-)) within 1e-12 A. Jacobian values from the FP64
evaluation kernel within 4 ulp of the reference stamps where the kernel keeps
the reference's term order; values with hundreds of terms (the supply node's
diagonal), whose sums the kernel splits over warps, within twice the
recursive-summation bound (n - 1) eps sum|t|.
"""
import numpy as np
import pytest

from karam_b200 import _abi as A
from karam_b200 import circuits

pytestmark = pytest.mark.gpu

POLISH = dict(polish_max=8)
KES_MAX_DEV = 48  # devices one evaluation block holds (nr_types.h)


def scaled_err(v, v_ref, rel=1e-9, abs_=1e-12):
    return float(np.max(np.abs(v - v_ref) / (rel * np.abs(v_ref) + abs_)))


def branch_currents(nl, v, vs_values=None):
    out = []
    for k, (p, q, dc, kind, pulse) in enumerate(nl.vsrc):
        val = dc if vs_values is None else vs_values[k]
        vp = v[p - 1] if p > 0 else 0.0
        vq = v[q - 1] if q > 0 else 0.0
        out.append(1e3 * (val - (vp - vq)))
    return np.array(out)


def test_eval_stamp_fp64_matches_reference_stamps(product, ctx, port):
    nl = circuits.config2()
    inst = circuits.mc_instances(nl, 3)
    prob = product.Problem(ctx, nl, max_instances=3)
    prob.set_instances(inst)
    rng = np.random.default_rng(7)
    vs = rng.uniform(-0.2, 2.0, size=(3, prob.n))
    jac, f = prob.eval_stamp(vs, A.PREC_FP64)
    rp, col = port.pattern(nl)
    eps = np.finfo(np.float64).eps
    for i in range(3):
        vals, rhs = port.stamp(nl, vs[i], inst, i)
        absum, nterms = port.stamp_abs(nl, vs[i], inst, i)
        # the gmin diagonal is not part of the evaluated Jacobian
        scale = np.maximum(np.abs(vals), 1e-300)
        ulp = np.abs(jac[i] - vals) / (np.spacing(scale))
        # values with few terms are summed in the reference's term order
        few = nterms <= 4 * KES_MAX_DEV
        assert ulp[few].max() <= 4, f"Jacobian differs by {ulp[few].max()} ulp"
        # hub values (hundreds of terms, split over warps): within the
        # recursive-summation bound (n - 1) eps sum|t| of the reordered sum
        hub = ~few
        bound = 2 * np.maximum(nterms[hub] - 1, 1) * eps * absum[hub]
        assert np.all(np.abs(jac[i][hub] - vals[hub]) <= bound)
        # KCL residual: device currents vs J v - rhs of the reference stamps
        jv = np.array([np.dot(vals[rp[r]:rp[r + 1]], vs[i][col[rp[r]:rp[r + 1]]]) for r in range(prob.n)])
        fref = jv - rhs
        assert np.max(np.abs(f[i] - fref)) <= 1e-12 * (1 + np.max(np.abs(fref)))


def test_eval_stamp_mixed_is_fp32_rounding(product, ctx, port):
    nl = circuits.config1()
    prob = product.Problem(ctx, nl, max_instances=1)
    prob.set_instances(None)
    v = np.linspace(0, 1.8, prob.n)
    jac, _ = prob.eval_stamp(v[None], A.PREC_MIXED)
    vals, _ = port.stamp(nl, v)
    assert np.array_equal(jac[0], vals.astype(np.float32).astype(np.float64))


@pytest.mark.parametrize("prec", [A.PREC_FP64, A.PREC_MIXED])
def test_dc_config1_matches_oracle(product, ctx, port, prec):
    nl = circuits.config1()
    v_ref, st_ref = port.solve_dc(nl, **POLISH)
    prob = product.Problem(ctx, nl, max_instances=1)
    prob.set_instances(None)
    v, st = prob.solve_dc(product.options(precision=prec, **POLISH))
    assert st[0]["status"] == A.ST_CONVERGED
    assert scaled_err(v[0], v_ref) <= 1.0
    dI = np.abs(branch_currents(nl, v[0]) - branch_currents(nl, v_ref))
    assert dI.max() <= 1e-12, dI
    # iteration counts reported side by side; FP64 follows the reference closely
    if prec == A.PREC_FP64:
        assert abs(st[0]["iterations"] - st_ref["iterations"]) <= 8


def test_dc_config1_reference_stopping_rule(product, ctx, port):
    """Without polishing, the FP64 path stops where the reference does."""
    nl = circuits.config1()
    v_ref, st_ref = port.solve_dc(nl)
    prob = product.Problem(ctx, nl, max_instances=1)
    prob.set_instances(None)
    v, st = prob.solve_dc(product.options(precision=A.PREC_FP64))
    assert st[0]["status"] == A.ST_CONVERGED
    print("NR iterations: oracle", st_ref["iterations"], "GPU FP64", st[0]["iterations"])
    assert abs(st[0]["iterations"] - st_ref["iterations"]) <= 4
    assert np.max(np.abs(v[0] - v_ref)) < 1e-6


@pytest.mark.parametrize("prec", [A.PREC_FP64, A.PREC_MIXED])
def test_dc_config2_mc_batch(product, ctx, port, prec):
    nl = circuits.config2()
    ni = 6
    inst = circuits.mc_instances(nl, ni)
    prob = product.Problem(ctx, nl, max_instances=ni)
    prob.set_instances(inst)
    v, st = prob.solve_dc(product.options(precision=prec, **POLISH))
    for i in range(ni):
        v_ref, st_ref = port.solve_dc(nl, inst, i, linear_solver=1, **POLISH)
        assert st_ref["converged"] == 1
        assert st[i]["status"] == A.ST_CONVERGED, st[i]
        assert scaled_err(v[i], v_ref) <= 1.0, (i, scaled_err(v[i], v_ref))
        dI = np.abs(branch_currents(nl, v[i]) - branch_currents(nl, v_ref))
        assert dI.max() <= 1e-12, (i, dI)


@pytest.mark.parametrize("prec", [A.PREC_FP64, A.PREC_MIXED])
def test_transient_config2_backward_euler(product, ctx, port, prec):
    nl = circuits.config2()
    ni, steps, dt = 2, 60, 1e-12
    inst = circuits.mc_instances(nl, ni)
    prob = product.Problem(ctx, nl, max_instances=ni)
    prob.set_instances(inst)
    opts = product.options(precision=prec, **POLISH)
    vdc, st = prob.solve_dc(opts)
    nodes = [2, 3, 4, 5, 10, 20, 259]
    v, st, wave = prob.step_transient(dt, steps, A.TRAN_BE, opts, wave_nodes=nodes)
    for i in range(ni):
        vd_ref, _ = port.solve_dc(nl, inst, i, linear_solver=1, **POLISH)
        assert scaled_err(vdc[i], vd_ref) <= 1.0
        v_ref, st_ref, w_ref = port.transient(nl, vd_ref, dt, steps, A.TRAN_BE, inst, i,
                                              wave_nodes=nodes, linear_solver=1, **POLISH)
        assert st_ref["converged"] == 1 and st[i]["status"] == A.ST_CONVERGED
        assert scaled_err(v[i], v_ref, rel=1e-9, abs_=1e-12) <= 1.0
        assert np.max(np.abs(wave[i] - w_ref)) <= 1e-9 * np.max(np.abs(w_ref)) + 1e-12


def test_run_mc_matches_separate_calls(product, ctx):
    nl = circuits.config2()
    ni = 4
    inst = circuits.mc_instances(nl, ni)
    prob = product.Problem(ctx, nl, max_instances=ni)
    opts = product.options(precision=A.PREC_MIXED, **POLISH)
    v1, st1 = prob.run_mc(inst, 1e-12, 20, A.TRAN_BE, opts)
    prob.set_instances(inst)
    prob.solve_dc(opts)
    v2, st2, _ = prob.step_transient(1e-12, 20, A.TRAN_BE, opts)
    assert all(s["status"] == A.ST_CONVERGED for s in st1 + st2)
    assert scaled_err(v1, v2, rel=1e-10, abs_=1e-13) <= 1.0
