"""The resistor-grid family of the uneven batch on the GPU: every factor/solve
schedule (a warp per instance with the level schedule in shared memory, a CTA
per instance with the instance's slots in shared or global memory) against
the reference-built fixture and the CPU oracle, and the schedules against
each other (they run the same level-scheduled elimination in the same order,
so their results are identical)."""
import os
import sys

import numpy as np
import pytest

from karam_b200 import _abi as A
from karam_b200 import circuits

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(HERE, "golden"))

pytestmark = pytest.mark.gpu

POLISH = dict(polish_max=8)
KIND = {1: 1, -1: 2, -2: 3, -3: 4, -4: 5}  # schedule option -> karam_timing.level_schedule


def scaled_err(v, v_ref, rel=1e-9, abs_=1e-12):
    return float(np.max(np.abs(v - v_ref) / (rel * np.abs(v_ref) + abs_)))


def solve(product, ctx, nl, inst, ni, prec, schedule):
    prob = product.Problem(ctx, nl, max_instances=ni)
    prob.set_instances(inst)
    v, st = prob.solve_dc(product.options(precision=prec, schedule=schedule, **POLISH))
    return prob, v, st


@pytest.mark.parametrize("prec", [A.PREC_FP64, A.PREC_MIXED])
@pytest.mark.parametrize("schedule", [1, -1, -2, -3])
def test_grid8_dc_matches_reference_fixture(product, ctx, prec, schedule):
    g = np.load(os.path.join(HERE, "golden", "grid8.npz"))
    nl = circuits.grid_circuit(8)
    prob, v, st = solve(product, ctx, nl, None, 1, prec, schedule)
    assert prob.timing()["level_schedule"] == KIND[schedule]
    assert st[0]["status"] == A.ST_CONVERGED
    assert scaled_err(v[0], g["dc_v"]) <= 1.0


@pytest.mark.parametrize("prec", [A.PREC_FP64, A.PREC_MIXED])
def test_schedules_give_identical_results(product, ctx, prec):
    nl = circuits.grid_circuit(10)
    inst = circuits.mc_instances(nl, 5)
    out = []
    for schedule in (1, -1, -2, -3):
        prob, v, st = solve(product, ctx, nl, inst, 5, prec, schedule)
        assert prob.timing()["level_schedule"] == KIND[schedule]
        out.append((v, [s["iterations"] for s in st]))
    for v, its in out[1:]:
        assert np.array_equal(v, out[0][0]) and its == out[0][1]


@pytest.mark.parametrize("schedule", [0, -2])
def test_grid24_dc_mc_batch(product, ctx, port, schedule):
    """578 unknowns: beyond the warp-per-instance program; a CTA per instance."""
    nl = circuits.grid_circuit(24)
    ni = 3
    inst = circuits.mc_instances(nl, ni)
    prob, v, st = solve(product, ctx, nl, inst, ni, A.PREC_MIXED, schedule)
    assert prob.timing()["level_schedule"] in (2, 3, 5)
    for i in range(ni):
        v_ref, st_ref = port.solve_dc(nl, inst, i, linear_solver=1, **POLISH)
        assert st_ref["converged"] == 1 and st[i]["status"] == A.ST_CONVERGED
        assert scaled_err(v[i], v_ref) <= 1.0, (i, scaled_err(v[i], v_ref))


@pytest.mark.parametrize("prec", [A.PREC_FP64, A.PREC_MIXED])
def test_grid_trapezoidal_transient(product, ctx, port, prec):
    nl = circuits.grid_circuit(12)
    ni, steps, dt = 2, 30, 20e-12
    inst = circuits.mc_instances(nl, ni)
    prob = product.Problem(ctx, nl, max_instances=ni)
    prob.set_instances(inst)
    opts = product.options(precision=prec, schedule=-1, **POLISH)
    vdc, st = prob.solve_dc(opts)
    nodes = [2, 3, 40, 100, 146]
    v, st, wave = prob.step_transient(dt, steps, A.TRAN_TRAP, opts, wave_nodes=nodes)
    for i in range(ni):
        vd_ref, _ = port.solve_dc(nl, inst, i, linear_solver=1, **POLISH)
        assert scaled_err(vdc[i], vd_ref) <= 1.0
        v_ref, st_ref, w_ref = port.transient(nl, vd_ref, dt, steps, A.TRAN_TRAP, inst, i,
                                              wave_nodes=nodes, linear_solver=1, **POLISH)
        assert st_ref["converged"] == 1 and st[i]["status"] == A.ST_CONVERGED
        assert scaled_err(v[i], v_ref) <= 1.0
        assert np.max(np.abs(wave[i] - w_ref)) <= 1e-9 * np.max(np.abs(w_ref)) + 1e-12


def test_tuned_schedule_is_used_and_feasible(product, ctx):
    nl = circuits.grid_circuit(12)
    ni = 6
    inst = circuits.mc_instances(nl, ni)
    prob = product.Problem(ctx, nl, max_instances=ni)
    prob.set_instances(inst)
    opts = product.options(precision=A.PREC_MIXED, **POLISH)
    sch, ms = prob.tune_schedule(opts, rounds=8)
    assert ms > 0 and (sch in (-1, -2, -3, -4) or 1 <= sch <= 32)
    v_tuned, st_tuned = prob.solve_dc(opts)  # opts.schedule == 0: the tuned choice
    kind_tuned = prob.timing()["level_schedule"]
    v_explicit, st_explicit = prob.solve_dc(product.options(precision=A.PREC_MIXED,
                                                            schedule=sch, **POLISH))
    assert prob.timing()["level_schedule"] == kind_tuned
    assert np.array_equal(v_tuned, v_explicit)
    assert all(s["status"] == A.ST_CONVERGED for s in st_tuned)


@pytest.mark.parametrize("prec", [A.PREC_MIXED, A.PREC_FP64])
def test_tail_switch_keeps_results(product, ctx, prec):
    """A batch larger than the SM count runs its last rounds with a CTA per
    live instance over the live list (karam_timing.tail_rounds); the results
    equal a run on that kernel from the start, and one on the warp kernel."""
    nl = circuits.config2()
    ni = 320
    inst = circuits.mc_instances(nl, ni)
    prob = product.Problem(ctx, nl, max_instances=ni)
    prob.set_instances(inst)
    runs = []
    for schedule in (0, -1, -3):
        opts = product.options(precision=prec, schedule=schedule, **POLISH)
        prob.run_mc_device(1e-12, 20, A.TRAN_BE, opts)
        t = prob.timing()
        v, st = prob.read_results()
        runs.append((t, v, st))
    (t0, v0, s0), (t1, v1, s1), (t3, v3, s3) = runs
    assert t0["level_schedule"] == 1 and t0["tail_rounds"] > 0
    assert t1["level_schedule"] == 2 and t1["tail_rounds"] == 0
    assert t3["level_schedule"] == 4 and t3["tail_rounds"] == 0
    assert np.array_equal(v0, v1) and np.array_equal(v0, v3)
    assert [s["iterations"] for s in s0] == [s["iterations"] for s in s1]
    assert sum(s["status"] == A.ST_CONVERGED for s in s0) >= ni - 2


# The larger grids against their reference-built fixtures (tests/golden/
# grid16/32/64.npz): DC of two Monte-Carlo instances and a trapezoidal waveform
# across the gate ramp. Slots in shared memory where they fit (FP32 slots up to
# grid 32, FP64 up to grid 16), in global memory everywhere.
LARGE = [("grid16", -1, A.PREC_FP64), ("grid16", -1, A.PREC_MIXED), ("grid16", -2, A.PREC_MIXED),
         ("grid32", -1, A.PREC_MIXED), ("grid32", -2, A.PREC_FP64), ("grid32", -2, A.PREC_MIXED),
         ("grid64", -2, A.PREC_FP64), ("grid64", -2, A.PREC_MIXED)]


@pytest.mark.parametrize("name,schedule,prec", LARGE)
def test_large_grid_matches_reference_fixture(product, ctx, name, schedule, prec):
    import cases
    g = np.load(os.path.join(HERE, "golden", f"{name}.npz"))
    nl = circuits.grid_circuit(cases.GRIDS[name])
    inst = circuits.Instances(2, g["mc_kp"], g["mc_vto"])
    tr = cases.GRID_TRAN
    prob = product.Problem(ctx, nl, max_instances=2)
    prob.set_instances(inst)
    opts = product.options(precision=prec, schedule=schedule, max_halvings=tr["max_halvings"],
                           **POLISH)
    v, st = prob.solve_dc(opts)
    assert prob.timing()["level_schedule"] == KIND[schedule]
    for i in range(2):
        assert st[i]["status"] == A.ST_CONVERGED
        assert scaled_err(v[i], g["dc_v"][i]) <= 1.0, (i, scaled_err(v[i], g["dc_v"][i]))
    nodes = [int(x) for x in g["tran_wave_nodes"]]
    vt, st, wave = prob.step_transient(tr["dt"], tr["steps"], A.TRAN_TRAP, opts, wave_nodes=nodes)
    assert st[0]["status"] == A.ST_CONVERGED
    assert scaled_err(vt[0], g["tran_v"]) <= 1.0, scaled_err(vt[0], g["tran_v"])
    w_ref = g["tran_wave"]
    assert np.max(np.abs(wave[0] - w_ref)) <= 1e-9 * np.max(np.abs(w_ref)) + 1e-12
