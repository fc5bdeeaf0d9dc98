"""The oracle restatement and the product's host symbolic layer against the
golden fixtures generated from the reference's own code (tests/golden/).

The reference ships no tests or known-answer vectors for this path; the
fixtures come from the oracle library compiled from the reference sources
(see tests/golden/make_golden.py), so they pin both the restatement and the
product without the reference tree present. CPU only.
"""
import os
import sys

import numpy as np
import pytest

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(HERE, "golden"))

import cases  # noqa: E402
from karam_b200 import _abi as A  # noqa: E402
from karam_b200 import circuits  # noqa: E402

ALL = {**cases.SMALL, **cases.BENCH}
STAT_KEYS = ("converged", "iterations", "polish_iters", "damped", "gmin_step", "singular")


def golden(name):
    with np.load(os.path.join(HERE, "golden", f"{name}.npz")) as z:
        return {k: z[k] for k in z.files}


def stats_arr(st):
    return np.array([st[k] for k in STAT_KEYS], np.int64)


def instances_for(name, nl, g):
    if name != "config2":
        return None
    return circuits.Instances(2, g["mc_kp"], g["mc_vto"])


# ---------------------------------------------------------------------------
# Monte-Carlo sampler vs PortableRNG / PortableNormalDist (math/portable_rng.h)
# ---------------------------------------------------------------------------
def test_sampler_matches_reference_rng():
    g = golden("rng_normals")
    rng = circuits.PCG32(g["seeds"])
    draws = []
    for _ in range(g["normals"].shape[1] // 2):
        c, s = circuits.normal_pairs(rng)
        draws += [c, s]
    ours = np.stack(draws, axis=1)
    # libm vs numpy transcendental rounding: a few ulp at most
    assert np.allclose(ours, g["normals"], rtol=4e-15, atol=4e-15)


def test_mc_parameters_are_reproducible():
    g = golden("config2")
    inst = circuits.mc_instances(circuits.config2(), 2)
    assert np.array_equal(inst.mos_kp, g["mc_kp"]) and np.array_equal(inst.mos_vto, g["mc_vto"])


# ---------------------------------------------------------------------------
# oracle restatement (port) vs the reference-generated fixtures
# ---------------------------------------------------------------------------
@pytest.mark.parametrize("name", list(ALL))
def test_port_symbolic(port, name):
    nl, g = ALL[name](), golden(name)
    rp, col = port.pattern(nl, transient=True)
    assert np.array_equal(rp, g["rp_tran"]) and np.array_equal(col, g["col_tran"])
    rp, col = port.pattern(nl, transient=False)
    assert np.array_equal(rp, g["rp_dc"]) and np.array_equal(col, g["col_dc"])
    assert np.array_equal(port.stamp_map(nl), g["stamp_map"])
    mo, do = port.tensorize(nl)
    assert np.array_equal(mo, g["mos_order"]) and np.array_equal(do, g["dio_order"])
    raw, perm, tw = port.ordering(nl)
    assert np.array_equal(raw, g["raw_order"]) and np.array_equal(perm, g["perm_translated"])
    assert tw == int(g["treewidth"])
    sym = port.symbolic(nl)
    for k, gk in (("perm", "perm"), ("iperm", "iperm"), ("row_ptr", "f_row_ptr"), ("col", "f_col")):
        assert np.array_equal(sym[k], g[gk]), k
    assert sym["fill_in"] == int(g["fill_in"])


@pytest.mark.parametrize("name", list(ALL))
def test_port_stamps(port, name):
    nl, g = ALL[name](), golden(name)
    inst = instances_for(name, nl, g)
    vals, rhs = port.stamp(nl, g["probe_v"], inst, 0)
    assert np.array_equal(vals, g["stamp_dc_vals"]) and np.array_equal(rhs, g["stamp_dc_rhs"])
    if "stamp_tr_vals" in g:
        vals, rhs = port.stamp(nl, g["probe_v"], inst, 0, h=1e-12, method=A.TRAN_BE,
                               cap_vprev=g["cap_vprev"], t=2e-12)
        assert np.array_equal(vals, g["stamp_tr_vals"]) and np.array_equal(rhs, g["stamp_tr_rhs"])


@pytest.mark.parametrize("name", list(cases.SMALL) + ["config1"])
def test_port_dc(port, name):
    nl, g = ALL[name](), golden(name)
    v, st = port.solve_dc(nl)
    assert np.array_equal(stats_arr(st), g["dc_stats_ref_rule"])
    assert np.allclose(v, g["dc_v_ref_rule"], rtol=1e-12, atol=1e-15)
    v, st = port.solve_dc(nl, polish_max=8)
    assert np.array_equal(stats_arr(st), g["dc_stats"])
    assert np.allclose(v, g["dc_v"], rtol=1e-12, atol=1e-15)


def test_port_dc_config2(port):
    from oracle import pyoracle
    nl, g = circuits.config2(), golden("config2")
    inst = instances_for("config2", nl, g)
    for i in range(2):
        v, st = port.solve_dc(nl, inst, i, linear_solver=pyoracle.LS_SPARSE, polish_max=8)
        assert np.array_equal(stats_arr(st), g["dc_stats"][i])
        assert np.allclose(v, g["dc_v"][i], rtol=1e-12, atol=1e-15)


@pytest.mark.parametrize("name", ["diode_rc", "grid8", "config2"])
def test_port_transient(port, name):
    from oracle import pyoracle
    nl, g = ALL[name](), golden(name)
    inst = instances_for(name, nl, g)
    v0 = g["dc_v"][0] if name == "config2" else g["dc_v"]
    steps = 20 if name == "config2" else 40
    v, st, wave = port.transient(nl, v0, 1e-12, steps, A.TRAN_BE, inst, 0,
                                 wave_nodes=g["tran_wave_nodes"],
                                 linear_solver=pyoracle.LS_SPARSE if inst is not None else 0,
                                 polish_max=8)
    assert np.array_equal(stats_arr(st), g["tran_stats"])
    assert np.allclose(v, g["tran_v"], rtol=1e-12, atol=1e-15)
    assert np.allclose(wave, g["tran_wave"], rtol=1e-12, atol=1e-15)


def test_reference_build_reproduces_fixtures(ref):
    """Where the reference-built oracle exists, the fixtures are current."""
    nl, g = circuits.config1(), golden("config1")
    assert np.array_equal(ref.stamp_map(nl), g["stamp_map"])
    v, st = ref.solve_dc(nl)
    assert np.array_equal(stats_arr(st), g["dc_stats_ref_rule"])
    assert np.array_equal(v, g["dc_v_ref_rule"])


# ---------------------------------------------------------------------------
# product host symbolic layer (no device needed) vs the fixtures: bit-exact
# ---------------------------------------------------------------------------
@pytest.mark.parametrize("name", list(ALL))
def test_product_symbolic(product, name):
    nl, g = ALL[name](), golden(name)
    prob = product.Problem(None, nl)
    rp, col = prob.pattern()
    assert np.array_equal(rp, g["rp_tran"]) and np.array_equal(col, g["col_tran"])
    assert np.array_equal(prob.stamp_map(), g["stamp_map"])
    raw, perm, tw = prob.ordering()
    assert np.array_equal(raw, g["raw_order"]) and np.array_equal(perm, g["perm_translated"])
    assert tw == int(g["treewidth"])
    frp, fcol = prob.filled_pattern()
    assert np.array_equal(frp, g["f_row_ptr"]) and np.array_equal(fcol, g["f_col"])
    assert prob.info["fill_in"] == int(g["fill_in"])
    mo, do = prob.device_order()
    assert np.array_equal(mo, g["mos_order"]) and np.array_equal(do, g["dio_order"])


# ---------------------------------------------------------------------------
# larger grids of the uneven-batch family: bit-exact symbolic layer of the
# product, and the restatement's solutions, against the reference build
# ---------------------------------------------------------------------------
def grid_case(name):
    N = cases.GRIDS[name]
    g = golden(name)
    nl = circuits.grid_circuit(N)
    return nl, g, circuits.Instances(2, g["mc_kp"], g["mc_vto"])


@pytest.mark.parametrize("name", list(cases.GRIDS))
def test_product_symbolic_grids(product, name):
    nl, g, inst = grid_case(name)
    assert np.array_equal(inst.mos_kp, circuits.mc_instances(nl, 2).mos_kp)
    prob = product.Problem(None, nl)
    rp, col = prob.pattern()
    assert np.array_equal(rp, g["rp_tran"]) and np.array_equal(col, g["col_tran"])
    assert np.array_equal(prob.stamp_map(), g["stamp_map"])
    raw, perm, tw = prob.ordering()
    assert np.array_equal(raw, g["raw_order"]) and np.array_equal(perm, g["perm_translated"])
    assert tw == int(g["treewidth"])
    frp, fcol = prob.filled_pattern()
    assert np.array_equal(frp, g["f_row_ptr"]) and np.array_equal(fcol, g["f_col"])
    assert prob.info["fill_in"] == int(g["fill_in"])
    mo, do = prob.device_order()
    assert np.array_equal(mo, g["mos_order"]) and np.array_equal(do, g["dio_order"])


@pytest.mark.parametrize("name", ["grid16", "grid32"])
def test_port_grids(port, name):
    from oracle import pyoracle
    nl, g, inst = grid_case(name)
    raw, perm, tw = port.ordering(nl)
    assert np.array_equal(raw, g["raw_order"]) and np.array_equal(perm, g["perm_translated"])
    vals, rhs = port.stamp(nl, g["probe_v"], inst, 0)
    assert np.array_equal(vals, g["stamp_dc_vals"]) and np.array_equal(rhs, g["stamp_dc_rhs"])
    for i in range(2):
        v, st = port.solve_dc(nl, inst, i, linear_solver=pyoracle.LS_SPARSE, polish_max=8)
        assert np.array_equal(stats_arr(st), g["dc_stats"][i])
        assert np.allclose(v, g["dc_v"][i], rtol=1e-12, atol=1e-15)
    if name == "grid16":
        tr = cases.GRID_TRAN
        v, st, wave = port.transient(nl, g["dc_v"][0], tr["dt"], tr["steps"], A.TRAN_TRAP, inst, 0,
                                     wave_nodes=g["tran_wave_nodes"], linear_solver=pyoracle.LS_SPARSE,
                                     max_halvings=tr["max_halvings"], polish_max=8)
        assert np.array_equal(stats_arr(st), g["tran_stats"])
        assert np.allclose(wave, g["tran_wave"], rtol=1e-12, atol=1e-15)


def ac_inputs(name):
    g = np.load(os.path.join(HERE, "golden", f"ac_{name}.npz"))
    make, node, f0, f1, npts = cases.AC_CASES[name]
    nl = make()
    inst = circuits.Instances(2, g["mc_kp"], g["mc_vto"]) if "mc_kp" in g else None
    return g, nl, inst, (f0, f1, npts, node)


@pytest.mark.parametrize("name", sorted(cases.AC_CASES))
def test_port_ac_matches_reference_fixture(port, name):
    """The restated AC sweep (the NR Jacobian at the DC point + jwC, dense
    complex LU with partial pivoting) against the reference build's sweep of
    the same rule (its stamps, its solveComplexLU_Sparse), at the fixture's DC
    point: bit for bit."""
    g, nl, inst, (f0, f1, npts, node) = ac_inputs(name)
    x, sing = port.ac(nl, g["v_dc"], f0, f1, npts, node, inst=inst, idx=0)
    assert sing == int(g["singular"]) == 0
    assert np.array_equal(x, g["x_rule1"])


def test_ac_rule_equals_reference_build_where_they_coincide():
    """Without MOSFETs and with every diode forward-biased the reference's own
    admittance build (ACSolver::solveAC_Sparse as it stands) and the
    NR-Jacobian rule stamp the same matrix, and their sweeps agree to rounding
    (|dv| / (1e-9 |v| + 1e-12 V) below 1e-3);
    with MOSFETs (config 2) they differ, because the reference's build
    linearises every MOSFET with fixed NMOS parameters."""
    scaled = lambda g: np.max(np.abs(g["x_rule0"] - g["x_rule1"]) /
                              (1e-9 * np.abs(g["x_rule1"]) + 1e-12))
    g, *_ = ac_inputs("rc_ladder_diodes")
    assert scaled(g) < 1e-3  # the same stamps, summed in another order
    g, *_ = ac_inputs("config2")
    assert scaled(g) > 1.0


def test_lte_step_control_in_the_oracle(port, ref):
    """The LTE rule of the transient (the product's documented step control)
    runs in the oracle driver over both backends: over the gate ramp of the
    8 x 8 grid it redoes sub-steps, the restatement and the reference-built
    stamps take the same decisions and reach the same waveform, and with the
    rule off no step is halved."""
    nl = circuits.grid_circuit(8)
    v, _ = port.solve_dc(nl, polish_max=8)
    kw = dict(wave_nodes=[3, 10, 30], max_halvings=6, polish_max=8)
    vp, sp, wp = port.transient(nl, v, 40e-12, 20, A.TRAN_TRAP, lte_rel=1e-3, lte_abs=1e-4, **kw)
    vr, sr, wr = ref.transient(nl, v, 40e-12, 20, A.TRAN_TRAP, lte_rel=1e-3, lte_abs=1e-4, **kw)
    assert sp["converged"] == sr["converged"] == 1
    assert sp["lte_rejects"] == sr["lte_rejects"] > 0
    assert sp["halvings"] == sr["halvings"] and sp["iterations"] == sr["iterations"]
    assert np.max(np.abs(wp - wr)) <= 1e-9 * np.max(np.abs(wr)) + 1e-12
    _, s0, _ = port.transient(nl, v, 40e-12, 20, A.TRAN_TRAP, **kw)
    assert s0["lte_rejects"] == 0 and s0["halvings"] == 0


def test_kcl_residual_check_in_the_oracle(port):
    """The residual check the large mesh tiles are held to (Oracle.kcl_residual)
    accepts the oracle's own converged DC point and every backward-Euler step
    across the gates' edge of a 16 x 16 mesh tile (all nodes recorded per
    step), and rejects a point moved by 1e-6 relative, a step checked
    against the wrong previous point and one checked at the wrong time."""
    nl = circuits.power_grid_mesh(16)
    vd, st = port.solve_dc(nl, linear_solver=1, polish_max=8)
    assert st["converged"] == 1 and port.kcl_residual(nl, vd) < 1e-11
    assert port.kcl_residual(nl, vd * (1 + 1e-6)) > 1e-7
    dt, steps = 5e-12, 30
    _, s1, w = port.transient(nl, vd, dt, steps, A.TRAN_BE, wave_nodes=np.arange(1, nl.n_nodes + 1),
                              linear_solver=1, polish_max=8)
    assert s1["converged"] == 1 and s1["halvings"] == 0
    prev = vd
    for k in range(steps):
        assert port.kcl_residual(nl, w[k], h=dt, v_prev=prev, t=(k + 1) * dt) < 1e-11
        prev = w[k]
    assert np.max(np.abs(w[-1] - vd)) > 1e-3  # the loads switched on
    # the capacitor currents are small beside the 0.1-1 ohm segment currents
    assert port.kcl_residual(nl, w[-1], h=dt, v_prev=vd, t=steps * dt) > 1e-9
    assert port.kcl_residual(nl, w[-1], h=dt, v_prev=w[-2], t=dt) > 1e-7


@pytest.mark.parametrize("name", list(cases.MESH_ORDERINGS))
def test_product_ordering_mesh_tiles(product, name):
    """The product's Min-Fill (sparse adjacency, incremental fill counts) on
    power-grid mesh tiles equals the reference build's ordering bit for bit:
    64 x 64 (n = 4098) with its filled pattern, and 128 x 128 (n = 16386),
    whose fixture took the reference's own Min-Fill about 14 minutes."""
    g = golden(name)
    nl = circuits.power_grid_mesh(cases.MESH_ORDERINGS[name])
    assert nl.n_nodes == int(g["n"])
    prob = product.Problem(None, nl)
    raw, perm, tw = prob.ordering()
    assert np.array_equal(raw, g["raw_order"]) and np.array_equal(perm, g["perm_translated"])
    assert tw == int(g["treewidth"])
    if "filled_sha256" in g:
        frp, fcol = prob.filled_pattern()
        assert cases.filled_digest(frp, fcol) == str(g["filled_sha256"])
        assert prob.info["fill_in"] == int(g["fill_in"])
    prob.close()
