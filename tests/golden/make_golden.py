#!/usr/bin/env python
"""Generates the golden fixtures of the NR inner loop from the oracle library
compiled from the reference's own sources (oracle/_ref/libkaram_ref.so, built
by ``make -C oracle ref`` where the reference tree is present).

Every array comes from reference code: the stamp pattern and slot map
(MatrixConstructor::buildPattern / CachedCsrPattern::indexOf), the SoA order of
tensorizeNetlist, the Min-Fill ordering (FactorGraph + TreewidthAnalyzer), the
filled pattern of symbolicFactorize, the stamps of stampSoABlock, the NR
solutions of the oracle driver over those stamps and solveLU_Pivoted /
solveSparse_LU, PortableNormalDist draws, and AC sweeps solved by
solveComplexLU_Sparse (and by ACSolver::solveAC_Sparse as it stands).

    python tests/golden/make_golden.py          # rewrites tests/golden/*.npz
    python tests/golden/make_golden.py grid8    # only the named cases
    python tests/golden/make_golden.py grid64   # a large grid (minutes: dense-workspace LU)
    python tests/golden/make_golden.py ac_grid8 # one AC sweep fixture (ac_<case>)
    python tests/golden/make_golden.py mesh128  # a mesh tile's ordering (14 min: the reference's Min-Fill)
"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)
sys.path.insert(0, HERE)

import ctypes as C  # noqa: E402

import cases  # noqa: E402
from karam_b200 import _abi as A  # noqa: E402
from karam_b200 import circuits  # noqa: E402
from oracle import pyoracle  # noqa: E402

POLISH = dict(polish_max=8)
WAVE_NODES = {"config2": [2, 3, 4, 5, 10, 20, 259], "diode_rc": [1, 2, 3, 4],
              "grid8": [2, 3, 10, 30, 66]}


def probe_voltages(n, seed=11):
    return np.random.default_rng(seed).uniform(-0.2, 2.0, size=n)


def symbolic(ref, nl):
    out = {}
    out["rp_tran"], out["col_tran"] = ref.pattern(nl, transient=True)
    out["rp_dc"], out["col_dc"] = ref.pattern(nl, transient=False)
    out["stamp_map"] = ref.stamp_map(nl)
    out["mos_order"], out["dio_order"] = ref.tensorize(nl)
    raw, perm, tw = ref.ordering(nl)
    out["raw_order"], out["perm_translated"], out["treewidth"] = raw, perm, np.int32(tw)
    sym = ref.symbolic(nl)
    out["perm"], out["iperm"] = sym["perm"], sym["iperm"]
    out["f_row_ptr"], out["f_col"], out["fill_in"] = sym["row_ptr"], sym["col"], np.int32(sym["fill_in"])
    return out


def stamps(ref, nl, inst=None):
    n = nl.n_nodes
    v = probe_voltages(n)
    out = {"probe_v": v}
    out["stamp_dc_vals"], out["stamp_dc_rhs"] = ref.stamp(nl, v, inst, 0)
    if nl.cap:
        cv = np.linspace(-0.1, 0.3, len(nl.cap))
        out["cap_vprev"] = cv
        out["stamp_tr_vals"], out["stamp_tr_rhs"] = ref.stamp(nl, v, inst, 0, h=1e-12,
                                                              method=A.TRAN_BE, cap_vprev=cv,
                                                              t=2e-12)
    return out


def grid_fixture(ref, name, N):
    """Symbolic layer, probe stamps, DC of MC instances 0 and 1 and a
    trapezoidal waveform of instance 0 on the N x N grid, from the reference
    build; the linear solves use solveSparse_LU on the translated ordering."""
    nl = circuits.grid_circuit(N)
    inst = circuits.mc_instances(nl, 2)
    out = symbolic(ref, nl)
    out.update(stamps(ref, nl, inst))
    out["mc_kp"], out["mc_vto"] = inst.mos_kp, inst.mos_vto
    vs, sts = [], []
    for i in range(2):
        v, st = ref.solve_dc(nl, inst, i, linear_solver=pyoracle.LS_SPARSE, **POLISH)
        vs.append(v)
        sts.append(stats_arr(st))
    out["dc_v"], out["dc_stats"] = np.array(vs), np.array(sts)
    tr = cases.GRID_TRAN
    wave_nodes = cases.GRID_WAVE[N]
    vt, st, wave = ref.transient(nl, vs[0], tr["dt"], tr["steps"], A.TRAN_TRAP, inst, 0,
                                 wave_nodes=wave_nodes, linear_solver=pyoracle.LS_SPARSE,
                                 max_halvings=tr["max_halvings"], **POLISH)
    out["tran_v"], out["tran_stats"], out["tran_wave"] = vt, stats_arr(st), wave
    out["tran_wave_nodes"] = np.array(wave_nodes, np.int32)
    np.savez_compressed(os.path.join(HERE, f"{name}.npz"), **out)
    print(name, "n =", nl.n_nodes, "nnz =", len(out["col_tran"]), "dc stats",
          out["dc_stats"].tolist(), "tran stats", out["tran_stats"].tolist(), flush=True)


def mesh_ordering_fixture(ref, name, N):
    """Min-Fill ordering of an N x N power-grid mesh tile from the reference
    build (its ordering rescans every vertex per step: about 20 s at N = 64,
    14 min at N = 128), with the filled pattern's digest where it is cheap."""
    nl = circuits.power_grid_mesh(N)
    raw, perm, tw = ref.ordering(nl)
    out = dict(raw_order=raw, perm_translated=perm, treewidth=np.int32(tw), n=np.int32(nl.n_nodes))
    if name in cases.MESH_FILLED:
        sym = ref.symbolic(nl)
        out["filled_sha256"] = np.array(cases.filled_digest(sym["row_ptr"], sym["col"]))
        out["fill_in"] = np.int32(sym["fill_in"])
    np.savez_compressed(os.path.join(HERE, f"{name}.npz"), **out)
    print(name, "n =", nl.n_nodes, "treewidth", tw)


def ac_fixture(ref, name):
    """Small-signal AC sweep at a DC point, from the reference build: the
    NR-Jacobian rule (the reference's stamps at the DC point + jwC, solved by
    the reference's solveComplexLU_Sparse) and the reference's own admittance
    build (ACSolver::solveAC_Sparse as it stands)."""
    make, node, f0, f1, npts = cases.AC_CASES[name]
    nl = make()
    inst = circuits.mc_instances(nl, 2) if nl.n_mos else None
    v, st = ref.solve_dc(nl, inst, 0, linear_solver=pyoracle.LS_SPARSE, **POLISH)
    x1, s1 = ref.ac(nl, v, f0, f1, npts, node, inst=inst, idx=0, rule=1)
    x0, _ = ref.ac(nl, v, f0, f1, npts, node, inst=inst, idx=0, rule=0)
    out = dict(v_dc=v, dc_stats=stats_arr(st), x_rule1=x1, x_rule0=x0, singular=np.int64(s1),
               sweep=np.array([f0, f1, npts, node], np.float64))
    if inst is not None:
        out["mc_kp"], out["mc_vto"] = inst.mos_kp, inst.mos_vto
    np.savez_compressed(os.path.join(HERE, f"ac_{name}.npz"), **out)
    print(f"ac_{name}", "n =", nl.n_nodes, "dc", stats_arr(st).tolist(), "singular", s1, flush=True)


def stats_arr(st):
    keys = ("converged", "iterations", "polish_iters", "damped", "gmin_step", "singular")
    return np.array([st[k] for k in keys], np.int64)


def main():
    if not os.path.isdir(os.environ.get("KARAM_REFERENCE_TREE", "/root/reference")):
        sys.exit("the reference tree is needed to build the reference oracle")
    pyoracle.build("ref")
    ref = pyoracle.Oracle("ref")

    seeds = np.array(cases.RNG_SEEDS, np.uint64)
    if len(sys.argv) > 1:
        seeds = seeds[:0]
    normals = np.zeros((len(seeds), cases.RNG_COUNT))
    for k, s in enumerate(seeds):
        ref.lib.oracle_ref_normals.argtypes = [C.c_uint64, C.c_double, C.c_double, C.c_int32,
                                               C.POINTER(C.c_double)]
        ref.lib.oracle_ref_normals(int(s), 0.0, 1.0, cases.RNG_COUNT,
                                   normals[k].ctypes.data_as(C.POINTER(C.c_double)))
    if len(seeds):
        np.savez_compressed(os.path.join(HERE, "rng_normals.npz"), seeds=seeds, normals=normals)

    only = set(sys.argv[1:])  # case names to regenerate (default: all)
    for name in cases.AC_CASES:
        if only and f"ac_{name}" not in only:
            continue
        ac_fixture(ref, name)
    for name, N in cases.GRIDS.items():
        if only and name not in only:
            continue
        grid_fixture(ref, name, N)
    for name, N in cases.MESH_ORDERINGS.items():
        if only and name not in only:
            continue
        mesh_ordering_fixture(ref, name, N)
    for name, make in {**cases.SMALL, **cases.BENCH}.items():
        if only and name not in only:
            continue
        nl = make()
        inst = circuits.mc_instances(nl, 2) if name == "config2" else None
        out = symbolic(ref, nl)
        out.update(stamps(ref, nl, inst))
        if name == "config2":
            out["mc_kp"], out["mc_vto"] = inst.mos_kp, inst.mos_vto
            vs, sts = [], []
            for i in range(2):
                v, st = ref.solve_dc(nl, inst, i, linear_solver=pyoracle.LS_SPARSE, **POLISH)
                vs.append(v)
                sts.append(stats_arr(st))
            out["dc_v"], out["dc_stats"] = np.array(vs), np.array(sts)
            vt, st, wave = ref.transient(nl, vs[0], 1e-12, 20, A.TRAN_BE, inst, 0,
                                         wave_nodes=WAVE_NODES[name],
                                         linear_solver=pyoracle.LS_SPARSE, **POLISH)
            out["tran_v"], out["tran_stats"], out["tran_wave"] = vt, stats_arr(st), wave
            out["tran_wave_nodes"] = np.array(WAVE_NODES[name], np.int32)
        else:
            v, st = ref.solve_dc(nl)
            out["dc_v_ref_rule"], out["dc_stats_ref_rule"] = v, stats_arr(st)
            v, st = ref.solve_dc(nl, **POLISH)
            out["dc_v"], out["dc_stats"] = v, stats_arr(st)
            if name in WAVE_NODES:
                vt, st, wave = ref.transient(nl, v, 1e-12, 40, A.TRAN_BE,
                                             wave_nodes=WAVE_NODES[name], **POLISH)
                out["tran_v"], out["tran_stats"], out["tran_wave"] = vt, stats_arr(st), wave
                out["tran_wave_nodes"] = np.array(WAVE_NODES[name], np.int32)
        np.savez_compressed(os.path.join(HERE, f"{name}.npz"), **out)
        print(name, "n =", nl.n_nodes, "nnz =", len(out["col_tran"]),
              "dc stats", out["dc_stats"].tolist())


if __name__ == "__main__":
    main()
