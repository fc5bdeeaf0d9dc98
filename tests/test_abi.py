"""The C ABI without a device: the library loads, exports exactly what
include/karam.h declares, and reports errors as status codes with messages
(no exceptions cross the boundary). No compute call is made here."""
import ctypes as C
import os
import re
import subprocess

import numpy as np
import pytest

from karam_b200 import _abi as A
from karam_b200 import circuits

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HEADER = os.path.join(ROOT, "include", "karam.h")


def declared():
    text = open(HEADER).read()
    return sorted(set(re.findall(r"KARAM_API\s+[^;(]*?\b(karam_\w+)\s*\(", text)))


def test_header_declares_the_entry_points():
    names = declared()
    for must in ("karam_ctx_create", "karam_problem_create", "karam_solve_dc",
                 "karam_step_transient", "karam_run_mc", "karam_last_error"):
        assert must in names


def test_library_exports_every_declared_symbol(product):
    lib = product.lib()
    for name in declared():
        assert hasattr(lib, name), f"{name} declared in karam.h but not exported"
    out = subprocess.run(["nm", "-D", "--defined-only", lib._name], capture_output=True,
                         text=True, check=True).stdout
    exported = sorted(set(re.findall(r"\bT (karam_\w+)", out)))
    assert exported == declared(), "exported karam_* symbols differ from the header"
    # everything else stays hidden (-fvisibility=hidden)
    others = [s for s in re.findall(r"\b[TW] (\S+)", out) if not s.startswith("karam_")]
    assert not [s for s in others if "knr" in s or "Topology" in s], others[:5]


def test_default_opts_follow_the_reference_solver(product):
    o = A.KaramSolverOpts()
    product.lib().karam_default_opts(C.byref(o))
    # circuitsim_solver.cpp: 50 NR iterations per GMIN step, 19 half-decade
    # GMIN steps; RELTOL/VNTOL circuitsim.h:1206-1207; KCL 1e-9 shortcut and
    # KCL_TOL 1e-12 (physics_constants.h:76)
    assert o.max_nr_iter == 50 and o.gmin_steps == 19
    assert o.reltol == 1e-3 and o.vntol == 1e-6
    assert o.kcl_shortcut == 1e-9 and o.kcl_tol == 1e-12


def test_context_without_device_is_an_error(product):
    import torch
    if torch.cuda.is_available():
        pytest.skip("a device is present")
    lib = product.lib()
    h = C.c_void_p()
    rc = lib.karam_ctx_create(0, C.byref(h))
    assert rc == A.KARAM_E_CUDA
    assert lib.karam_last_error(None)


def _bad(product, nl, expect=A.KARAM_E_INVALID):
    lib = product.lib()
    s = nl.as_struct()
    h = C.c_void_p()
    rc = lib.karam_problem_create(None, C.byref(s), 1, C.byref(h))
    assert rc == expect, rc
    msg = lib.karam_last_error(None).decode()
    assert msg
    return msg


def test_malformed_netlists_are_rejected(product):
    nl = circuits.Netlist()
    nl.vsource(1, 0, 1.0)
    nl.resistor(1, 0, 1e3)
    nl.res[0] = (1, -2, 1e3)  # negative node id
    _bad(product, nl)
    nl = circuits.Netlist()
    nl.vsource(1, 0, 1.0)
    nl.resistor(1, 0, 0.0)  # zero resistance
    _bad(product, nl)
    nl = circuits.Netlist()
    nl.vsource(1, 0, 1.0)
    nl.mosfet(1, 1, 0, 0, 3, 1e-6, 1e-6)  # unknown model card
    _bad(product, nl)
    empty = circuits.Netlist()
    _bad(product, empty)


def test_node_count_follows_the_highest_node_id(product):
    """As tensorizeNetlist does, the unknowns run up to the highest node id
    any device names, even past the declared node count."""
    nl = circuits.Netlist()
    nl.vsource(1, 0, 1.0)
    nl.resistor(1, 0, 1e3)
    nl.res[0] = (1, 5, 1e3)
    assert product.Problem(None, nl).info["n"] == 5


def test_null_arguments_are_rejected(product):
    lib = product.lib()
    h = C.c_void_p()
    assert lib.karam_problem_create(None, None, 1, C.byref(h)) == A.KARAM_E_INVALID
    assert lib.karam_problem_info_get(None, None) == A.KARAM_E_INVALID
    assert lib.karam_solve_dc(None, None, None, None, None) == A.KARAM_E_INVALID


def test_symbolic_problem_refuses_solves(product):
    """A problem made without a context holds no device memory: solves fail
    with a status, symbolic queries work."""
    prob = product.Problem(None, circuits.config1())
    assert prob.info["n"] == 34 and prob.info["nnz"] == 131
    with pytest.raises(product.KaramError) as e:
        prob.solve_dc()
    assert e.value.code == A.KARAM_E_STATE


def test_instances_are_validated(product):
    nl = circuits.config1()
    prob = product.Problem(None, nl)
    bad = circuits.Instances(2, np.zeros((2, 3), np.float32), np.zeros((2, 3), np.float32))
    with pytest.raises(product.KaramError):
        prob.set_instances(bad)
