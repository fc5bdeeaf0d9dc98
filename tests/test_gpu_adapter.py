"""The reference-side adapter (karam_b200/adapter/karam_adapter.cpp), compiled
against the reference's headers with its AnalysisRegistry and linked to the
product library (oracle/Makefile, target adapter): a config-1 netlist becomes a
reference TensorNetlist through the reference's adders, and its DC point and a
backward-Euler transient come back as SolverStep / SimulationResponseDTO
through CircuitSim::solveDC's replacement and through the registry handlers
it registers. Both follow the oracle's NR path (the same iteration count under
the reference stopping rule) to the oracle's voltages."""
import ctypes as C
import os
import sys

import numpy as np
import pytest

from karam_b200 import _abi as A
from karam_b200 import circuits

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, os.path.join(ROOT, "tests", "golden"))
LIB = os.path.join(ROOT, "oracle", "_ref", "libkaram_adapter.so")
P = C.POINTER


@pytest.fixture(scope="module")
def adapter(product):
    if not os.path.exists(LIB):
        pytest.skip("the adapter library is built where the reference tree is present")
    lib = C.CDLL(LIB)
    lib.adapter_test_dc.argtypes = [C.c_void_p, C.c_int32, P(C.c_double), P(C.c_int32),
                                    P(C.c_int32), P(C.c_int32), C.c_char_p]
    lib.adapter_test_tran.argtypes = [C.c_void_p, C.c_double, C.c_int32, P(C.c_double),
                                      P(C.c_int32), C.c_char_p]
    return lib


def test_registry_serves_dc_transient_and_mc(adapter):
    assert adapter.adapter_test_registered() == 1


@pytest.mark.parametrize("via_registry", [0, 1])
def test_adapter_dc_matches_oracle(adapter, port, via_registry):
    nl = circuits.config1()
    s = nl.as_struct()
    v = np.zeros(nl.n_nodes)
    n, its, conv = C.c_int32(), C.c_int32(), C.c_int32()
    err = C.create_string_buffer(256)
    rc = adapter.adapter_test_dc(C.cast(C.pointer(s), C.c_void_p), via_registry,
                                 v.ctypes.data_as(P(C.c_double)), C.byref(n), C.byref(its),
                                 C.byref(conv), err)
    assert rc == 0, err.value.decode()
    v_ref, st_ref = port.solve_dc(nl)  # the reference stopping rule, as the adapter's defaults
    assert conv.value == 1 and n.value == nl.n_nodes
    assert its.value == st_ref["iterations"]
    assert np.max(np.abs(v - v_ref) / (1e-6 * np.abs(v_ref) + 1e-9)) <= 1.0


def test_adapter_transient_matches_oracle(adapter, port):
    """A PULSE-driven diode clamp with node capacitors (the diode_rc fixture
    circuit), 20 backward-Euler steps of 1 ps through the TRANSIENT handler."""
    import cases
    nl = cases.diode_rc()
    s = nl.as_struct()
    steps, dt = 20, 1e-12
    wave = np.zeros((steps, nl.n_nodes))
    conv = C.c_int32()
    err = C.create_string_buffer(256)
    rc = adapter.adapter_test_tran(C.cast(C.pointer(s), C.c_void_p), dt, steps,
                                   wave.ctypes.data_as(P(C.c_double)), C.byref(conv), err)
    assert rc == 0, err.value.decode()
    assert conv.value == 1
    v0, _ = port.solve_dc(nl)
    nodes = list(range(1, nl.n_nodes + 1))
    _, st, w_ref = port.transient(nl, v0, dt, steps, A.TRAN_BE, wave_nodes=nodes)
    assert st["converged"] == 1
    assert np.max(np.abs(wave - w_ref) / (1e-6 * np.abs(w_ref) + 1e-9)) <= 1.0
