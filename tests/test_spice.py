"""The SPICE front-end (karam_spice_parse): netlists written as SPICE text
equal the programmatic builders' array for array, and so do their symbolic
analyses and oracle solutions; the reference parser's defects (W= / L=
dropped, diode cards ignored, case-sensitive model lookup, SIN vs SINE) are
fixed; elements the engine cannot solve are errors."""
import numpy as np
import pytest

from karam_b200 import _abi as A
from karam_b200 import circuits


def chain_text(stages=32, vin="0.9", extra=""):
    lines = ["* 32-stage CMOS inverter chain", "V1 vdd 0 DC 1.8", f"V2 in 0 {vin}"]
    prev = "in"
    for k in range(stages):
        out = f"n{k + 1}"
        lines.append(f"Mp{k} {out} {prev} vdd vdd pmos W=4e-6 L=0.18e-6")
        lines.append(f"Mn{k} {out} {prev} 0 0 nmos w=2e-6 l=0.18e-6")
        prev = out
    # exponent notation: "110u" is 110 * 1e-6, one rounding away from 110e-6
    lines += [".model NMOS nmos (kp=110e-6 vto=0.7 lambda=0.04)",
              ".MODEL PMOS PMOS KP=40E-6 VTO=-0.7", "+ LAMBDA=0.05", extra, ".op", ".end"]
    return "\n".join(lines)


FIELDS_I = ["vs_pos", "vs_neg", "vs_kind", "is_pos", "is_neg", "r_n1", "r_n2", "c_n1", "c_n2",
            "d_anode", "d_cathode", "d_model", "m_d", "m_g", "m_s", "m_b", "m_model", "model_type"]
FIELDS_D = ["vs_dc", "vs_pulse", "is_amp", "r_ohm", "c_farad", "d_is", "d_n", "d_vt", "m_w", "m_l",
            "model_kp", "model_vto", "model_lambda"]
COUNT = {"vs": "n_vsrc", "is": "n_isrc", "r": "n_res", "c": "n_cap", "d": "n_dio", "m": "n_mos",
         "model": "n_models"}


def arrays(s):
    out = {"n_nodes": s.n_nodes, "temp_k": s.temp_k}
    for f in FIELDS_I + FIELDS_D:
        n = getattr(s, COUNT[f.rsplit("_", 1)[0] if not f.startswith("model") else "model"])
        if f == "vs_pulse":
            n *= 7
        p = getattr(s, f)
        out[f] = np.array([p[i] for i in range(n)]) if (n and p) else np.zeros(0)
    out["names"] = [s.model_name[i].decode() for i in range(s.n_models)]
    return out


def same(a, b):
    for k in a:
        if isinstance(a[k], np.ndarray):
            assert a[k].shape == b[k].shape and np.array_equal(a[k], b[k], equal_nan=True), k
        else:
            assert a[k] == b[k], k


def test_config1_text_equals_builder(product):
    sp = product.parse_spice(chain_text())
    ref = circuits.config1()  # alive while its struct is read
    same(arrays(sp.as_struct()), arrays(ref.as_struct()))
    assert sp.node("VDD") == 1 and sp.node("In") == 2 and sp.node("n32") == 34
    assert sp.node("gnd") == 0 and sp.node("nowhere") == -1
    assert sp.analysis()[0] is True


def test_config1_text_symbolic_and_oracle(product, port):
    sp = product.parse_spice(chain_text())
    ref = circuits.config1()
    a, b = product.Problem(None, sp), product.Problem(None, ref)
    for q in ("pattern", "ordering", "filled_pattern", "stamp_map"):
        x, y = getattr(a, q)(), getattr(b, q)()
        x, y = (x, y) if isinstance(x, tuple) else ((x,), (y,))
        for xi, yi in zip(x, y):
            assert np.array_equal(np.asarray(xi), np.asarray(yi)), q
    v1, st1 = port.solve_dc(sp)
    v2, st2 = port.solve_dc(ref)
    assert np.array_equal(v1, v2) and st1["iterations"] == st2["iterations"]


def test_clamped_chain_with_pulse_equals_config2(product):
    lines = ["config 2", "V1 vdd 0 1.8", "V2 in 0 PULSE(0 1.8 0 200e-12 200e-12 1e-9 0)"]
    prev = "in"
    for k in range(256):
        out = f"o{k}"
        lines += [f"MP{k} {out} {prev} vdd vdd PMOS W=4e-6 L=0.18e-6",
                  f"MN{k} {out} {prev} 0 0 NMOS W=2e-6 L=0.18e-6"]
        prev = out
    for j in range(64):
        lines += [f"RS{j} o{(j + 1) * 4 - 1} c{j} 10", f"D{j} 0 c{j} dclamp"]
    for k in range(256):
        lines.append(f"C{k} o{k} 0 1e-15")
    for j in range(64):
        lines.append(f"CC{j} c{j} 0 1e-15")
    lines += [".model dclamp D(IS=1e-14 N=1)", ".model nmos NMOS(KP=110e-6 VTO=0.7 LAMBDA=0.04)",
              ".model pmos PMOS(KP=40e-6 VTO=-0.7 LAMBDA=0.05)", ".tran 1p 200p", ".end"]
    sp = product.parse_spice("\n".join(lines))
    ref = circuits.config2()
    got, want = arrays(sp.as_struct()), arrays(ref.as_struct())
    # the builder's diodes carry no model card (index -1, "diode_generic"); the
    # parsed ones name theirs, so the model tables differ by that card only
    assert got["names"] == ["dclamp", "nmos", "pmos"] and want["names"] == ["NMOS", "PMOS"]
    assert np.array_equal(got["m_model"] - 1, want["m_model"])
    for k in list(got):
        if k in ("names", "m_model", "d_model", "model_type", "model_kp", "model_vto",
                 "model_lambda"):
            continue
        if isinstance(got[k], np.ndarray):
            assert np.array_equal(got[k], want[k], equal_nan=True), k
        else:
            assert got[k] == want[k], k
    assert sp.analysis()[1] is True
    assert sp.analysis()[2:4] == pytest.approx((1e-12, 200e-12), rel=1e-15)


def test_reference_parser_defects_fixed(product):
    sp = product.parse_spice("\n".join([
        "defects", "V1 a 0 1", "R1 a b 1k", "D1 b 0 MyDiode", "M1 b a 0 0 Nch W=3u L=0.5u",
        ".MODEL mydiode D IS=2e-15 N=1.5", ".model NCH nmos KP=1e-4", ".temp 50", ".end"]))
    s = sp.as_struct()
    assert (s.d_is[0], s.d_n[0], s.d_vt[0]) == (2e-15, 1.5, 0.02585)  # diode card applied
    assert (s.m_w[0], s.m_l[0]) == (3e-6, 0.5e-6)                     # W= / L= read
    assert s.model_name[s.m_model[0]].decode() == "NCH"               # case-insensitive
    assert np.isnan(s.model_vto[s.m_model[0]]) and s.model_kp[s.m_model[0]] == 1e-4
    assert s.temp_k == pytest.approx(323.15)


@pytest.mark.parametrize("line, msg", [
    ("V2 a 0 SIN(0 1 1meg)", "SIN sources"),
    ("V2 a 0 SINE(0 1 1meg)", "SIN sources"),
    ("L1 a 0 1n", "not supported"),
    ("E1 a 0 b 0 2", "not supported"),
    ("I1 a 0 PULSE(0 1m 0 1n 1n 5n 10n)", "current sources"),
    ("M1 a a 0 0 undefined", "'UNDEFINED' is not defined"),
    ("R9 a", "too few fields"),
])
def test_unsupported_input_is_an_error(product, line, msg):
    text = "\n".join(["t", "V1 a 0 1", "R1 a 0 1k", line, ".model N nmos", ".end"])
    with pytest.raises(product.KaramError, match=msg):
        product.parse_spice(text)
    with pytest.raises(product.KaramError, match="line 4"):
        product.parse_spice(text)


def test_values_and_continuations(product):
    sp = product.parse_spice("\n".join([
        "units", "R1 a 0 1meg ; inline comment", "R2 a b 10k", "* comment line", "R3 b 0 2.5",
        "+", "C1 b 0 2.5pF", "C2 a 0 1mil", "V1 a 0 DC 1.2 AC 1 0", "I1 0 b 3mA", ".end"]))
    s = sp.as_struct()
    assert [s.r_ohm[i] for i in range(3)] == [1e6, 1e4, 2.5]
    assert s.c_farad[0] == pytest.approx(2.5e-12) and s.c_farad[1] == pytest.approx(25.4e-6)
    assert s.vs_dc[0] == 1.2 and s.is_amp[0] == pytest.approx(3e-3)
    assert s.n_nodes == 2
