"""A SPICE netlist solved on the GPU through the C ABI equals the same
circuit built programmatically, and matches the oracle."""
import numpy as np
import pytest

from karam_b200 import _abi as A
from karam_b200 import circuits

pytestmark = pytest.mark.gpu


def grid_text(N=6):
    nl = circuits.grid_circuit(N)  # the builder's values, written out exactly
    lines = ["grid as SPICE", f"V1 n1 0 {nl.vsrc[0][2]!r}",
             "V2 n2 0 PULSE(" + " ".join(repr(x) for x in nl.vsrc[1][4]) + ")"]
    for k, (a, b, ohm) in enumerate(nl.res):
        lines.append(f"R{k} n{a} n{b} {ohm!r}")
    for k, (a, b, f) in enumerate(nl.cap):
        lines.append(f"C{k} n{a} {'0' if b == 0 else 'n' + str(b)} {f!r}")
    for k, d in enumerate(nl.dio):
        lines.append(f"D{k} 0 n{d[1]} dclamp")
    for k, m in enumerate(nl.mos):
        lines.append(f"M{k} n{m[0]} n{m[1]} 0 0 NMOS W={m[4]!r} L={m[5]!r}")
    lines += [".model dclamp D(IS=1e-14 N=1)",
              f".model NMOS NMOS(KP={circuits.NMOS_CARD['kp']!r} VTO={circuits.NMOS_CARD['vto']!r} "
              f"LAMBDA={circuits.NMOS_CARD['lam']!r})", ".end"]
    return nl, "\n".join(lines)


@pytest.mark.parametrize("prec", [A.PREC_FP64, A.PREC_MIXED])
def test_spice_grid_solves_like_the_builder(product, ctx, port, prec):
    nl, text = grid_text()
    sp = product.parse_spice(text)
    # node names n1..n38 appear in an order of their own: map them back
    idx = np.array([sp.node(f"n{k}") for k in range(1, nl.n_nodes + 1)]) - 1
    opts = product.options(precision=prec, polish_max=8)
    a = product.Problem(ctx, sp, max_instances=1)
    a.set_instances(None)
    va, sa = a.solve_dc(opts)
    b = product.Problem(ctx, nl, max_instances=1)
    b.set_instances(None)
    vb, sb = b.solve_dc(opts)
    assert sa[0]["status"] == A.ST_CONVERGED and sb[0]["status"] == A.ST_CONVERGED
    assert np.max(np.abs(va[0][idx] - vb[0]) / (1e-9 * np.abs(vb[0]) + 1e-12)) <= 1.0
    v_ref, st_ref = port.solve_dc(sp, polish_max=8)
    assert np.max(np.abs(va[0] - v_ref) / (1e-9 * np.abs(v_ref) + 1e-12)) <= 1.0
