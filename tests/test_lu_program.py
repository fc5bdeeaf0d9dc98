"""The static-pivot LU program of the host symbolic layer (value slots on the
reference's Min-Fill ordering), executed on the CPU with numpy: on any matrix
whose non-zeros lie on the value slots, it must reproduce a dense solve.
This pins the slot structure, the fill the program creates and the fused
forward substitution the device kernels run."""
import os
import sys

import numpy as np
import pytest

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(HERE, "golden"))

import cases  # noqa: E402

ALL = {**cases.SMALL, **cases.BENCH}


def run_program(hdr, data, vals, rhs):
    A = vals.copy()
    y = rhs.copy()
    n = len(hdr)
    for k in range(n):
        off, nl, nu, d = (int(v) for v in hdr[k])
        lr = data[off:off + nl]
        ls = data[off + nl:off + 2 * nl]
        us = data[off + 2 * nl + nu:off + 2 * nl + 2 * nu]
        tt = data[off + 2 * nl + 2 * nu:off + 2 * nl + 2 * nu + nl * nu].reshape(nl, nu)
        r = 1.0 / A[d]
        A[d] = r
        for a in range(nl):
            l = A[ls[a]] * r
            A[ls[a]] = l
            y[lr[a]] -= l * y[k]
            for b in range(nu):
                A[tt[a, b]] -= l * A[us[b]]
    for k in range(n - 1, -1, -1):
        off, nl, nu, d = (int(v) for v in hdr[k])
        uc = data[off + 2 * nl:off + 2 * nl + nu]
        us = data[off + 2 * nl + nu:off + 2 * nl + 2 * nu]
        s = y[k] - np.dot(A[us], y[uc])
        y[k] = s * A[d]
    return y


@pytest.mark.parametrize("name", list(ALL))
def test_program_solves_matrices_on_its_slots(product, name):
    nl = ALL[name]()
    prob = product.Problem(None, nl)
    hdr, data, rc = prob.lu_program()
    n, nv = prob.n, prob.info["n_slots"]
    assert rc.shape == (nv, 2) and (rc >= 0).all() and (rc < n).all()
    # every slot is a position of the filled pattern (permuted space)
    frp, fcol = prob.filled_pattern()
    filled = {(i, int(c)) for i in range(n) for c in fcol[frp[i]:frp[i + 1]]}
    assert all((int(r), int(c)) in filled for r, c in rc)
    # diagonals are slots and every pivot's diagonal slot is (k, k)
    assert all(tuple(rc[hdr[k, 3]]) == (k, k) for k in range(n))
    rng = np.random.default_rng(3)
    for _ in range(3):
        vals = rng.uniform(-1.0, 1.0, nv)
        dense = np.zeros((n, n))
        dense[rc[:, 0], rc[:, 1]] = vals
        # diagonal dominance keeps the static pivots well conditioned
        for k in range(n):
            s = hdr[k, 3]
            vals[s] = np.sign(vals[s] or 1.0) * (1.0 + np.abs(dense[k]).sum() + np.abs(dense[:, k]).sum())
        dense[rc[:, 0], rc[:, 1]] = vals
        rhs = rng.uniform(-1.0, 1.0, n)
        x = run_program(hdr, data, vals, rhs)
        ref = np.linalg.solve(dense, rhs)
        assert np.allclose(x, ref, rtol=1e-10, atol=1e-12)


def test_program_size_matches_info(product):
    prob = product.Problem(None, cases.BENCH["config2"]())
    hdr, data, _ = prob.lu_program()
    ops = sum(int(nl) + int(nl) * int(nu) for _, nl, nu, _ in hdr)
    assert ops == prob.info["lu_ops"]
    # chain circuits: every pivot is small (the packed-record schedule applies)
    assert hdr[:, 1].max() <= 2 and hdr[:, 2].max() <= 2
