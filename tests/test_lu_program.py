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


def run_records(rec, rec2, vals, rhs):
    """The device's packed-record schedule: a chain pivot takes its L value,
    second target and L-row right-hand side from the previous pivot's
    registers instead of memory; the back substitution takes the unknown the
    previous step solved from a register where the forwarding bit says so."""
    A = vals.copy()
    y = rhs.copy()
    n = len(rec)

    def load(k):
        meta, d, ls, lr, us0, us1, t0, t1 = (int(v) for v in rec[k])
        chain, nl, nu = (meta >> 8) & 1, meta & 15, (meta >> 4) & 15
        return dict(piv=A[d], yk=y[k], u0=A[us0] if nu > 0 else 0.0,
                    u1=A[us1] if nu > 1 else 0.0, b00=A[t0] if nl and nu else 0.0,
                    a0=A[ls] if nl and not chain else 0.0, y0=y[lr] if nl and not chain else 0.0,
                    b01=A[t1] if nl and nu > 1 and not chain else 0.0)

    w00 = w01 = wy0 = 0.0
    cur = load(0)
    for k in range(n):
        meta, d, ls, lr, us0, us1, t0, t1 = (int(v) for v in rec[k])
        chain, nl, nu = (meta >> 8) & 1, meta & 15, (meta >> 4) & 15
        a0 = w00 if chain else cur["a0"]
        y0 = wy0 if chain else cur["y0"]
        b01 = w01 if chain else cur["b01"]
        r = 1.0 / cur["piv"]
        A[d] = r
        if nl:
            l = a0 * r
            wy0 = y0 - l * cur["yk"]
            y[lr] = wy0
            if nu > 0:
                w00 = cur["b00"] - l * cur["u0"]
                A[t0] = w00
            if nu > 1:
                w01 = b01 - l * cur["u1"]
                A[t1] = w01
        if k + 1 < n:
            cur = load(k + 1)

    def bvals(k):
        meta, d, ls, lr, us0, us1, t0, t1 = (int(v) for v in rec[k])
        nu, fb = (meta >> 4) & 15, (meta >> 9) & 3
        c0, c1 = (int(v) for v in rec2[k])
        return dict(yk=y[k], u0=A[us0] if nu > 0 else 0.0, u1=A[us1] if nu > 1 else 0.0,
                    x0=y[c0] if nu > 0 and not fb & 1 else 0.0,
                    x1=y[c1] if nu > 1 and not fb & 2 else 0.0, r=A[d])

    yprev = 0.0
    for k in range(n - 1, -1, -1):
        cur = bvals(k)
        meta = int(rec[k][0])
        nu, fb = (meta >> 4) & 15, (meta >> 9) & 3
        sv = cur["yk"]
        if nu > 0:
            sv -= cur["u0"] * (yprev if fb & 1 else cur["x0"])
        if nu > 1:
            sv -= cur["u1"] * (yprev if fb & 2 else cur["x1"])
        sv *= cur["r"]
        y[k] = sv
        yprev = sv
    return y


@pytest.mark.parametrize("name", list(ALL))
def test_packed_records_schedule_solves(product, name):
    nl = ALL[name]()
    prob = product.Problem(None, nl)
    recs = prob.lu_records()
    if recs is None:
        pytest.skip("program has pivots beyond the packed-record shape")
    rec, rec2 = recs
    hdr, _, rc = prob.lu_program()
    n, nv = prob.n, prob.info["n_slots"]
    assert (rec[:, 1] == hdr[:, 3]).all()
    rng = np.random.default_rng(5)
    for _ in range(3):
        vals = rng.uniform(-1.0, 1.0, nv)
        dense = np.zeros((n, n))
        dense[rc[:, 0], rc[:, 1]] = vals
        for k in range(n):
            s = hdr[k, 3]
            vals[s] = np.sign(vals[s] or 1.0) * (1.0 + np.abs(dense[k]).sum() + np.abs(dense[:, k]).sum())
        dense[rc[:, 0], rc[:, 1]] = vals
        rhs = rng.uniform(-1.0, 1.0, n)
        x = run_records(rec, rec2, vals, rhs)
        assert np.allclose(x, np.linalg.solve(dense, rhs), rtol=1e-10, atol=1e-12)
    if name == "config2":
        # nearly every pivot of the chain circuit keeps the recurrence in registers
        assert int(((rec[:, 0] >> 8) & 1).sum()) >= n // 2


def run_schedule(sch, vals_nd, rhs_nd):
    """The level schedule as the factor/solve kernel runs it, one level at a
    time: pivot reciprocals, L values, update targets and right-hand-side rows,
    then the back substitution from the last level down."""
    A = vals_nd.copy()
    y = rhs_nd.copy()
    lp, diag = sch["lv_piv_ptr"], sch["nd_diag"]
    for lv in range(sch["levels"]):
        piv = sch["lv_piv"][lp[lv]:lp[lv + 1]]
        A[diag[piv]] = 1.0 / A[diag[piv]]
        e0, e1 = sch["lv_l_ptr"][lv], sch["lv_l_ptr"][lv + 1]
        ls = sch["l_slot"][e0:e1]
        A[ls] = A[ls] * A[diag[sch["l_piv"][e0:e1]]]
        for t in range(sch["lv_ts_ptr"][lv], sch["lv_ts_ptr"][lv + 1]):
            q0, q1 = sch["t_off"][t], sch["t_off"][t + 1]
            A[sch["t_slot"][t]] -= np.dot(A[sch["pr_l"][q0:q1]], A[sch["pr_u"][q0:q1]])
        for r in range(sch["lv_ys_ptr"][lv], sch["lv_ys_ptr"][lv + 1]):
            q0, q1 = sch["y_off"][r], sch["y_off"][r + 1]
            y[sch["y_row"][r]] -= np.dot(A[sch["yp_l"][q0:q1]], y[sch["yp_k"][q0:q1]])
    for lv in range(sch["levels"] - 1, -1, -1):
        for k in sch["lv_piv"][lp[lv]:lp[lv + 1]]:
            b0, b1 = sch["bs_off"][k], sch["bs_off"][k + 1]
            y[k] = (y[k] - np.dot(A[sch["bs_u"][b0:b1]], y[sch["bs_c"][b0:b1]])) * A[diag[k]]
    return y


@pytest.mark.parametrize("name", list(ALL))
def test_level_schedule_solves(product, name):
    nl = ALL[name]()
    prob = product.Problem(None, nl)
    sch = prob.lu_schedule()
    if sch is None:
        pytest.skip("no level schedule")
    hdr, _, rc = prob.lu_program()
    n, nv = prob.n, prob.info["n_slots"]
    perm = sch["nd_perm"]
    assert sorted(perm) == list(range(n)) and sch["n"] == n
    # the long-list threshold splits every level's targets and rows
    assert (sch["lv_ts_ptr"][1:] >= sch["lv_tl_ptr"][:-1]).all()
    # no pivot of a level writes what another pivot of the same level reads
    level = np.zeros(n, int)
    for lv in range(sch["levels"]):
        level[sch["lv_piv"][sch["lv_piv_ptr"][lv]:sch["lv_piv_ptr"][lv + 1]]] = lv
    owner = np.repeat(np.arange(n), np.diff(sch["bs_off"]))
    assert (level[sch["bs_c"]] > level[owner]).all()  # U columns are solved in later levels
    # the ND structure holds every stamped position; Min-Fill slots outside
    # it are fill of the Min-Fill order that no stamp reaches, zero in every
    # Jacobian (the evaluation kernel writes them as 0)
    src = sch["nd_src"]
    covered = np.zeros(nv, bool)
    covered[src[src >= 0]] = True
    _, perm_mf, _ = prob.ordering()
    iperm = np.empty(n, int)
    iperm[perm_mf] = np.arange(n)
    rp, col = prob.pattern()
    slot_of = {(int(r), int(c)): s for s, (r, c) in enumerate(rc)}
    for r in range(n):
        for c in col[rp[r]:rp[r + 1]]:
            assert covered[slot_of[(iperm[r], iperm[c])]]
    rng = np.random.default_rng(9)
    for _ in range(3):
        vals = np.where(covered, rng.uniform(-1.0, 1.0, nv), 0.0)
        dense = np.zeros((n, n))
        dense[rc[:, 0], rc[:, 1]] = vals
        for k in range(n):
            s = hdr[k, 3]
            vals[s] = np.sign(vals[s] or 1.0) * (1.0 + np.abs(dense[k]).sum() + np.abs(dense[:, k]).sum())
        dense[rc[:, 0], rc[:, 1]] = vals
        rhs = rng.uniform(-1.0, 1.0, n)
        vals_nd = np.where(src >= 0, vals[np.maximum(src, 0)], 0.0)
        y = run_schedule(sch, vals_nd, rhs[perm])
        x = np.empty(n)
        x[perm] = y
        assert np.allclose(x, np.linalg.solve(dense, rhs), rtol=1e-10, atol=1e-12)


def run_packed(prog, vals_mf, rhs_mf, n, n_slots):
    """The packed schedule as the kernel reads it: gather the ND slots and the
    right-hand side through the packed maps, then run every level."""
    P = np.asarray(prog, np.int64) & 0xFFFFFFFF
    lo = lambda v: int(v) & 0xFFFF
    hi = lambda v: (int(v) >> 16) & 0xFFFF
    half = lambda base, i: (int(P[base + i // 2]) >> (16 * (i & 1))) & 0xFFFF
    nl, lvt, tpb, ypb, bpb, srcb, posb = (int(P[i]) for i in range(7))
    A = np.array([0.0 if half(srcb, s) == 0xFFFF else vals_mf[half(srcb, s)] for s in range(n_slots)])
    y = np.zeros(n)
    for i in range(n):
        y[half(posb, i)] = rhs_mf[i]
    for lv in range(nl):
        L = [int(P[lvt + 12 * lv + f]) for f in range(12)]
        for q in range(L[1]):
            d = int(P[L[0] + q])
            A[d] = 1.0 / A[d]
        for e in range(L[3]):
            v = P[L[2] + e]
            A[lo(v)] *= A[hi(v)]
        for t in range(L[5] + L[6]):
            h, off = P[L[4] + 2 * t], int(P[L[4] + 2 * t + 1])
            for q in range(hi(h)):
                pr = P[tpb + off + q]
                A[lo(h)] -= A[lo(pr)] * A[hi(pr)]
        for r in range(L[8] + L[9]):
            h, off = P[L[7] + 2 * r], int(P[L[7] + 2 * r + 1])
            for q in range(hi(h)):
                pr = P[ypb + off + q]
                y[lo(h)] -= A[lo(pr)] * y[hi(pr)]
    for lv in range(nl - 1, -1, -1):
        L = [int(P[lvt + 12 * lv + f]) for f in range(12)]
        for q in range(L[11]):
            a, b = P[L[10] + 2 * q], P[L[10] + 2 * q + 1]
            k, d, cnt, off = lo(a), hi(a), lo(b), hi(b)
            sv = y[k]
            for j in range(cnt):
                pr = P[bpb + off + j]
                sv -= A[lo(pr)] * y[hi(pr)]
            y[k] = sv * A[d]
    x = np.empty(n)
    for i in range(n):
        x[i] = y[half(posb, i)]
    return x


@pytest.mark.parametrize("name", list(ALL))
def test_packed_level_program_solves(product, name):
    nl = ALL[name]()
    prob = product.Problem(None, nl)
    sch = prob.lu_schedule()
    if sch is None or len(sch["nd_prog"]) == 0:
        pytest.skip("no packed level program")
    hdr, _, rc = prob.lu_program()
    n, nv = prob.n, prob.info["n_slots"]
    assert int(sch["nd_prog"][7]) == len(sch["nd_prog"])
    src = sch["nd_src"]
    covered = np.zeros(nv, bool)  # zero outside the ND structure (see above)
    covered[src[src >= 0]] = True
    rng = np.random.default_rng(13)
    vals = np.where(covered, rng.uniform(-1.0, 1.0, nv), 0.0)
    dense = np.zeros((n, n))
    dense[rc[:, 0], rc[:, 1]] = vals
    for k in range(n):
        s = hdr[k, 3]
        vals[s] = np.sign(vals[s] or 1.0) * (1.0 + np.abs(dense[k]).sum() + np.abs(dense[:, k]).sum())
    dense[rc[:, 0], rc[:, 1]] = vals
    rhs = rng.uniform(-1.0, 1.0, n)
    x = run_packed(sch["nd_prog"], vals, rhs, n, sch["n_slots"])
    assert np.allclose(x, np.linalg.solve(dense, rhs), rtol=1e-10, atol=1e-12)
