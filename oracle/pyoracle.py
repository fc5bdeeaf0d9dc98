"""ctypes binding of the CPU oracle (TEST INFRASTRUCTURE ONLY).

Loads either the restatement (``port``: oracle/_build/liboracle_port.so) or the
library built from the reference's own sources (``ref``:
oracle/_ref/libkaram_ref.so). Only tests, the smoke check and the benchmark's
CPU-baseline leg import this module; the product never does.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

from karam_b200 import _abi as A

HERE = os.path.dirname(os.path.abspath(__file__))
LIBS = {
    "port": os.path.join(HERE, "_build", "liboracle_port.so"),
    "ref": os.path.join(HERE, "_ref", "libkaram_ref.so"),
}
LS_DENSE = 0
LS_SPARSE = 1


class OracleOpts(C.Structure):
    _fields_ = [("max_nr_iter", C.c_int32), ("gmin_steps", C.c_int32),
                ("reltol", C.c_double), ("vntol", C.c_double),
                ("kcl_shortcut", C.c_double), ("kcl_tol", C.c_double),
                ("polish_max", C.c_int32), ("polish_rel", C.c_double),
                ("polish_abs", C.c_double), ("linear_solver", C.c_int32),
                ("seeded", C.c_int32), ("seed_max_iter", C.c_int32),
                ("max_halvings", C.c_int32), ("lte_rel", C.c_double), ("lte_abs", C.c_double)]


class OracleStats(C.Structure):
    _fields_ = [("converged", C.c_int32), ("iterations", C.c_int32),
                ("polish_iters", C.c_int32), ("damped", C.c_int32),
                ("gmin_step", C.c_int32), ("singular", C.c_int32),
                ("seeded_ok", C.c_int32), ("max_step_iters", C.c_int32),
                ("residual", C.c_double), ("failure_type", C.c_int32),
                ("stagnation", C.c_int32), ("divergence", C.c_int32),
                ("history_len", C.c_int32), ("halvings", C.c_int32),
                ("lte_rejects", C.c_int32)]

    def as_dict(self):
        return {k: getattr(self, k) for k, _ in self._fields_}


def build(kind="port"):
    """Builds the requested oracle library with make (no-op when up to date)."""
    target = {"port": "port", "ref": "ref"}[kind]
    subprocess.run(["make", "-s", "-C", HERE, target], check=True)


def available(kind):
    return os.path.exists(LIBS[kind])


_i32p = C.POINTER(C.c_int32)
_u32p = C.POINTER(C.c_uint32)
_f64p = C.POINTER(C.c_double)


class Oracle:
    def __init__(self, kind="port"):
        self.kind = kind
        self.lib = C.CDLL(LIBS[kind])
        L = self.lib
        L.oracle_default_opts.argtypes = [C.POINTER(OracleOpts)]
        L.oracle_tensorize.argtypes = [C.POINTER(A.KaramNetlist), _i32p, _i32p]
        L.oracle_pattern.argtypes = [C.POINTER(A.KaramNetlist), C.c_int32, _i32p, _i32p, C.c_int32]
        L.oracle_stamp_map.argtypes = [C.POINTER(A.KaramNetlist), _i32p, C.c_int32]
        L.oracle_stamp.argtypes = [C.POINTER(A.KaramNetlist), C.POINTER(A.KaramInstances), C.c_int32,
                                   _f64p, C.c_double, C.c_int32, _f64p, _f64p, C.c_double,
                                   _f64p, _f64p]
        if hasattr(L, "oracle_stamp_abs"):  # restatement only
            L.oracle_stamp_abs.argtypes = [C.POINTER(A.KaramNetlist), C.POINTER(A.KaramInstances),
                                           C.c_int32, _f64p, C.c_double, C.c_int32, _f64p, _f64p,
                                           C.c_double, _f64p, _i32p]
        L.oracle_ordering.argtypes = [C.POINTER(A.KaramNetlist), _u32p, _i32p, _i32p]
        L.oracle_symbolic.argtypes = [C.POINTER(A.KaramNetlist), _i32p, _i32p, _i32p, _i32p,
                                      _i32p, C.c_int32]
        L.oracle_linsolve.argtypes = [C.POINTER(A.KaramNetlist), _f64p, C.c_double, _f64p,
                                      C.c_int32, _f64p]
        L.oracle_solve_dc.argtypes = [C.POINTER(A.KaramNetlist), C.POINTER(A.KaramInstances),
                                      C.c_int32, C.POINTER(OracleOpts), _f64p, _f64p,
                                      C.POINTER(OracleStats)]
        L.oracle_transient.argtypes = [C.POINTER(A.KaramNetlist), C.POINTER(A.KaramInstances),
                                       C.c_int32, C.POINTER(OracleOpts), _f64p, C.c_double,
                                       C.c_int32, C.c_int32, _i32p, C.c_int32, _f64p, _f64p,
                                       C.POINTER(OracleStats)]
        L.oracle_run_batch.argtypes = [C.POINTER(A.KaramNetlist), C.POINTER(A.KaramInstances),
                                       C.c_int32, C.c_int32, C.POINTER(OracleOpts), C.c_double,
                                       C.c_int32, C.c_int32, C.c_int32, _f64p,
                                       C.POINTER(OracleStats)]
        L.oracle_ac.argtypes = [C.POINTER(A.KaramNetlist), C.POINTER(A.KaramInstances), C.c_int32,
                                _f64p, C.c_double, C.c_double, C.c_int32, C.c_int32, C.c_double,
                                C.c_int32, _f64p, _f64p]

    def opts(self, **kw):
        o = OracleOpts()
        self.lib.oracle_default_opts(C.byref(o))
        for k, v in kw.items():
            setattr(o, k, v)
        return o

    @staticmethod
    def _inst(inst):
        return None if inst is None else C.byref(inst.as_struct())

    def tensorize(self, nl):
        s = nl.as_struct()
        mo = np.zeros(max(1, s.n_mos), np.int32)
        do = np.zeros(max(1, s.n_dio), np.int32)
        rc = self.lib.oracle_tensorize(C.byref(s), A.ptr(mo, C.c_int32), A.ptr(do, C.c_int32))
        assert rc == 0
        return mo[: s.n_mos], do[: s.n_dio]

    def pattern(self, nl, transient=True):
        s = nl.as_struct()
        rp = np.zeros(s.n_nodes + 1, np.int32)
        nnz = self.lib.oracle_pattern(C.byref(s), int(transient), A.ptr(rp, C.c_int32), None, 0)
        assert nnz >= 0
        col = np.zeros(nnz, np.int32)
        self.lib.oracle_pattern(C.byref(s), int(transient), A.ptr(rp, C.c_int32),
                                A.ptr(col, C.c_int32), nnz)
        return rp, col

    def stamp_map(self, nl):
        s = nl.as_struct()
        nt = self.lib.oracle_stamp_map(C.byref(s), None, 0)
        out = np.zeros(nt, np.int32)
        self.lib.oracle_stamp_map(C.byref(s), A.ptr(out, C.c_int32), nt)
        return out

    def stamp(self, nl, v, inst=None, idx=0, h=0.0, method=A.TRAN_BE, cap_vprev=None,
              cap_iprev=None, t=0.0):
        s = nl.as_struct()
        rp, col = self.pattern(nl)
        vals = np.zeros(len(col))
        rhs = np.zeros(s.n_nodes)
        v = np.ascontiguousarray(v, dtype=np.float64)
        cv = None if cap_vprev is None else np.ascontiguousarray(cap_vprev, np.float64)
        ci = None if cap_iprev is None else np.ascontiguousarray(cap_iprev, np.float64)
        rc = self.lib.oracle_stamp(C.byref(s), self._inst(inst), idx, A.ptr(v, C.c_double), h,
                                   method, A.ptr(cv, C.c_double), A.ptr(ci, C.c_double), t,
                                   A.ptr(vals, C.c_double), A.ptr(rhs, C.c_double))
        assert rc == 0
        return vals, rhs

    def stamp_abs(self, nl, v, inst=None, idx=0):
        """Per CSR value: sum of |triplet| and the triplet count of a DC stamp at v."""
        s = nl.as_struct()
        rp, col = self.pattern(nl)
        a = np.zeros(len(col))
        cnt = np.zeros(len(col), np.int32)
        v = np.ascontiguousarray(v, dtype=np.float64)
        rc = self.lib.oracle_stamp_abs(C.byref(s), self._inst(inst), idx, A.ptr(v, C.c_double), 0.0,
                                       A.TRAN_BE, None, None, 0.0, A.ptr(a, C.c_double),
                                       A.ptr(cnt, C.c_int32))
        assert rc == 0
        return a, cnt

    def ordering(self, nl):
        s = nl.as_struct()
        n = s.n_nodes
        raw = np.zeros(2 * n + s.n_vsrc + 8, np.uint32)
        rl = C.c_int32(0)
        perm = np.zeros(n, np.int32)
        tw = self.lib.oracle_ordering(C.byref(s), raw.ctypes.data_as(_u32p), C.byref(rl),
                                      A.ptr(perm, C.c_int32))
        return raw[: rl.value], perm, tw

    def symbolic(self, nl):
        s = nl.as_struct()
        n = s.n_nodes
        perm = np.zeros(n, np.int32)
        iperm = np.zeros(n, np.int32)
        rp = np.zeros(n + 1, np.int32)
        fill = C.c_int32(0)
        nnz = self.lib.oracle_symbolic(C.byref(s), A.ptr(perm, C.c_int32), A.ptr(iperm, C.c_int32),
                                       A.ptr(rp, C.c_int32), None, C.byref(fill), 0)
        col = np.zeros(nnz, np.int32)
        self.lib.oracle_symbolic(C.byref(s), None, None, None, A.ptr(col, C.c_int32), None, nnz)
        return dict(perm=perm, iperm=iperm, row_ptr=rp, col=col, fill_in=fill.value)

    def linsolve(self, nl, vals, rhs, gmin=1e-12, solver=LS_DENSE):
        s = nl.as_struct()
        x = np.zeros(s.n_nodes)
        vals = np.ascontiguousarray(vals, np.float64)
        rhs = np.ascontiguousarray(rhs, np.float64)
        rc = self.lib.oracle_linsolve(C.byref(s), A.ptr(vals, C.c_double), gmin,
                                      A.ptr(rhs, C.c_double), solver, A.ptr(x, C.c_double))
        return rc, x

    def solve_dc(self, nl, inst=None, idx=0, v0=None, **opt):
        s = nl.as_struct()
        o = self.opts(**opt)
        v = np.zeros(s.n_nodes)
        st = OracleStats()
        v0a = None if v0 is None else np.ascontiguousarray(v0, np.float64)
        rc = self.lib.oracle_solve_dc(C.byref(s), self._inst(inst), idx, C.byref(o),
                                      A.ptr(v0a, C.c_double), A.ptr(v, C.c_double), C.byref(st))
        assert rc == 0
        return v, st.as_dict()

    def ac(self, nl, v_dc, f_start, f_stop, n_points, input_node, amplitude=1.0, inst=None, idx=0,
           rule=1):
        """Small-signal AC sweep at the DC point v_dc (oracle_ac): complex node
        voltages [n_points][n] and the number of singular points."""
        s = nl.as_struct()
        v = np.ascontiguousarray(v_dc, np.float64)
        re = np.zeros((n_points, s.n_nodes))
        im = np.zeros((n_points, s.n_nodes))
        rc = self.lib.oracle_ac(C.byref(s), self._inst(inst), idx, A.ptr(v, C.c_double), f_start,
                                f_stop, n_points, input_node, amplitude, rule,
                                A.ptr(re, C.c_double), A.ptr(im, C.c_double))
        assert rc >= 0, rc
        return re + 1j * im, rc

    def kcl_residual(self, nl, v, inst=None, idx=0, h=0.0, v_prev=None, t=0.0):
        """Scaled KCL residual of v: the stamp at v (a DC stamp when h == 0,
        else a backward-Euler step of h from v_prev at time t) gives the
        Newton system J x = rhs whose fixed point is a solution, so r = J v -
        rhs is the node current imbalance (branch equations for sources).
        Returns max_i |r_i| / (sum_j |J_ij v_j| + |rhs_i|): about 1e-13 at a
        converged point, and about half the relative error of a perturbed one.
        Needs no factorisation, so it checks problems the oracle's own solve
        is too slow for."""
        rp, col = self.pattern(nl)
        cvp = None
        if v_prev is not None:
            vn = np.concatenate([[0.0], np.asarray(v_prev, np.float64)])
            cvp = np.array([vn[a] - vn[b] for a, b, _ in nl.cap])
        vals, rhs = self.stamp(nl, v, inst, idx, h=h, method=A.TRAN_BE, cap_vprev=cvp, t=t)
        v = np.asarray(v, np.float64)
        rows = np.repeat(np.arange(len(rp) - 1), np.diff(rp))
        r = np.bincount(rows, vals * v[col], minlength=len(v)) - rhs
        scale = np.bincount(rows, np.abs(vals * v[col]), minlength=len(v)) + np.abs(rhs)
        return float(np.max(np.abs(r) / (scale + 1e-300)))

    def transient(self, nl, v_start, dt, n_steps, method=A.TRAN_BE, inst=None, idx=0,
                  wave_nodes=None, **opt):
        s = nl.as_struct()
        o = self.opts(**opt)
        v = np.zeros(s.n_nodes)
        st = OracleStats()
        vs = np.ascontiguousarray(v_start, np.float64)
        wn = None if wave_nodes is None else np.ascontiguousarray(wave_nodes, np.int32)
        nw = 0 if wn is None else len(wn)
        wave = np.zeros((n_steps, max(1, nw)))
        rc = self.lib.oracle_transient(C.byref(s), self._inst(inst), idx, C.byref(o),
                                       A.ptr(vs, C.c_double), dt, n_steps, method,
                                       A.ptr(wn, C.c_int32), nw, A.ptr(wave, C.c_double),
                                       A.ptr(v, C.c_double), C.byref(st))
        assert rc == 0
        return v, st.as_dict(), wave[:, :nw]

    def run_batch(self, nl, inst, i0, i1, dt=0.0, n_steps=0, method=A.TRAN_BE, n_threads=1,
                  **opt):
        s = nl.as_struct()
        o = self.opts(**opt)
        count = i1 - i0
        v = np.zeros((count, s.n_nodes))
        st = (OracleStats * count)()
        rc = self.lib.oracle_run_batch(C.byref(s), self._inst(inst), i0, i1, C.byref(o), dt,
                                       n_steps, method, n_threads, A.ptr(v, C.c_double), st)
        assert rc == 0
        return v, [x.as_dict() for x in st]
