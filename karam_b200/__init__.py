"""karam_b200 -- B200-native Newton-Raphson inner loop of the Karam circuit engine.

Python binding of the in-tree C ABI (include/karam.h, libkaram_b200.so). The
classes mirror how the reference drives its solver: a ``Problem`` is the
analog of a compiled block (CircuitSim + NetlistCompiler::compile) for one
topology, batched over Monte-Carlo instances; ``solve_dc`` / ``step_transient``
are CircuitSim::solveDC / stepTransient (physics/circuitsim.h:1110-1115) for
every instance at once; ``run_mc`` replaces SessionImpl::runMonteCarlo's
sequential loop (engine_impl.cpp:259-281).

There is no CPU fallback: loading fails loudly when the library is missing.
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

from . import _abi as A
from .circuits import Instances, Netlist  # noqa: F401  (re-exported)

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libkaram_b200.so")

_lib = None


class KaramError(RuntimeError):
    def __init__(self, code, msg):
        super().__init__(f"karam error {code}: {msg}")
        self.code = code


def lib():
    """The loaded libkaram_b200.so (raises when it has not been built)."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise ImportError(f"{LIB_PATH} is missing: run `python -m karam_b200.build` "
                          "(the product has no CPU fallback)")
    L = C.CDLL(LIB_PATH)
    P = C.POINTER
    vp = C.c_void_p
    sig = {
        "karam_ctx_create": (C.c_int, [C.c_int, P(vp)]),
        "karam_ctx_destroy": (None, [vp]),
        "karam_last_error": (C.c_char_p, [vp]),
        "karam_default_opts": (None, [P(A.KaramSolverOpts)]),
        "karam_problem_create": (C.c_int, [vp, P(A.KaramNetlist), C.c_int32, P(vp)]),
        "karam_problem_destroy": (None, [vp]),
        "karam_problem_info_get": (C.c_int, [vp, P(A.KaramProblemInfo)]),
        "karam_set_instances": (C.c_int, [vp, P(A.KaramInstances)]),
        "karam_solve_dc": (C.c_int, [vp, P(A.KaramSolverOpts), P(C.c_double), P(C.c_double),
                                     P(A.KaramInstanceStats)]),
        "karam_step_transient": (C.c_int, [vp, P(A.KaramSolverOpts), C.c_double, C.c_int32,
                                           C.c_int32, P(C.c_int32), C.c_int32, P(C.c_double),
                                           P(C.c_double), P(A.KaramInstanceStats)]),
        "karam_run_mc": (C.c_int, [vp, P(A.KaramInstances), P(A.KaramSolverOpts), C.c_double,
                                   C.c_int32, C.c_int32, P(C.c_double),
                                   P(A.KaramInstanceStats)]),
        "karam_run_mc_device": (C.c_int, [vp, P(A.KaramSolverOpts), C.c_double, C.c_int32,
                                          C.c_int32]),
        "karam_run_mc_multi": (C.c_int, [P(vp), C.c_int32, P(A.KaramSolverOpts), C.c_double,
                                         C.c_int32, C.c_int32]),
        "karam_ac_sweep": (C.c_int, [vp, C.c_double, C.c_double, C.c_int32, C.c_int32, C.c_double,
                                     P(C.c_double), P(C.c_double), P(C.c_double), P(C.c_int32)]),
        "karam_tune_schedule": (C.c_int, [vp, P(A.KaramSolverOpts), C.c_int32, P(C.c_int32),
                                          P(C.c_double)]),
        "karam_spice_parse": (C.c_int, [C.c_char_p, P(vp), C.c_char_p, C.c_int32]),
        "karam_spice_netlist": (P(A.KaramNetlist), [vp]),
        "karam_spice_node": (C.c_int32, [vp, C.c_char_p]),
        "karam_spice_analysis": (C.c_int, [vp, P(C.c_int32), P(C.c_int32), P(C.c_double),
                                           P(C.c_double), P(C.c_double)]),
        "karam_spice_free": (None, [vp]),
        "karam_netlist_hash": (C.c_int, [P(A.KaramNetlist), P(C.c_uint64)]),
        "karam_symbolic_cache_info": (C.c_int, [P(C.c_int32), P(C.c_int64), P(C.c_int64)]),
        "karam_symbolic_cache_clear": (None, []),
        "karam_read_results": (C.c_int, [vp, P(C.c_double), P(A.KaramInstanceStats)]),
        "karam_get_history": (C.c_int, [vp, C.c_int32, P(C.c_double), P(C.c_double),
                                        P(C.c_int32)]),
        "karam_sync": (C.c_int, [vp]),
        "karam_get_pattern": (C.c_int, [vp, P(C.c_int32), P(C.c_int32)]),
        "karam_get_stamp_map": (C.c_int, [vp, P(C.c_int32)]),
        "karam_get_ordering": (C.c_int, [vp, P(C.c_uint32), P(C.c_int32), P(C.c_int32)]),
        "karam_get_filled_pattern": (C.c_int, [vp, P(C.c_int32), P(C.c_int32)]),
        "karam_get_device_order": (C.c_int, [vp, P(C.c_int32), P(C.c_int32)]),
        "karam_get_lu_program": (C.c_int, [vp, P(C.c_int32), P(C.c_int32), P(C.c_int32),
                                           P(C.c_int32)]),
        "karam_get_lu_records": (C.c_int, [vp, P(C.c_int32), P(C.c_int32)]),
        "karam_get_lu_schedule": (C.c_int, [vp, P(C.c_int32), C.c_int64, P(C.c_int64)]),
        "karam_seeder_create": (C.c_int, [vp, C.c_int32, C.c_int32, C.c_uint64, P(vp)]),
        "karam_seeder_destroy": (None, [vp]),
        "karam_seeder_add_dc": (C.c_int, [vp, vp, P(C.c_int32)]),
        "karam_seeder_train": (C.c_int, [vp, C.c_int32, C.c_int32, C.c_float, C.c_uint64,
                                         P(C.c_float)]),
        "karam_problem_set_seeder": (C.c_int, [vp, vp]),
        "karam_seeder_predict": (C.c_int, [vp, vp, P(C.c_double)]),
        "karam_seeder_gemm": (C.c_int, [C.c_int32, C.c_int32, C.c_int32, P(C.c_float), C.c_int32,
                                        C.c_int32, P(C.c_float), C.c_int32, C.c_int32,
                                        P(C.c_float)]),
        "karam_eval_stamp": (C.c_int, [vp, C.c_int32, P(C.c_double), P(C.c_double),
                                       P(C.c_double)]),
        "karam_last_timing": (C.c_int, [vp, P(A.KaramTiming)]),
        "karam_eval_stamp_noalloc": (C.c_int, [vp, C.c_int32, C.c_void_p, C.c_void_p,
                                               C.c_void_p]),
    }
    for name, (res, args) in sig.items():
        fn = getattr(L, name)
        fn.restype = res
        fn.argtypes = args
    _lib = L
    return L


def options(**kw) -> A.KaramSolverOpts:
    """Solver options: the reference constants, overridden by keyword."""
    o = A.KaramSolverOpts()
    lib().karam_default_opts(C.byref(o))
    for k, v in kw.items():
        if not hasattr(o, k):
            raise AttributeError(f"unknown solver option {k}")
        setattr(o, k, v)
    return o


class SpiceNetlist:
    """A SPICE netlist read by the library's front-end (karam_spice_parse);
    usable wherever a circuits.Netlist is (Problem, the oracle)."""

    def __init__(self, text: str):
        h = C.c_void_p()
        err = C.create_string_buffer(512)
        rc = lib().karam_spice_parse(text.encode(), C.byref(h), err, len(err))
        if rc != A.KARAM_OK:
            raise KaramError(rc, err.value.decode())
        self.h = h
        self._s = lib().karam_spice_netlist(h).contents
        self.n_nodes = self._s.n_nodes

    def as_struct(self) -> A.KaramNetlist:
        return self._s

    def node(self, name: str) -> int:
        """Node index of a name (0 = ground, -1 = unknown)."""
        return lib().karam_spice_node(self.h, name.encode())

    def analysis(self):
        """(.OP given, .TRAN given, tran step, tran stop, tran start)."""
        op, tr = C.c_int32(0), C.c_int32(0)
        st, sp, s0 = C.c_double(0), C.c_double(0), C.c_double(0)
        lib().karam_spice_analysis(self.h, C.byref(op), C.byref(tr), C.byref(st), C.byref(sp),
                                   C.byref(s0))
        return bool(op.value), bool(tr.value), st.value, sp.value, s0.value

    @property
    def n_mos(self):
        return self._s.n_mos

    def close(self):
        if getattr(self, "h", None):
            lib().karam_spice_free(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def parse_spice(text: str) -> SpiceNetlist:
    return SpiceNetlist(text)


def netlist_hash(nl) -> int:
    """64-bit fingerprint of a netlist's content (karam_netlist_hash)."""
    h = C.c_uint64(0)
    rc = lib().karam_netlist_hash(C.byref(nl.as_struct()), C.byref(h))
    if rc != A.KARAM_OK:
        raise KaramError(rc, "netlist hash")
    return h.value


def symbolic_cache_info():
    """(entries, hits, misses) of the symbolic-analysis cache."""
    e, h, m = C.c_int32(0), C.c_int64(0), C.c_int64(0)
    lib().karam_symbolic_cache_info(C.byref(e), C.byref(h), C.byref(m))
    return e.value, h.value, m.value


def symbolic_cache_clear():
    lib().karam_symbolic_cache_clear()


class Context:
    """One CUDA device + stream (karam_ctx)."""

    def __init__(self, device=0):
        h = C.c_void_p()
        rc = lib().karam_ctx_create(device, C.byref(h))
        if rc != A.KARAM_OK:
            raise KaramError(rc, lib().karam_last_error(None).decode())
        self.h = h

    def close(self):
        if self.h:
            lib().karam_ctx_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class Problem:
    """One topology + its batch of instances (karam_problem).

    With ``ctx=None`` only the host symbolic analysis is built (no device
    memory); the symbolic queries work, solves raise.
    """

    def __init__(self, ctx: Context | None, nl: Netlist, max_instances=1):
        self.ctx = ctx
        self.nl = nl
        self._nls = nl.as_struct()
        h = C.c_void_p()
        rc = lib().karam_problem_create(ctx.h if ctx else None, C.byref(self._nls),
                                        max_instances, C.byref(h))
        if rc != A.KARAM_OK:
            raise KaramError(rc, lib().karam_last_error(ctx.h if ctx else None).decode())
        self.h = h
        self.info = self._info()
        self.n = self.info["n"]
        self.ni = 1

    def _check(self, rc):
        if rc != A.KARAM_OK:
            raise KaramError(rc, lib().karam_last_error(self.ctx.h if self.ctx else None).decode())

    def close(self):
        if getattr(self, "h", None):
            lib().karam_problem_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def _info(self):
        inf = A.KaramProblemInfo()
        self._check(lib().karam_problem_info_get(self.h, C.byref(inf)))
        return {k: getattr(inf, k) for k, _ in A.KaramProblemInfo._fields_}

    # -- symbolic queries ---------------------------------------------------
    def pattern(self):
        rp = np.zeros(self.n + 1, np.int32)
        col = np.zeros(self.info["nnz"], np.int32)
        self._check(lib().karam_get_pattern(self.h, A.ptr(rp, C.c_int32), A.ptr(col, C.c_int32)))
        return rp, col

    def stamp_map(self):
        out = np.zeros(self.info["n_triplets"], np.int32)
        self._check(lib().karam_get_stamp_map(self.h, A.ptr(out, C.c_int32)))
        return out

    def ordering(self):
        raw = np.zeros(2 * self.n + self.info["n_vsrc"] + 8, np.uint32)
        rl = C.c_int32(0)
        perm = np.zeros(self.n, np.int32)
        self._check(lib().karam_get_ordering(self.h, raw.ctypes.data_as(C.POINTER(C.c_uint32)),
                                             C.byref(rl), A.ptr(perm, C.c_int32)))
        return raw[: rl.value], perm, self.info["treewidth"]

    def filled_pattern(self):
        rp = np.zeros(self.n + 1, np.int32)
        col = np.zeros(self.info["nnz_filled"], np.int32)
        self._check(lib().karam_get_filled_pattern(self.h, A.ptr(rp, C.c_int32),
                                                   A.ptr(col, C.c_int32)))
        return rp, col

    def device_order(self):
        mo = np.zeros(max(1, self.info["n_mos"]), np.int32)
        do = np.zeros(max(1, self.info["n_dio"]), np.int32)
        self._check(lib().karam_get_device_order(self.h, A.ptr(mo, C.c_int32),
                                                 A.ptr(do, C.c_int32)))
        return mo[: self.info["n_mos"]], do[: self.info["n_dio"]]

    def lu_program(self):
        """(hdr[n, 4], data, slot_rc[n_slots, 2]) of the static-pivot LU program."""
        n, nv = self.n, self.info["n_slots"]
        ln = C.c_int32(0)
        self._check(lib().karam_get_lu_program(self.h, None, None, C.byref(ln), None))
        hdr = np.zeros(4 * n, np.int32)
        data = np.zeros(max(1, ln.value), np.int32)
        rc = np.zeros(2 * nv, np.int32)
        self._check(lib().karam_get_lu_program(self.h, A.ptr(hdr, C.c_int32),
                                               A.ptr(data, C.c_int32), C.byref(ln),
                                               A.ptr(rc, C.c_int32)))
        return hdr.reshape(n, 4), data[: ln.value], rc.reshape(nv, 2)

    def lu_records(self):
        """(rec[n, 8], rec2[n, 2]) pivot records of the device's packed schedule,
        or None when some pivot has nL > 1 or nU > 2."""
        n = self.n
        rec = np.zeros(8 * n, np.int32)
        rec2 = np.zeros(2 * n, np.int32)
        rc = lib().karam_get_lu_records(self.h, A.ptr(rec, C.c_int32), A.ptr(rec2, C.c_int32))
        if rc == A.KARAM_E_UNSUPPORTED:
            return None
        self._check(rc)
        return rec.reshape(n, 8), rec2.reshape(n, 2)

    _SCHED = ("nd_perm nd_src nd_diag lv_piv lv_piv_ptr lv_l_ptr l_slot l_piv lv_ts_ptr "
              "lv_tl_ptr t_slot t_off pr_l pr_u lv_ys_ptr lv_yl_ptr y_row y_off yp_l yp_k "
              "bs_off bs_u bs_c nd_prog").split()

    def lu_schedule(self):
        """The level schedule of the factor/solve kernel's LU as a dict of arrays
        (plus n, n_slots, levels, long), or None when the problem has none."""
        ln = C.c_int64(0)
        rc = lib().karam_get_lu_schedule(self.h, None, 0, C.byref(ln))
        if rc == A.KARAM_E_UNSUPPORTED:
            return None
        self._check(rc)
        buf = np.zeros(ln.value, np.int32)
        self._check(lib().karam_get_lu_schedule(self.h, A.ptr(buf, C.c_int32), ln.value,
                                                C.byref(ln)))
        out = dict(n=int(buf[0]), n_slots=int(buf[1]), levels=int(buf[2]), long=int(buf[3]))
        i = 4
        for name in self._SCHED:
            m = int(buf[i])
            out[name] = buf[i + 1:i + 1 + m].copy()
            i += 1 + m
        return out

    # -- batches and solves -------------------------------------------------
    def set_instances(self, inst: Instances | None):
        self._inst = inst.as_struct() if inst is not None else None
        self._check(lib().karam_set_instances(self.h, C.byref(self._inst) if inst else None))
        self.ni = inst.n if inst is not None else 1

    @staticmethod
    def _stats(st):
        return [{k: getattr(s, k) for k, _ in A.KaramInstanceStats._fields_} for s in st]

    def solve_dc(self, opts=None, seed=None):
        opts = opts or options()
        v = np.zeros((self.ni, self.n))
        st = (A.KaramInstanceStats * self.ni)()
        sd = None if seed is None else np.ascontiguousarray(seed, np.float64)
        self._check(lib().karam_solve_dc(self.h, C.byref(opts), A.ptr(sd, C.c_double),
                                         A.ptr(v, C.c_double), st))
        return v, self._stats(st)

    def step_transient(self, dt, n_steps, method=A.TRAN_BE, opts=None, wave_nodes=None):
        opts = opts or options()
        v = np.zeros((self.ni, self.n))
        st = (A.KaramInstanceStats * self.ni)()
        wn = None if wave_nodes is None else np.ascontiguousarray(wave_nodes, np.int32)
        nw = 0 if wn is None else len(wn)
        wave = np.zeros((self.ni, n_steps, max(1, nw)))
        self._check(lib().karam_step_transient(self.h, C.byref(opts), dt, n_steps, method,
                                               A.ptr(wn, C.c_int32), nw,
                                               A.ptr(wave, C.c_double) if nw else None,
                                               A.ptr(v, C.c_double), st))
        return v, self._stats(st), wave[:, :, :nw]

    def run_mc(self, inst: Instances, dt=0.0, n_steps=0, method=A.TRAN_BE, opts=None):
        opts = opts or options()
        self._inst = inst.as_struct()
        self.ni = inst.n
        v = np.zeros((self.ni, self.n))
        st = (A.KaramInstanceStats * self.ni)()
        self._check(lib().karam_run_mc(self.h, C.byref(self._inst), C.byref(opts), dt, n_steps,
                                       method, A.ptr(v, C.c_double), st))
        return v, self._stats(st)

    def run_mc_device(self, dt=0.0, n_steps=0, method=A.TRAN_BE, opts=None):
        opts = opts or options()
        self._check(lib().karam_run_mc_device(self.h, C.byref(opts), dt, n_steps, method))

    def ac_sweep(self, f_start, f_stop, n_points, input_node, amplitude=1.0):
        """Small-signal AC sweep at every instance's DC point (karam_ac_sweep):
        (frequencies[n_points], complex voltages [ni][n_points][n],
        status [ni][n_points])."""
        f = np.zeros(n_points)
        re = np.zeros((self.ni, n_points, self.n))
        im = np.zeros((self.ni, n_points, self.n))
        st = np.zeros((self.ni, n_points), np.int32)
        self._check(lib().karam_ac_sweep(self.h, f_start, f_stop, n_points, input_node, amplitude,
                                         A.ptr(f, C.c_double), A.ptr(re, C.c_double),
                                         A.ptr(im, C.c_double), A.ptr(st, C.c_int32)))
        return f, re + 1j * im, st

    def tune_schedule(self, opts=None, rounds=16):
        """Measured factor/solve schedule (karam_tune_schedule): returns the
        opts.schedule value kept for this problem and its trial time (ms)."""
        opts = opts or options()
        sch = C.c_int32(0)
        ms = C.c_double(0.0)
        self._check(lib().karam_tune_schedule(self.h, C.byref(opts), rounds, C.byref(sch),
                                              C.byref(ms)))
        return sch.value, ms.value

    def read_results(self, want_stats=True):
        v = np.zeros((self.ni, self.n))
        st = (A.KaramInstanceStats * self.ni)() if want_stats else None
        self._check(lib().karam_read_results(self.h, A.ptr(v, C.c_double), st))
        return v, (self._stats(st) if want_stats else None)

    def history(self, instance):
        """(residual[m], max_dv[m]) of the instance's last m <= HISTORY_MAX DC NR
        iterations, oldest first (karam_get_history)."""
        f = np.zeros(A.HISTORY_MAX)
        dv = np.zeros(A.HISTORY_MAX)
        m = C.c_int32(0)
        self._check(lib().karam_get_history(self.h, instance, A.ptr(f, C.c_double),
                                            A.ptr(dv, C.c_double), C.byref(m)))
        return f[: m.value], dv[: m.value]

    def sync(self):
        self._check(lib().karam_sync(self.h))

    def eval_stamp(self, v, precision=A.PREC_FP64):
        v = np.ascontiguousarray(v, np.float64).reshape(self.ni, self.n)
        jac = np.zeros((self.ni, self.info["nnz"]))
        f = np.zeros((self.ni, self.n))
        self._check(lib().karam_eval_stamp(self.h, precision, A.ptr(v, C.c_double),
                                           A.ptr(jac, C.c_double), A.ptr(f, C.c_double)))
        return jac, f

    def set_seeder(self, seeder):
        """Attach (or with None detach) the learned seeder used by
        options(seeded=SEED_MLP)."""
        self._check(lib().karam_problem_set_seeder(self.h, seeder.h if seeder else None))
        self._seeder = seeder

    def timing(self):
        """Device accounting of the last solve call (karam_timing as a dict)."""
        t = A.KaramTiming()
        self._check(lib().karam_last_timing(self.h, C.byref(t)))
        return {k: getattr(t, k) for k, _ in A.KaramTiming._fields_}


def run_mc_multi(problems, dt=0.0, n_steps=0, method=A.TRAN_BE, opts=None):
    """karam_run_mc_multi: the device-resident job of every problem (one
    context, instances already set) in one persistent launch; results per
    problem through Problem.read_results()."""
    opts = opts or options()
    if not problems:
        raise ValueError("no problems")
    hs = (C.c_void_p * len(problems))(*[p.h for p in problems])
    rc = lib().karam_run_mc_multi(hs, len(problems), C.byref(opts), dt, n_steps, method)
    problems[0]._check(rc)


class Seeder:
    """Learned NR seeder (karam_seeder): a BF16 MLP trained on a problem's
    plain-NR DC solutions; used by solves with options(seeded=SEED_MLP) once
    attached with Problem.set_seeder."""

    def __init__(self, prob: Problem, width=512, hidden_layers=3, init_seed=1):
        self.ctx = prob.ctx
        h = C.c_void_p()
        rc = lib().karam_seeder_create(prob.h, width, hidden_layers, init_seed, C.byref(h))
        if rc != A.KARAM_OK:
            raise KaramError(rc, lib().karam_last_error(self.ctx.h).decode())
        self.h = h

    def _check(self, rc):
        if rc != A.KARAM_OK:
            raise KaramError(rc, lib().karam_last_error(self.ctx.h).decode())

    def add_dc(self, prob: Problem) -> int:
        """Add the converged DC solutions of prob's last (DC) solve; returns the count."""
        n = C.c_int32(0)
        self._check(lib().karam_seeder_add_dc(self.h, prob.h, C.byref(n)))
        return n.value

    def train(self, epochs=40, batch=256, lr=1e-3, shuffle_seed=0) -> float:
        loss = C.c_float(0.0)
        self._check(lib().karam_seeder_train(self.h, epochs, batch, lr, shuffle_seed,
                                             C.byref(loss)))
        return loss.value

    def predict(self, prob: Problem) -> np.ndarray:
        out = np.zeros((prob.ni, prob.n))
        self._check(lib().karam_seeder_predict(self.h, prob.h, A.ptr(out, C.c_double)))
        return out

    def close(self):
        if getattr(self, "h", None):
            lib().karam_seeder_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def bf16_gemm(a: np.ndarray, b: np.ndarray, trans_a=False, trans_b=False) -> np.ndarray:
    """The seeder's tensor-core GEMM on host arrays: op(a) @ op(b) with BF16
    operands and FP32 accumulation (op = transpose when the flag is set)."""
    a = np.ascontiguousarray(a, np.float32)
    b = np.ascontiguousarray(b, np.float32)
    M, K = (a.shape[1], a.shape[0]) if trans_a else a.shape
    K2, N = (b.shape[1], b.shape[0]) if trans_b else b.shape
    assert K == K2
    c = np.zeros((M, N), np.float32)
    rc = lib().karam_seeder_gemm(M, N, K, A.ptr(a, C.c_float), a.shape[1], int(trans_a),
                                 A.ptr(b, C.c_float), b.shape[1], int(trans_b), A.ptr(c, C.c_float))
    if rc != A.KARAM_OK:
        raise KaramError(rc, lib().karam_last_error(None).decode())
    return c
