"""ctypes mirror of include/karam.h (structs and constants)."""
import ctypes as C

KARAM_OK = 0
KARAM_E_INVALID = -1
KARAM_E_CUDA = -2
KARAM_E_NOMEM = -3
KARAM_E_UNSUPPORTED = -4
KARAM_E_STATE = -5

ST_CONVERGED = 0
ST_NOCONV = 1
ST_SINGULAR = 2
ST_NAN = 3
ST_TIMEOUT = 4
# ConvergenceFailureType (include/karam.h KARAM_FAIL_*)
FAIL_NONE, FAIL_SINGULAR_MATRIX, FAIL_DIVERGENCE, FAIL_LIMIT_CYCLE = 0, 1, 2, 3
FAIL_SLOW_CONVERGENCE, FAIL_FLOATING_NODE_INDUCED, FAIL_EXPONENTIAL_OVERFLOW = 4, 5, 6
HISTORY_MAX = 16

PREC_FP64 = 0
PREC_MIXED = 1
TRAN_BE = 0
TRAN_TRAP = 1
SEED_NONE = 0
SEED_CALLER = 1
SEED_EMA = 2
SEED_HISTORY = 8
SEED_MLP = 3
SRC_DC = 0
SRC_PULSE = 1
MODEL_NMOS = 0
MODEL_PMOS = 1
MODEL_DIODE = 2

_i32p = C.POINTER(C.c_int32)
_f64p = C.POINTER(C.c_double)
_f32p = C.POINTER(C.c_float)


class KaramNetlist(C.Structure):
    _fields_ = [
        ("n_nodes", C.c_int32), ("temp_k", C.c_double),
        ("n_vsrc", C.c_int32), ("vs_pos", _i32p), ("vs_neg", _i32p), ("vs_dc", _f64p),
        ("vs_kind", _i32p), ("vs_pulse", _f64p),
        ("n_isrc", C.c_int32), ("is_pos", _i32p), ("is_neg", _i32p), ("is_amp", _f64p),
        ("n_res", C.c_int32), ("r_n1", _i32p), ("r_n2", _i32p), ("r_ohm", _f64p),
        ("n_cap", C.c_int32), ("c_n1", _i32p), ("c_n2", _i32p), ("c_farad", _f64p),
        ("n_dio", C.c_int32), ("d_anode", _i32p), ("d_cathode", _i32p), ("d_is", _f64p),
        ("d_n", _f64p), ("d_vt", _f64p), ("d_model", _i32p),
        ("n_mos", C.c_int32), ("m_d", _i32p), ("m_g", _i32p), ("m_s", _i32p), ("m_b", _i32p),
        ("m_w", _f64p), ("m_l", _f64p), ("m_model", _i32p),
        ("n_models", C.c_int32), ("model_name", C.POINTER(C.c_char_p)), ("model_type", _i32p),
        ("model_kp", _f64p), ("model_vto", _f64p), ("model_lambda", _f64p),
    ]


class KaramInstances(C.Structure):
    _fields_ = [("n_instances", C.c_int32), ("mos_kp", _f32p), ("mos_vto", _f32p),
                ("vs_dc", _f64p)]


class KaramSolverOpts(C.Structure):
    _fields_ = [
        ("precision", C.c_int32), ("max_nr_iter", C.c_int32), ("gmin_steps", C.c_int32),
        ("reltol", C.c_double), ("vntol", C.c_double), ("kcl_shortcut", C.c_double),
        ("kcl_tol", C.c_double), ("polish_max", C.c_int32), ("polish_rel", C.c_double),
        ("polish_abs", C.c_double), ("lu_growth_limit", C.c_double), ("seeded", C.c_int32),
        ("seed_max_iter", C.c_int32), ("schedule", C.c_int32), ("max_rounds", C.c_int32),
        ("max_halvings", C.c_int32), ("kernel_timing", C.c_int32),
        ("lte_reltol", C.c_double), ("lte_abstol", C.c_double),
    ]


class KaramProblemInfo(C.Structure):
    _fields_ = [(name, C.c_int32) for name in (
        "n", "nnz", "nnz_filled", "fill_in", "treewidth", "n_triplets", "n_instances",
        "n_mos", "n_dio", "n_res", "n_cap", "n_vsrc", "n_isrc", "lu_ops", "n_slots", "es_blocks",
        "es_device_evals")]


class KaramInstanceStats(C.Structure):
    _fields_ = [("status", C.c_int32), ("iterations", C.c_int32),
                ("polish_iters", C.c_int32), ("damped", C.c_int32),
                ("gmin_step", C.c_int32), ("seeded_ok", C.c_int32),
                ("rescued", C.c_int32), ("halvings", C.c_int32),
                ("max_step_iters", C.c_int32), ("residual", C.c_double),
                ("failure_type", C.c_int32), ("stagnation", C.c_int32),
                ("divergence", C.c_int32), ("history_len", C.c_int32),
                ("lte_rejects", C.c_int32), ("reserved_", C.c_int32)]


class KaramTiming(C.Structure):
    _fields_ = [("job_ms", C.c_double), ("eval_ms", C.c_double), ("lu_ms", C.c_double),
                ("rescue_ms", C.c_double), ("rounds", C.c_int32), ("eval_launches", C.c_int32),
                ("lu_launches", C.c_int32), ("rescue_launches", C.c_int32),
                ("other_launches", C.c_int32),
                ("lanes", C.c_int32), ("level_schedule", C.c_int32),
                ("evals_dc", C.c_int64), ("evals_tran", C.c_int64),
                ("solves", C.c_int64), ("rescues", C.c_int64),
                ("rescues_dense", C.c_int64), ("tail_rounds", C.c_int32),
                ("persistent_rounds", C.c_int32), ("seed_ms", C.c_double),
                ("resident_instances", C.c_int32), ("reserved_", C.c_int32)]


def ptr(arr, ctype):
    """Pointer to a contiguous numpy array (or NULL for None)."""
    if arr is None:
        return C.cast(None, C.POINTER(ctype))
    return arr.ctypes.data_as(C.POINTER(ctype))
