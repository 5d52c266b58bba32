"""ctypes binding of libphc_b200.so (include/polyhomocont_b200.h).

The structures mirror the C header field by field. Loading fails loudly:
if the library was not built, or no CUDA device is usable, the calls raise
instead of falling back to anything else.
"""
import ctypes
import os

import numpy as np

PKG = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(PKG, "libphc_b200.so")

PHC_OK = 0
PHC_ERR_INVALID_INPUT = 1
PHC_ERR_SINGULAR_MATRIX = 2
PHC_ERR_NUMERICAL = 3
PHC_ERR_CUDA = -1
PHC_ERR_UNSUPPORTED = -2
PHC_ERR_NO_DEVICE = -3
PHC_ERR_OOM = -4
PHC_ERR_ADMISSION = -5
PHC_ERR_DEADLINE = -6
PHC_ERR_ABORTED = -7
PHC_ERR_BAD_HANDLE = -8
PHC_ERR_NOT_READY = -9

PHC_PREC_FP64 = 0
PHC_PREC_MIXED = 1
PHC_SCHED_GRID = 0
PHC_SCHED_PERSISTENT = 1

c_i32, c_i64, c_u64, c_dbl, c_vp = (ctypes.c_int32, ctypes.c_int64, ctypes.c_uint64,
                                    ctypes.c_double, ctypes.c_void_p)
P = ctypes.POINTER


class TrackerOptions(ctypes.Structure):
    """type(tracker_options), src/tracker.f90:56-77"""
    _fields_ = [("step_init", c_dbl), ("step_max", c_dbl), ("step_min", c_dbl),
                ("corrector_tol", c_dbl), ("corrector_maxit", c_i32), ("grow_after", c_i32),
                ("contraction", c_dbl), ("max_steps", c_i32), ("pad_", c_i32)]


class EndgameOptions(ctypes.Structure):
    """type(endgame_options), src/endgame.f90:73-101"""
    _fields_ = [("t_start", c_dbl), ("radius_factor", c_dbl), ("radius_min", c_dbl),
                ("loop_radius", c_dbl), ("winding_agreement", c_dbl), ("tol", c_dbl),
                ("residual_tol", c_dbl), ("closure_factor", c_dbl), ("nsamples", c_i32),
                ("max_winding", c_i32)]


class SolveOptions(ctypes.Structure):
    """type(solve_options), src/solve.f90:57-84"""
    _fields_ = [("tracker", TrackerOptions), ("endgame", EndgameOptions),
                ("use_endgame", c_i32), ("seed", c_i32), ("refine_maxit", c_i32),
                ("pad_", c_i32), ("infinity_tol", c_dbl), ("singular_cond", c_dbl),
                ("real_tol", c_dbl), ("dedup_tol", c_dbl), ("singular_dedup_tol", c_dbl)]


class GpuOptions(ctypes.Structure):
    _fields_ = [("precision", c_i32), ("schedule", c_i32), ("device", c_i32),
                ("warps_per_block", c_i32), ("blocks_per_sm", c_i32), ("chunk", c_i32),
                ("fp64_sticky", c_i32), ("unit_budget_log2", c_i32)]


class SolveCounts(ctypes.Structure):
    _fields_ = [(k, c_i32) for k in ("n", "npaths", "nsolutions", "nreal", "nsingular",
                                      "ninfinite", "nfailed", "nduplicates")]


class SolveResultC(ctypes.Structure):
    _fields_ = [("counts", SolveCounts), ("paths", c_vp), ("z", P(c_dbl)), ("x", P(c_dbl)),
                ("solutions", P(c_dbl)), ("real_solutions", P(c_dbl)),
                ("singular_solutions", P(c_dbl)), ("multiplicities", P(c_i32))]


class SystemC(ctypes.Structure):
    _fields_ = [("n", c_i32), ("nterms", c_i32), ("first", P(c_i32)), ("deg", P(c_i32)),
                ("hexps", P(c_i32)), ("coefs", P(c_dbl))]


class HomotopyC(ctypes.Structure):
    _fields_ = [("gamma", c_dbl * 2), ("b", P(c_dbl)), ("patch", P(c_dbl))]


class ServerConfig(ctypes.Structure):
    _fields_ = [("device", c_i32), ("nslots", c_i32), ("max_batch_systems", c_i32),
                ("max_batch_paths", c_i32), ("mem_budget_bytes", c_i64), ("gpu", GpuOptions)]


PHC_TUNE_MAX = 32


class TuneReport(ctypes.Structure):
    _fields_ = [("ncand", c_i32), ("best", c_i32), ("schedule", c_i32 * PHC_TUNE_MAX),
                ("warps_per_block", c_i32 * PHC_TUNE_MAX), ("chunk", c_i32 * PHC_TUNE_MAX),
                ("ms", c_dbl * PHC_TUNE_MAX), ("sample_paths", c_i64)]


# phc_path_out
PATH_DTYPE = np.dtype([
    ("status", "<i4"), ("winding_number", "<i4"), ("endgame_status", "<i4"),
    ("at_infinity", "<i4"), ("singular", "<i4"), ("is_real", "<i4"),
    ("naccepted", "<i4"), ("nrejected", "<i4"), ("solution_index", "<i4"),
    ("singular_index", "<i4"), ("n_tangent", "<i4"), ("n_newton", "<i4"),
    ("n_refine", "<i4"), ("n_eval", "<i4"), ("n_cond", "<i4"),
    ("n_fp64_retry", "<i4"), ("t", "<f8"), ("endgame_error", "<f8"),
    ("cond", "<f8"), ("residual", "<f8")])
assert PATH_DTYPE.itemsize == 96

# sys%evaluate(x, f, jac) as a C callback (phc_evaluator)
EVALUATOR = ctypes.CFUNCTYPE(c_i32, c_vp, c_i32, P(c_dbl), P(c_dbl), P(c_dbl))

# every entry point the header declares: (name, restype, argtypes)
SIGNATURES = [
    ("phc_version", ctypes.c_char_p, []),
    ("phc_last_error", ctypes.c_char_p, []),
    ("phc_default_solve_options", None, [P(SolveOptions)]),
    ("phc_default_gpu_options", None, [P(GpuOptions)]),
    ("phc_sparse_create", c_vp, []),
    ("phc_sparse_destroy", None, [c_vp]),
    ("phc_sparse_init", c_i32, [c_vp, c_i32]),
    ("phc_sparse_add_equation", c_i32, [c_vp, c_i32, P(c_dbl), c_i32, c_i32, P(c_i32)]),
    ("phc_sparse_nvars", c_i32, [c_vp]),
    ("phc_sparse_nequations", c_i32, [c_vp]),
    ("phc_sparse_nterms", c_i32, [c_vp, c_i32]),
    ("phc_sparse_total_terms", c_i32, [c_vp]),
    ("phc_sparse_degrees", None, [c_vp, P(c_i32)]),
    ("phc_sparse_table", c_i32, [c_vp, P(SystemC)]),
    ("phc_sparse_evaluate", c_i32, [c_vp, P(c_dbl), P(c_dbl), P(c_dbl)]),
    ("phc_sparse_evaluate_homogeneous", c_i32, [c_vp, P(c_dbl), P(c_dbl), P(c_dbl)]),
    ("phc_sparse_sample", c_i32, [c_vp, c_i32, P(c_i32), EVALUATOR, c_vp, c_i32, P(c_dbl)]),
    ("phc_homotopy_init", c_i32, [P(SystemC), c_i32, P(c_dbl), P(c_dbl), P(c_dbl),
                                  P(c_i64)]),
    ("phc_bezout", c_i64, [P(SystemC)]),
    ("phc_finish_solve", c_i32, [c_i32, c_i64, P(SolveOptions), c_vp, P(c_dbl),
                                 P(SolveResultC)]),
    ("phc_solve_sparse", c_i32, [P(SystemC), P(SolveOptions), P(GpuOptions),
                                 P(SolveResultC)]),
    ("phc_solve_paths", c_i32, [P(SystemC), P(HomotopyC), P(SolveOptions), P(GpuOptions),
                                c_i64, c_i64, c_vp, P(c_dbl), P(c_dbl)]),
    ("phc_solve_paths_noalloc", c_i32, [P(SystemC), P(HomotopyC), P(SolveOptions),
                                        P(GpuOptions), c_i64, c_i64, c_vp, c_vp, c_vp, c_vp]),
    ("phc_plan_create", c_i32, [P(SystemC), P(HomotopyC), P(SolveOptions), P(GpuOptions),
                                P(c_vp)]),
    ("phc_plan_launch", c_i32, [c_vp, c_i64, c_i64, c_vp, c_vp, c_vp]),
    ("phc_plan_launch_count", c_i32, [c_vp]),
    ("phc_plan_destroy", c_i32, [c_vp]),
    ("phc_plan_config", c_i32, [c_vp, P(c_i32), P(c_i32), P(c_i32), P(c_i32), P(c_i32)]),
    ("phc_graph_create", c_i32, [c_vp, c_i64, c_i64, c_vp, c_vp, P(c_vp)]),
    ("phc_graph_launch", c_i32, [c_vp, c_vp]),
    ("phc_graph_destroy", c_i32, [c_vp]),
    ("phc_autotune", c_i32, [P(SystemC), P(SolveOptions), P(GpuOptions), c_i64,
                             P(TuneReport)]),
    ("phc_request_size", c_i64, [P(SystemC), c_i32]),
    ("phc_request_encode", c_i32, [P(SystemC), P(SolveOptions), c_vp, c_i64, P(c_i64)]),
    ("phc_request_decode", c_i32, [c_vp, c_i64, c_vp, P(SolveOptions)]),
    ("phc_server_create", c_i32, [P(ServerConfig), P(c_vp)]),
    ("phc_server_submit_request", c_i32, [c_vp, c_vp, c_i64, P(c_u64)]),
    ("phc_server_submit", c_i32, [c_vp, P(SystemC), P(SolveOptions), P(c_u64)]),
    ("phc_server_poll", c_i32, [c_vp, c_u64, P(c_i32)]),
    ("phc_server_wait", c_i32, [c_vp, c_u64, c_i64]),
    ("phc_server_result", c_i32, [c_vp, c_u64, P(SolveResultC), P(c_dbl)]),
    ("phc_server_npaths", c_i64, [c_vp, c_u64]),
    ("phc_server_stats", c_i32, [c_vp, P(c_i64), P(c_i64), P(c_i64), P(c_i64)]),
    ("phc_server_destroy", c_i32, [c_vp]),
    ("phc_measure_fma_peaks", c_i32, [c_i32, P(c_dbl), P(c_dbl)]),
]

_LIB = None


def lib():
    """Loads the in-tree library (raises if it was not built)."""
    global _LIB
    if _LIB is not None:
        return _LIB
    if not os.path.exists(LIB_PATH):
        raise RuntimeError(
            f"{LIB_PATH} is missing: build it with `python -m polyhomocont_b200.build` "
            "(the tracker has no CPU fallback)")
    L = ctypes.CDLL(LIB_PATH)
    for name, res, args in SIGNATURES:
        f = getattr(L, name)
        f.restype = res
        f.argtypes = args
    _LIB = L
    return L


def last_error():
    return lib().phc_last_error().decode(errors="replace")


def dptr(a):
    return a.ctypes.data_as(P(c_dbl))


def iptr(a):
    return a.ctypes.data_as(P(c_i32))
