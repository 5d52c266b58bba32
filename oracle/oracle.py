"""ctypes binding of the CPU restatement (TEST INFRASTRUCTURE ONLY).

Only tests/, __graft_entry__.smoke() and bench.py's cpu_baseline leg import
this module. It mirrors the reference's Fortran API (sparse_system,
solve_options, solve, solve_result, res%paths) closely enough that the
known-answer tests of the reference (test/*.f90) read the same way in
Python.
"""
import ctypes
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))

# status codes (src/config.f90:16-23) and path/end game codes
STATUS_OK = 0
ERR_INVALID_INPUT = 1
ERR_SINGULAR_MATRIX = 2
PATH_SUCCESS = 0
PATH_FAILED_MIN_STEP = 1
PATH_FAILED_MAX_STEPS = 2
PATH_ENDGAME_FAILED = 3
ENDGAME_CONVERGED = 0
ENDGAME_NOT_CONVERGED = 1
ENDGAME_FAILED = 2


class TrackerOptions(ctypes.Structure):
    _fields_ = [("step_init", ctypes.c_double), ("step_max", ctypes.c_double),
                ("step_min", ctypes.c_double), ("corrector_tol", ctypes.c_double),
                ("corrector_maxit", ctypes.c_int32), ("grow_after", ctypes.c_int32),
                ("contraction", ctypes.c_double), ("max_steps", ctypes.c_int32),
                ("pad_", ctypes.c_int32)]


class EndgameOptions(ctypes.Structure):
    _fields_ = [("t_start", ctypes.c_double), ("radius_factor", ctypes.c_double),
                ("radius_min", ctypes.c_double), ("loop_radius", ctypes.c_double),
                ("winding_agreement", ctypes.c_double), ("tol", ctypes.c_double),
                ("residual_tol", ctypes.c_double), ("closure_factor", ctypes.c_double),
                ("nsamples", ctypes.c_int32), ("max_winding", ctypes.c_int32)]


class SolveOptions(ctypes.Structure):
    _fields_ = [("tracker", TrackerOptions), ("endgame", EndgameOptions),
                ("use_endgame", ctypes.c_int32), ("seed", ctypes.c_int32),
                ("refine_maxit", ctypes.c_int32), ("pad_", ctypes.c_int32),
                ("infinity_tol", ctypes.c_double), ("singular_cond", ctypes.c_double),
                ("real_tol", ctypes.c_double), ("dedup_tol", ctypes.c_double),
                ("singular_dedup_tol", ctypes.c_double)]


class PathInfo(ctypes.Structure):
    _fields_ = [("status", ctypes.c_int32), ("naccepted", ctypes.c_int32),
                ("nrejected", ctypes.c_int32), ("pad_", ctypes.c_int32),
                ("s", ctypes.c_double), ("t_re", ctypes.c_double),
                ("t_im", ctypes.c_double), ("step", ctypes.c_double)]

    @property
    def t(self):
        return complex(self.t_re, self.t_im)


class EndgameResult(ctypes.Structure):
    _fields_ = [("status", ctypes.c_int32), ("winding_number", ctypes.c_int32),
                ("naccepted", ctypes.c_int32), ("nrejected", ctypes.c_int32),
                ("error", ctypes.c_double), ("residual", ctypes.c_double),
                ("radius", ctypes.c_double)]


class SolveCounts(ctypes.Structure):
    _fields_ = [(k, ctypes.c_int32) for k in
                ("n", "npaths", "nsolutions", "nreal", "nsingular", "ninfinite",
                 "nfailed", "nduplicates")]


# per-path record; same layout as phc_path_out of the product interface
PATH_DTYPE = np.dtype([
    ("status", "<i4"), ("winding_number", "<i4"), ("endgame_status", "<i4"),
    ("at_infinity", "<i4"), ("singular", "<i4"), ("is_real", "<i4"),
    ("naccepted", "<i4"), ("nrejected", "<i4"), ("solution_index", "<i4"),
    ("singular_index", "<i4"), ("n_tangent", "<i4"), ("n_newton", "<i4"),
    ("n_refine", "<i4"), ("n_eval", "<i4"), ("n_cond", "<i4"),
    ("n_fp64_retry", "<i4"), ("t", "<f8"), ("endgame_error", "<f8"),
    ("cond", "<f8"), ("residual", "<f8")])
assert PATH_DTYPE.itemsize == 96

_lib = {}


# evaluate(x, f, jac) of a user system as a C callback (orc_user_evaluator)
USER_EVALUATOR = ctypes.CFUNCTYPE(ctypes.c_int32, ctypes.c_void_p, ctypes.c_int32,
                                  ctypes.POINTER(ctypes.c_double), ctypes.POINTER(ctypes.c_double),
                                  ctypes.POINTER(ctypes.c_double))


def build(fast=False):
    """Compile the restatement with make (both libraries)."""
    subprocess.run(["make", "-s", "-C", HERE], check=True)


def lib(fast=False):
    key = "fast" if fast else "check"
    if key in _lib:
        return _lib[key]
    name = "liborcphc_fast.so" if fast else "liborcphc.so"
    path = os.path.join(HERE, name)
    if not os.path.exists(path):
        build()
    L = ctypes.CDLL(path)
    vp, i32, i64, dbl = ctypes.c_void_p, ctypes.c_int32, ctypes.c_int64, ctypes.c_double
    P = ctypes.POINTER
    dp = P(ctypes.c_double)
    ip = P(ctypes.c_int32)
    sig = {
        "orc_default_solve_options": (None, [P(SolveOptions)]),
        "orc_rng_new": (vp, []), "orc_rng_free": (None, [vp]),
        "orc_rng_seed": (None, [vp, i32]), "orc_rng_uniform": (dbl, [vp]),
        "orc_rng_unit_complex": (None, [vp, dp]),
        "orc_rng_normal_complex": (None, [vp, dp]),
        "orc_lu_factor": (i32, [i32, dp, ip]),
        "orc_lu_solve": (None, [i32, dp, ip, dp]),
        "orc_solve_linear": (i32, [i32, dp, dp, dp]),
        "orc_cond1": (dbl, [i32, dp]), "orc_norm_inf": (dbl, [i32, dp]),
        "orc_sparse_new": (vp, []), "orc_sparse_free": (None, [vp]),
        "orc_sparse_init": (None, [vp, i32]),
        "orc_sparse_add_equation": (i32, [vp, i32, dp, i32, i32, ip]),
        "orc_sparse_nvars": (i32, [vp]), "orc_sparse_nequations": (i32, [vp]),
        "orc_sparse_nterms": (i32, [vp, i32]),
        "orc_sparse_total_terms": (i32, [vp]), "orc_sparse_maxexp": (i32, [vp]),
        "orc_sparse_degrees": (None, [vp, ip]),
        "orc_sparse_table": (None, [vp, ip, ip, dp]),
        "orc_sparse_evaluate": (None, [vp, dp, dp, dp]),
        "orc_sparse_evaluate_homogeneous": (None, [vp, dp, dp, dp]),
        "orc_sparse_set_user": (None, [vp, i32, ip, USER_EVALUATOR, vp]),
        "orc_hom_new": (vp, []), "orc_hom_free": (None, [vp]),
        "orc_hom_init": (i32, [vp, vp, vp]), "orc_hom_nstart": (i32, [vp]),
        "orc_hom_constants": (None, [vp, dp, dp, dp]),
        "orc_hom_start_solution": (None, [vp, i32, dp]),
        "orc_hom_evaluate": (None, [vp, dp, dp, dp, dp, dp]),
        "orc_track_path": (None, [vp, dp, dbl, dbl, P(TrackerOptions), P(PathInfo)]),
        "orc_track_line": (None, [vp, dp, dp, dp, P(TrackerOptions), P(PathInfo)]),
        "orc_track_arc": (None, [vp, dp, dbl, dbl, dbl, P(TrackerOptions), P(PathInfo)]),
        "orc_cauchy_endgame": (None, [vp, dp, P(EndgameOptions), P(TrackerOptions),
                                      P(EndgameResult), dp]),
        "orc_bezout": (i64, [vp]),
        "orc_solve_paths": (i32, [vp, P(SolveOptions), i64, i64, i32, vp, dp, dp]),
        "orc_solve": (i32, [vp, P(SolveOptions), i32, vp, dp, dp, P(SolveCounts),
                            dp, dp, dp, ip]),
    }
    for name, (res, args) in sig.items():
        f = getattr(L, name)
        f.restype = res
        f.argtypes = args
    _lib[key] = L
    return L


def _dp(a):
    return a.ctypes.data_as(ctypes.POINTER(ctypes.c_double))


def _ip(a):
    return a.ctypes.data_as(ctypes.POINTER(ctypes.c_int32))


def cbuf(n):
    return np.zeros(n, dtype=np.complex128)


def default_options():
    o = SolveOptions()
    lib().orc_default_solve_options(ctypes.byref(o))
    return o


def default_tracker_options():
    return default_options().tracker


def default_endgame_options():
    return default_options().endgame


class Rng:
    """type(rng), src/random.f90:29-38"""

    def __init__(self, seed=None):
        self._L = lib()
        self.h = self._L.orc_rng_new()
        if seed is not None:
            self.seed(seed)

    def __del__(self):
        try:
            self._L.orc_rng_free(self.h)
        except Exception:
            pass

    def seed(self, s):
        self._L.orc_rng_seed(self.h, int(s))

    def uniform(self):
        return self._L.orc_rng_uniform(self.h)

    def unit_complex(self):
        z = cbuf(1)
        self._L.orc_rng_unit_complex(self.h, _dp(z))
        return complex(z[0])

    def normal_complex(self):
        z = cbuf(1)
        self._L.orc_rng_normal_complex(self.h, _dp(z))
        return complex(z[0])


class SparseSystem:
    """type(sparse_system), src/sparse.f90:31-61"""

    def __init__(self, n=None, fast=False):
        self._L = lib(fast)
        self.h = self._L.orc_sparse_new()
        if n is not None:
            self.init(n)

    def __del__(self):
        try:
            self._L.orc_sparse_free(self.h)
        except Exception:
            pass

    def init(self, n):
        self._L.orc_sparse_init(self.h, int(n))

    def add_equation(self, coefs, exps):
        """coefs: sequence of numbers; exps: array of shape (rows, cols),
        the Fortran exponent matrix (one column per term). Returns status."""
        c = np.ascontiguousarray(np.asarray(coefs, dtype=np.complex128).ravel())
        e = np.asarray(exps, dtype=np.int32)
        if e.ndim == 1:
            e = e.reshape(-1, 1)
        ef = np.asfortranarray(e)
        flat = np.ascontiguousarray(ef.ravel(order="F"))
        return self._L.orc_sparse_add_equation(self.h, c.size, _dp(c), e.shape[0],
                                               e.shape[1], _ip(flat))

    def nvars(self):
        return self._L.orc_sparse_nvars(self.h)

    def nequations(self):
        return self._L.orc_sparse_nequations(self.h)

    def nterms(self, i):
        return self._L.orc_sparse_nterms(self.h, int(i))

    def total_terms(self):
        return self._L.orc_sparse_total_terms(self.h)

    def degrees(self):
        d = np.zeros(self.nequations(), dtype=np.int32)
        self._L.orc_sparse_degrees(self.h, _ip(d))
        return d

    def maxexp(self):
        return self._L.orc_sparse_maxexp(self.h)

    def table(self):
        """(first[neq+1], hexps[T, n+1], coefs[T])"""
        neq, n, T = self.nequations(), self.nvars(), self.total_terms()
        first = np.zeros(neq + 1, dtype=np.int32)
        hexps = np.zeros(T * (n + 1), dtype=np.int32)
        coefs = cbuf(T)
        self._L.orc_sparse_table(self.h, _ip(first), _ip(hexps), _dp(coefs))
        return first, hexps.reshape(T, n + 1), coefs

    def evaluate(self, x):
        x = np.ascontiguousarray(x, dtype=np.complex128)
        n = self.nvars()
        f = cbuf(n)
        jac = np.zeros((n, n), dtype=np.complex128, order="F")
        self._L.orc_sparse_evaluate(self.h, _dp(x), _dp(f), _dp(jac))
        return f, jac

    def evaluate_homogeneous(self, z):
        z = np.ascontiguousarray(z, dtype=np.complex128)
        n = self.nvars()
        f = cbuf(n)
        jac = np.zeros((n, n + 1), dtype=np.complex128, order="F")
        self._L.orc_sparse_evaluate_homogeneous(self.h, _dp(z), _dp(f), _dp(jac))
        return f, jac


class UserSystem(SparseSystem):
    """A user system, class(poly_system) of src/system.f90:27-67: usys has
    nvars(), degrees() and evaluate(x) -> (f, jac[i, j] = dF_i/dx_j). The
    restatement evaluates F^h through the reference's default
    homogenization (poly_system_evaluate_homogeneous, src/system.f90:71-119)
    and solves it like any system; use nthreads=1 (the callback runs
    Python)."""

    def __init__(self, usys, fast=False):
        super().__init__(fast=fast)
        n = int(usys.nvars())
        self._deg = np.ascontiguousarray(np.asarray(usys.degrees(), dtype=np.int32).ravel())

        def cb(_ctx, m, xp, fp, jp):
            x = np.ctypeslib.as_array(xp, shape=(2 * m,)).view(np.complex128).copy()
            f, jac = usys.evaluate(x)
            np.ctypeslib.as_array(fp, shape=(2 * m,))[:] = (
                np.asarray(f, dtype=np.complex128).reshape(m).view(np.float64))
            np.ctypeslib.as_array(jp, shape=(2 * m * m,))[:] = np.asfortranarray(
                np.asarray(jac, dtype=np.complex128).reshape(m, m)).ravel(order="F").view(
                    np.float64)
            return 0

        self._cb = USER_EVALUATOR(cb)
        self._L.orc_sparse_set_user(self.h, n, _ip(self._deg), self._cb, None)


class Homotopy:
    """type(total_degree_homotopy), src/homotopy.f90:45-68"""

    def __init__(self):
        self._L = lib()
        self.h = self._L.orc_hom_new()
        self.sys = None

    def __del__(self):
        try:
            self._L.orc_hom_free(self.h)
        except Exception:
            pass

    def init(self, sys, gen):
        self.sys = sys
        return self._L.orc_hom_init(self.h, sys.h, gen.h)

    @property
    def n(self):
        return self.sys.nvars()

    @property
    def nstart(self):
        return self._L.orc_hom_nstart(self.h)

    def nunknowns(self):
        return self.n + 1

    def constants(self):
        n = self.n
        g, b, a = cbuf(1), cbuf(n), cbuf(n + 1)
        self._L.orc_hom_constants(self.h, _dp(g), _dp(b), _dp(a))
        return complex(g[0]), b, a

    def start_solution(self, k):
        z = cbuf(self.n + 1)
        self._L.orc_hom_start_solution(self.h, int(k), _dp(z))
        return z

    def evaluate(self, z, t):
        N = self.n + 1
        z = np.ascontiguousarray(z, dtype=np.complex128)
        tt = np.array([complex(t)], dtype=np.complex128)
        h, ht = cbuf(N), cbuf(N)
        hz = np.zeros((N, N), dtype=np.complex128, order="F")
        self._L.orc_hom_evaluate(self.h, _dp(z), _dp(tt), _dp(h), _dp(hz), _dp(ht))
        return h, hz, ht


def track_path(hom, z, t_start, t_end, opts=None):
    z = np.array(z, dtype=np.complex128)
    info = PathInfo()
    o = opts if opts is not None else default_tracker_options()
    lib().orc_track_path(hom.h, _dp(z), t_start, t_end, ctypes.byref(o),
                         ctypes.byref(info))
    return z, info


def track_arc(hom, z, radius, theta0, dtheta, opts=None):
    z = np.array(z, dtype=np.complex128)
    info = PathInfo()
    o = opts if opts is not None else default_tracker_options()
    lib().orc_track_arc(hom.h, _dp(z), radius, theta0, dtheta, ctypes.byref(o),
                        ctypes.byref(info))
    return z, info


def cauchy_endgame(hom, z, eopts=None, topts=None):
    z = np.array(z, dtype=np.complex128)
    zres = cbuf(z.size)
    r = EndgameResult()
    eo = eopts if eopts is not None else default_endgame_options()
    to = topts if topts is not None else default_tracker_options()
    lib().orc_cauchy_endgame(hom.h, _dp(z), ctypes.byref(eo), ctypes.byref(to),
                             ctypes.byref(r), _dp(zres))
    return z, zres, r


def lu_factor(a):
    a = np.array(a, dtype=np.complex128, order="F")
    n = a.shape[0]
    ipiv = np.zeros(n, dtype=np.int32)
    st = lib().orc_lu_factor(n, _dp(a), _ip(ipiv))
    return a, ipiv, st


def lu_solve(lu, ipiv, b):
    b = np.array(b, dtype=np.complex128)
    lu = np.asfortranarray(lu, dtype=np.complex128)
    lib().orc_lu_solve(lu.shape[0], _dp(lu), _ip(np.asarray(ipiv, dtype=np.int32)),
                       _dp(b))
    return b


def solve_linear(a, b):
    a = np.asfortranarray(a, dtype=np.complex128)
    b = np.ascontiguousarray(b, dtype=np.complex128)
    x = cbuf(a.shape[0])
    st = lib().orc_solve_linear(a.shape[0], _dp(a), _dp(b), _dp(x))
    return x, st


def cond1(a):
    a = np.asfortranarray(a, dtype=np.complex128)
    return lib().orc_cond1(a.shape[0], _dp(a))


def norm_inf(z):
    z = np.ascontiguousarray(z, dtype=np.complex128)
    return lib().orc_norm_inf(z.size, _dp(z))


class SolveResult:
    """type(solve_result), src/solve.f90:121-150 (arrays 0-based; index
    fields of the paths keep the reference's 1-based meaning)."""

    def __init__(self):
        self.n = 0
        self.npaths = 0
        self.paths = np.zeros(0, dtype=PATH_DTYPE)
        self.z = np.zeros((0, 1), dtype=np.complex128)
        self.x = np.zeros((0, 1), dtype=np.complex128)
        self.nsolutions = 0
        self.solutions = np.zeros((0, 0), dtype=np.complex128)
        self.nreal = 0
        self.real_solutions = np.zeros((0, 0))
        self.nsingular = 0
        self.singular_solutions = np.zeros((0, 0), dtype=np.complex128)
        self.multiplicities = np.zeros(0, dtype=np.int32)
        self.ninfinite = 0
        self.nfailed = 0
        self.nduplicates = 0


def solve(sys, options=None, nthreads=1):
    """solve(sys, res, status, options), src/solve.f90:154-215.
    Returns (res, status). Solutions are stored as rows (nsolutions, n)."""
    L = sys._L
    o = options if options is not None else default_options()
    n = sys.nvars()
    res = SolveResult()
    if sys.nequations() != n or n < 1:
        npaths = 0
    else:
        npaths = int(L.orc_bezout(sys.h))
    if npaths > 2**31 - 1:
        npaths = 0
    m = max(npaths, 1)
    paths = np.zeros(m, dtype=PATH_DTYPE)
    z = np.zeros((m, n + 1), dtype=np.complex128)
    x = np.zeros((m, max(n, 1)), dtype=np.complex128)
    counts = SolveCounts()
    sols = np.zeros((m, max(n, 1)), dtype=np.complex128)
    ssols = np.zeros((m, max(n, 1)), dtype=np.complex128)
    realsols = np.zeros((m, max(n, 1)))
    mult = np.zeros(m, dtype=np.int32)
    st = L.orc_solve(sys.h, ctypes.byref(o), int(nthreads),
                     paths.ctypes.data_as(ctypes.c_void_p), _dp(z), _dp(x),
                     ctypes.byref(counts), _dp(sols), _dp(realsols), _dp(ssols),
                     _ip(mult))
    if st != STATUS_OK:
        return res, st
    res.n = counts.n
    res.npaths = counts.npaths
    res.paths = paths[:npaths]
    res.z = z[:npaths]
    res.x = x[:npaths, :n]
    res.nsolutions = counts.nsolutions
    res.solutions = sols[:counts.nsolutions, :n]
    res.nreal = counts.nreal
    res.real_solutions = realsols[:counts.nreal, :n]
    res.nsingular = counts.nsingular
    res.singular_solutions = ssols[:counts.nsingular, :n]
    res.multiplicities = mult[:counts.nsingular]
    res.ninfinite = counts.ninfinite
    res.nfailed = counts.nfailed
    res.nduplicates = counts.nduplicates
    return res, st


def solve_paths(sys, options=None, k0=1, count=None, nthreads=1):
    """Per-path numerics only (start_solution + endpoint + classify) for
    1-based paths k0 .. k0+count-1. Returns (paths, z, x, status)."""
    L = sys._L
    o = options if options is not None else default_options()
    n = sys.nvars()
    if count is None:
        count = int(L.orc_bezout(sys.h)) - k0 + 1
    paths = np.zeros(max(count, 1), dtype=PATH_DTYPE)
    z = np.zeros((max(count, 1), n + 1), dtype=np.complex128)
    x = np.zeros((max(count, 1), n), dtype=np.complex128)
    st = L.orc_solve_paths(sys.h, ctypes.byref(o), int(k0), int(count), int(nthreads),
                           paths.ctypes.data_as(ctypes.c_void_p), _dp(z), _dp(x))
    return paths[:count], z[:count], x[:count], st
