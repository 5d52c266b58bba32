"""polyhomocont_b200 -- B200 path tracker for polyhomocont's solve().

Python mirror of the reference's Fortran API over the C ABI of
libphc_b200.so (include/polyhomocont_b200.h):

    type(sparse_system)   -> SparseSystem   (init, add_equation, nvars, ...)
    class(poly_system)    -> PolySystem     (nvars, degrees, evaluate; sampled
                                             into a SparseSystem by sample_system)
    type(solve_options)   -> SolveOptions   (tracker, endgame, seed, tolerances)
    solve(sys, res, status, options) -> res, status = solve(sys, options)
    type(solve_result)    -> SolveResult    (paths, solutions, counts, ...)

The per-path numerics run on the GPU (one warp per path, sm_100a); the
order-dependent bookkeeping runs on the host in path order, as in the
reference. There is no CPU fallback: without the built library or a CUDA
device the calls raise.
"""
import ctypes

import numpy as np

from . import _abi
from ._abi import (PATH_DTYPE, PHC_ERR_INVALID_INPUT, PHC_OK, PHC_PREC_FP64,  # noqa: F401
                   PHC_PREC_MIXED, PHC_SCHED_GRID, PHC_SCHED_PERSISTENT, EndgameOptions,
                   GpuOptions, SolveOptions, TrackerOptions)

STATUS_OK = 0
ERR_INVALID_INPUT = 1
ERR_SINGULAR_MATRIX = 2
ERR_NUMERICAL = 3
PATH_SUCCESS = 0
PATH_FAILED_MIN_STEP = 1
PATH_FAILED_MAX_STEPS = 2
PATH_ENDGAME_FAILED = 3
ENDGAME_CONVERGED = 0
ENDGAME_NOT_CONVERGED = 1


class PhcError(RuntimeError):
    def __init__(self, code, what):
        super().__init__(f"{what} failed with status {code}: {_abi.last_error()}")
        self.code = code


def _check_device_status(st, what):
    """Negative codes are device/runtime errors: raise. Codes 0..3 are the
    reference's solve statuses and are returned to the caller."""
    if st < 0:
        raise PhcError(st, what)
    return st


def default_options():
    o = SolveOptions()
    _abi.lib().phc_default_solve_options(ctypes.byref(o))
    return o


def default_gpu_options(precision=PHC_PREC_MIXED, schedule=PHC_SCHED_PERSISTENT, device=0,
                        warps_per_block=0):
    g = GpuOptions()
    _abi.lib().phc_default_gpu_options(ctypes.byref(g))
    g.precision = precision
    g.schedule = schedule
    g.device = device
    g.warps_per_block = warps_per_block
    return g


class SparseSystem:
    """type(sparse_system), src/sparse.f90:31-61"""

    def __init__(self, n=None):
        self._L = _abi.lib()
        self.h = self._L.phc_sparse_create()
        if not self.h:
            raise MemoryError("phc_sparse_create")
        if n is not None:
            self.init(n)

    def __del__(self):
        try:
            self._L.phc_sparse_destroy(self.h)
        except Exception:
            pass

    def init(self, n):
        """sys%init(n), src/sparse.f90:65-81"""
        return self._L.phc_sparse_init(self.h, int(n))

    def add_equation(self, coefs, exps):
        """sys%add_equation(coefs, exps, status), src/sparse.f90:83-141.
        exps: (rows, cols) exponent matrix, one column per term."""
        c = np.ascontiguousarray(np.asarray(coefs, dtype=np.complex128).ravel())
        e = np.asarray(exps, dtype=np.int32)
        if e.ndim == 1:
            e = e.reshape(-1, 1)
        flat = np.ascontiguousarray(e.ravel(order="F"))
        cd = c.view(np.float64)
        return self._L.phc_sparse_add_equation(self.h, c.size, _abi.dptr(cd), e.shape[0],
                                               e.shape[1], _abi.iptr(flat))

    def nvars(self):
        return self._L.phc_sparse_nvars(self.h)

    def nequations(self):
        return self._L.phc_sparse_nequations(self.h)

    def nterms(self, i):
        return self._L.phc_sparse_nterms(self.h, int(i))

    def total_terms(self):
        return self._L.phc_sparse_total_terms(self.h)

    def degrees(self):
        d = np.zeros(max(self.nequations(), 1), dtype=np.int32)
        self._L.phc_sparse_degrees(self.h, _abi.iptr(d))
        return d[:self.nequations()]

    def evaluate(self, x):
        """sys%evaluate(x, f, jac), src/sparse.f90:197-207: (F(x), dF/dx) with
        jac[i, j] = dF_i/dx_j (host arithmetic)."""
        n = self.nvars()
        xv = np.ascontiguousarray(np.asarray(x, dtype=np.complex128).reshape(n))
        f = np.zeros(n, dtype=np.complex128)
        jac = np.zeros((n, n), dtype=np.complex128, order="F")
        st = self._L.phc_sparse_evaluate(self.h, _abi.dptr(xv.view(np.float64)),
                                         _abi.dptr(f.view(np.float64)),
                                         _abi.dptr(jac.reshape(-1, order="F").view(np.float64)))
        if st != PHC_OK:
            raise PhcError(st, "phc_sparse_evaluate")
        return f, jac

    def evaluate_homogeneous(self, z):
        """sys%evaluate_homogeneous(z, f, jac), src/sparse.f90:209-221:
        (F^h(z), dF^h/dz) at z = (z_1, ..., z_n, w), exact also at w = 0."""
        n = self.nvars()
        zv = np.ascontiguousarray(np.asarray(z, dtype=np.complex128).reshape(n + 1))
        f = np.zeros(n, dtype=np.complex128)
        jac = np.zeros((n, n + 1), dtype=np.complex128, order="F")
        st = self._L.phc_sparse_evaluate_homogeneous(
            self.h, _abi.dptr(zv.view(np.float64)), _abi.dptr(f.view(np.float64)),
            _abi.dptr(jac.reshape(-1, order="F").view(np.float64)))
        if st != PHC_OK:
            raise PhcError(st, "phc_sparse_evaluate_homogeneous")
        return f, jac

    def table(self):
        """phc_system view of the packed table and its status (err_invalid_input
        if the system does not have n equations)."""
        t = _abi.SystemC()
        st = self._L.phc_sparse_table(self.h, ctypes.byref(t))
        return t, st

    def bezout(self):
        t, st = self.table()
        return int(self._L.phc_bezout(ctypes.byref(t))) if st == 0 else 0


class PolySystem:
    """class(poly_system), src/system.f90:27-67: a user system given by
    nvars(), degrees() (exact total degrees d_i >= 1) and evaluate(x) ->
    (f, jac) with f = F(x) and jac[i, j] = dF_i/dx_j. solve() and
    solve_paths() turn it into a sparse table (sample_system) and track
    that on the GPU."""

    def nvars(self):
        raise NotImplementedError

    def degrees(self):
        raise NotImplementedError

    def evaluate(self, x):
        raise NotImplementedError


def sample_system(sys, seed=1):
    """phc_sparse_sample: the SparseSystem of the polynomial system that the
    PolySystem sys evaluates. Returns (SparseSystem, status, max_error);
    status is err_invalid_input when sys.evaluate is not a polynomial of
    the stated degrees or its Jacobian disagrees with F, and max_error is
    the worst relative error of the table against sys at the check points.
    An exception raised by sys.evaluate is raised again here."""
    n = int(sys.nvars())
    deg = np.ascontiguousarray(np.asarray(sys.degrees(), dtype=np.int32).ravel())
    if deg.size != n:
        return SparseSystem(), ERR_INVALID_INPUT, 0.0
    raised = []

    def cb(_ctx, m, xp, fp, jp):
        try:
            x = np.ctypeslib.as_array(xp, shape=(2 * m,)).view(np.complex128)
            f, jac = sys.evaluate(x.copy())
            f = np.asarray(f, dtype=np.complex128).reshape(m)
            jac = np.asarray(jac, dtype=np.complex128).reshape(m, m)
            np.ctypeslib.as_array(fp, shape=(2 * m,))[:] = f.view(np.float64)
            np.ctypeslib.as_array(jp, shape=(2 * m * m,))[:] = (
                np.asfortranarray(jac).ravel(order="F").view(np.float64))
            return 0
        except Exception as e:  # noqa: BLE001 - re-raised after the call
            raised.append(e)
            return 1

    s = SparseSystem()
    err = ctypes.c_double(0.0)
    fn = _abi.EVALUATOR(cb)
    st = s._L.phc_sparse_sample(s.h, n, _abi.iptr(deg), fn, None, int(seed), ctypes.byref(err))
    if raised:
        raise raised[0]
    return s, st, float(err.value)


def _as_sparse(sys):
    if isinstance(sys, SparseSystem):
        return sys, PHC_OK
    s, st, _ = sample_system(sys)
    return s, st


def encode_request(sys, options=None):
    """The system (and options, if given) in the compact request format of
    the serving path (phc_request_encode) as bytes. sys is a SparseSystem
    or a PolySystem (sampled first)."""
    L = _abi.lib()
    sys, st = _as_sparse(sys)
    if st != PHC_OK:
        raise PhcError(st, "sample_system")
    t, st = sys.table()
    if st != PHC_OK:
        raise PhcError(st, "table")
    optr = ctypes.byref(options) if options is not None else None
    size = int(L.phc_request_size(ctypes.byref(t), 1 if options is not None else 0))
    buf = ctypes.create_string_buffer(max(size, 1))
    n = ctypes.c_int64()
    st = L.phc_request_encode(ctypes.byref(t), optr, buf, size, ctypes.byref(n))
    if st != PHC_OK:
        raise PhcError(st, "phc_request_encode")
    return buf.raw[:n.value]


def decode_request(data):
    """(SparseSystem, solve_options, status) from a compact request
    (phc_request_decode); status != 0 for a malformed request."""
    s = SparseSystem()
    o = SolveOptions()
    buf = ctypes.create_string_buffer(bytes(data), max(len(data), 1))
    st = s._L.phc_request_decode(buf, len(data), s.h, ctypes.byref(o))
    return s, o, st


class SolveResult:
    """type(solve_result), src/solve.f90:121-150. Arrays are 0-based with
    solutions as rows; the path index fields keep the reference's 1-based
    meaning (0 = none)."""

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


def _result_buffers(n, npaths, alloc=None):
    """Host result arrays of one solve; alloc(shape, dtype) may provide
    page-locked memory."""
    alloc = alloc or (lambda shape, dtype: np.zeros(shape, dtype=dtype))
    m = max(npaths, 1)
    nn = max(n, 1)
    bufs = dict(
        paths=alloc((m,), PATH_DTYPE),
        z=alloc((m, n + 1), np.complex128),
        x=alloc((m, nn), np.complex128),
        sols=alloc((m, nn), np.complex128),
        realsols=alloc((m, nn), np.float64),
        ssols=alloc((m, nn), np.complex128),
        mult=alloc((m,), np.int32),
    )
    rc = _abi.SolveResultC()
    rc.paths = bufs["paths"].ctypes.data_as(ctypes.c_void_p)
    rc.z = _abi.dptr(bufs["z"].view(np.float64))
    rc.x = _abi.dptr(bufs["x"].view(np.float64))
    rc.solutions = _abi.dptr(bufs["sols"].view(np.float64))
    rc.real_solutions = _abi.dptr(bufs["realsols"])
    rc.singular_solutions = _abi.dptr(bufs["ssols"].view(np.float64))
    rc.multiplicities = _abi.iptr(bufs["mult"])
    return bufs, rc


def _fill_result(n, npaths, bufs, rc):
    c = rc.counts
    res = SolveResult()
    res.n = c.n
    res.npaths = c.npaths
    res.paths = bufs["paths"][:npaths]
    res.z = bufs["z"][:npaths]
    res.x = bufs["x"][:npaths, :n]
    res.nsolutions = c.nsolutions
    res.solutions = bufs["sols"][:c.nsolutions, :n]
    res.nreal = c.nreal
    res.real_solutions = bufs["realsols"][:c.nreal, :n]
    res.nsingular = c.nsingular
    res.singular_solutions = bufs["ssols"][:c.nsingular, :n]
    res.multiplicities = bufs["mult"][:c.nsingular]
    res.ninfinite = c.ninfinite
    res.nfailed = c.nfailed
    res.nduplicates = c.nduplicates
    return res


def solve(sys, options=None, gpu=None, buffers=None):
    """solve(sys, res, status, options), src/solve.f90:154-215, on the GPU.
    sys is a SparseSystem or a PolySystem (sampled first). Returns
    (res, status); status is err_invalid_input for systems the
    reference rejects. Device errors raise PhcError. buffers: optional
    (bufs, rc) from _result_buffers, reused across calls."""
    L = _abi.lib()
    o = options if options is not None else default_options()
    g = gpu if gpu is not None else default_gpu_options()
    sys, st = _as_sparse(sys)
    if st != PHC_OK:
        return SolveResult(), st
    t, st = sys.table()
    if st != PHC_OK:
        return SolveResult(), st
    n = sys.nvars()
    npaths = int(L.phc_bezout(ctypes.byref(t)))
    if npaths < 1:
        return SolveResult(), ERR_INVALID_INPUT
    bufs, rc = buffers if buffers is not None else _result_buffers(n, npaths)
    st = L.phc_solve_sparse(ctypes.byref(t), ctypes.byref(o), ctypes.byref(g), ctypes.byref(rc))
    _check_device_status(st, "phc_solve_sparse")
    if st != PHC_OK:
        return SolveResult(), st
    return _fill_result(n, npaths, bufs, rc), st


def homotopy_init(sys, seed=1):
    """gen%seed(seed); hom%init(sys, gen, status): returns (gamma, b, patch,
    nstart, status) as drawn by the reference generator."""
    L = _abi.lib()
    t, st = sys.table()
    if st != PHC_OK:
        return None, None, None, 0, st
    n = sys.nvars()
    g = np.zeros(1, dtype=np.complex128)
    b = np.zeros(n, dtype=np.complex128)
    a = np.zeros(n + 1, dtype=np.complex128)
    ns = ctypes.c_int64(0)
    st = L.phc_homotopy_init(ctypes.byref(t), int(seed), _abi.dptr(g.view(np.float64)),
                             _abi.dptr(b.view(np.float64)), _abi.dptr(a.view(np.float64)),
                             ctypes.byref(ns))
    return complex(g[0]), b, a, int(ns.value), st


def _homotopy_struct(gamma, b, patch):
    b = np.ascontiguousarray(b, dtype=np.complex128)
    patch = np.ascontiguousarray(patch, dtype=np.complex128)
    h = _abi.HomotopyC()
    h.gamma[0] = complex(gamma).real
    h.gamma[1] = complex(gamma).imag
    h.b = _abi.dptr(b.view(np.float64))
    h.patch = _abi.dptr(patch.view(np.float64))
    return h, (b, patch)


def solve_paths(sys, options=None, gpu=None, k0=1, count=None, seed=None):
    """Per-path numerics (start_solution + endpoint + classify) for the
    1-based paths k0 .. k0+count-1. Returns (paths, z, x, status)."""
    L = _abi.lib()
    o = options if options is not None else default_options()
    g = gpu if gpu is not None else default_gpu_options()
    sys, st = _as_sparse(sys)
    if st != PHC_OK:
        return None, None, None, st
    gamma, b, patch, nstart, st = homotopy_init(sys, o.seed if seed is None else seed)
    if st != PHC_OK:
        return None, None, None, st
    if count is None:
        count = nstart - k0 + 1
    n = sys.nvars()
    t, _ = sys.table()
    h, keep = _homotopy_struct(gamma, b, patch)
    paths = np.zeros(max(count, 1), dtype=PATH_DTYPE)
    z = np.zeros((max(count, 1), n + 1), dtype=np.complex128)
    x = np.zeros((max(count, 1), n), dtype=np.complex128)
    st = L.phc_solve_paths(ctypes.byref(t), ctypes.byref(h), ctypes.byref(o), ctypes.byref(g),
                           int(k0), int(count), paths.ctypes.data_as(ctypes.c_void_p),
                           _abi.dptr(z.view(np.float64)), _abi.dptr(x.view(np.float64)))
    _check_device_status(st, "phc_solve_paths")
    return paths[:count], z[:count], x[:count], st


class Graph:
    """An instantiated CUDA graph of one plan launch (phc_graph_*)."""

    def __init__(self, L, h):
        self._L, self.h = L, h

    def launch(self, stream=0):
        st = self._L.phc_graph_launch(self.h, ctypes.c_void_p(stream))
        if st != PHC_OK:
            raise PhcError(st, "phc_graph_launch")

    def close(self):
        if self.h:
            self._L.phc_graph_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def autotune(sys, options=None, gpu=None, sample_paths=0):
    """Chooses the launch configuration (schedule, warps per block, refill
    chunk) by timing the tracker on a sample of the system's paths
    (phc_autotune). Returns (gpu_options, report): the options carry the
    winner, and the report lists every candidate with its time in ms. The
    choice is also remembered for this process: later plans and solves
    that leave warps_per_block or chunk at 0 on the same device, precision,
    schedule and row width use it."""
    L = _abi.lib()
    t, st = sys.table()
    if st != PHC_OK:
        raise PhcError(st, "table")
    o = options if options is not None else default_options()
    g = gpu if gpu is not None else default_gpu_options()
    g2 = _abi.GpuOptions()
    ctypes.memmove(ctypes.byref(g2), ctypes.byref(g), ctypes.sizeof(g))
    rep = _abi.TuneReport()
    st = L.phc_autotune(ctypes.byref(t), ctypes.byref(o), ctypes.byref(g2), int(sample_paths),
                        ctypes.byref(rep))
    _check_device_status(st, "phc_autotune")
    if st != PHC_OK:
        raise PhcError(st, "phc_autotune")
    cands = [{"schedule": rep.schedule[i], "warps_per_block": rep.warps_per_block[i],
              "chunk": rep.chunk[i], "ms": rep.ms[i]} for i in range(rep.ncand)]
    return g2, {"candidates": cands, "best": rep.best, "sample_paths": rep.sample_paths}


class Plan:
    """Device-resident plan: the compiled table lives in device memory and
    launches write device buffers (phc_plan_create / phc_plan_launch)."""

    def __init__(self, sys, options=None, gpu=None, seed=None):
        self._L = _abi.lib()
        o = options if options is not None else default_options()
        g = gpu if gpu is not None else default_gpu_options()
        gamma, b, patch, nstart, st = homotopy_init(sys, o.seed if seed is None else seed)
        if st != PHC_OK:
            raise PhcError(st, "homotopy_init")
        t, _ = sys.table()
        h, keep = _homotopy_struct(gamma, b, patch)
        self.h = ctypes.c_void_p()
        st = self._L.phc_plan_create(ctypes.byref(t), ctypes.byref(h), ctypes.byref(o),
                                     ctypes.byref(g), ctypes.byref(self.h))
        if st != PHC_OK:
            raise PhcError(st, "phc_plan_create")
        self.n = sys.nvars()
        self.npaths = nstart

    def launch(self, k0, count, d_out, d_z, stream=0):
        st = self._L.phc_plan_launch(self.h, int(k0), int(count), ctypes.c_void_p(d_out),
                                     ctypes.c_void_p(d_z), ctypes.c_void_p(stream))
        if st != PHC_OK:
            raise PhcError(st, "phc_plan_launch")

    def graph(self, k0, count, d_out, d_z):
        """CUDA graph of launch(k0, count, d_out, d_z) (phc_graph_create);
        replay it with Graph.launch(stream)."""
        h = ctypes.c_void_p()
        st = self._L.phc_graph_create(self.h, int(k0), int(count), ctypes.c_void_p(d_out),
                                      ctypes.c_void_p(d_z), ctypes.byref(h))
        if st != PHC_OK:
            raise PhcError(st, "phc_graph_create")
        return Graph(self._L, h)

    def config(self):
        w, g, s, nm, tb = (ctypes.c_int32(), ctypes.c_int32(), ctypes.c_int32(),
                           ctypes.c_int32(), ctypes.c_int32())
        self._L.phc_plan_config(self.h, ctypes.byref(w), ctypes.byref(g), ctypes.byref(s),
                                ctypes.byref(nm), ctypes.byref(tb))
        return dict(warps_per_block=w.value, grid=g.value, smem=s.value, nm=nm.value,
                    table_bytes=tb.value)

    def close(self):
        if self.h:
            self._L.phc_plan_destroy(self.h)
            self.h = ctypes.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def result_from_arrays(n, paths, x, options=None):
    """Host bookkeeping of solve() (add_solution, add_singular, find,
    collect_real; src/solve.f90:193-213, :330-426) applied to per-path
    records in path order, through the library (phc_finish_solve): for
    paths produced by device-resident plans or gathered from several
    GPUs. z of the result is left zero."""
    L = _abi.lib()
    o = options if options is not None else default_options()
    npaths = len(paths)
    bufs, rc = _result_buffers(n, npaths)
    bufs["paths"][:npaths] = paths
    bufs["x"][:npaths, :n] = x
    st = L.phc_finish_solve(int(n), int(npaths), ctypes.byref(o),
                            bufs["paths"].ctypes.data_as(ctypes.c_void_p),
                            _abi.dptr(bufs["x"].view(np.float64)), ctypes.byref(rc))
    if st != PHC_OK:
        raise PhcError(st, "phc_finish_solve")
    return _fill_result(n, npaths, bufs, rc)


class Server:
    """Serving loop with continuous batching (phc_server_*): requests are
    whole solves; the library's engine thread admits them into batches as
    slots (CUDA streams) and the device-memory budget free up, while other
    batches are still running."""

    def __init__(self, device=0, nslots=4, max_batch_systems=64, max_batch_paths=1 << 16,
                 mem_budget_bytes=1 << 30, gpu=None):
        self._L = _abi.lib()
        cfg = _abi.ServerConfig()
        cfg.device = device
        cfg.nslots = nslots
        cfg.max_batch_systems = max_batch_systems
        cfg.max_batch_paths = max_batch_paths
        cfg.mem_budget_bytes = mem_budget_bytes
        cfg.gpu = gpu if gpu is not None else default_gpu_options(device=device)
        self.h = ctypes.c_void_p()
        st = self._L.phc_server_create(ctypes.byref(cfg), ctypes.byref(self.h))
        if st != PHC_OK:
            raise PhcError(st, "phc_server_create")
        self.n_of = {}

    def submit(self, sys, options=None):
        """Returns (ticket, status); status != 0 means the request was refused
        (err_invalid_input, PHC_ERR_ADMISSION, ...). sys is a SparseSystem or
        a PolySystem (sampled first; the server compiles its own copy)."""
        sys, st = _as_sparse(sys)
        if st != PHC_OK:
            return None, st
        t, st = sys.table()
        if st != PHC_OK:
            return None, st
        o = options if options is not None else default_options()
        ticket = ctypes.c_uint64()
        st = self._L.phc_server_submit(self.h, ctypes.byref(t), ctypes.byref(o),
                                       ctypes.byref(ticket))
        if st != PHC_OK:
            return None, st
        self.n_of[ticket.value] = sys.nvars()
        return ticket.value, st

    def submit_request(self, data, n):
        """Submits a request in the compact format (phc_server_submit_request);
        n is its number of unknowns (for sizing the result). Returns
        (ticket, status)."""
        buf = ctypes.create_string_buffer(bytes(data), max(len(data), 1))
        ticket = ctypes.c_uint64()
        st = self._L.phc_server_submit_request(self.h, buf, len(data), ctypes.byref(ticket))
        if st != PHC_OK:
            return None, st
        self.n_of[ticket.value] = int(n)
        return ticket.value, st

    def poll(self, ticket):
        done = ctypes.c_int32()
        st = self._L.phc_server_poll(self.h, ctypes.c_uint64(ticket), ctypes.byref(done))
        return st, bool(done.value)

    def wait(self, ticket, timeout_ms=-1):
        return self._L.phc_server_wait(self.h, ctypes.c_uint64(ticket), int(timeout_ms))

    def result(self, ticket):
        """(SolveResult, status, latency_s); releases the ticket."""
        n = self.n_of.pop(ticket)
        npaths = int(self._L.phc_server_npaths(self.h, ctypes.c_uint64(ticket)))
        bufs, rc = _result_buffers(n, max(npaths, 1))
        lat = ctypes.c_double()
        st = self._L.phc_server_result(self.h, ctypes.c_uint64(ticket), ctypes.byref(rc),
                                       ctypes.byref(lat))
        if st != PHC_OK:
            return None, st, lat.value
        return _fill_result(n, npaths, bufs, rc), st, lat.value

    def stats(self):
        v = [ctypes.c_int64() for _ in range(4)]
        self._L.phc_server_stats(self.h, *[ctypes.byref(x) for x in v])
        return dict(submitted=v[0].value, completed=v[1].value, batches=v[2].value,
                    in_flight=v[3].value)

    def close(self):
        if self.h:
            self._L.phc_server_destroy(self.h)
            self.h = ctypes.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
