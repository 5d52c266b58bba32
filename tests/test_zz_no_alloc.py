"""GPU test of phc_solve_paths_noalloc, the entry point for callers that
cannot allocate device memory: services whose device memory is reserved and
accounted for up front, and hosts that forbid device allocations after
start-up because an allocation can block or fail at an unpredictable moment.

The entry point is called through the C ABI, writing into device buffers
the test owns, and each result must match phc_solve_paths (which allocates
its own device buffers): identical path status and classification, and
endpoints within the parity tolerance of the tracker tests (1e-10). Every
case makes two calls in a row. Two different systems are enqueued back to
back on one stream with no synchronization in between, so the second call
must rewrite the compiled table and clear the queue counter that the first
left in the shared scratch array. A sub-range of paths (k0 > 1) with no x
output covers the remaining arguments. Kept in its own file, collected last.
"""
import ctypes

import numpy as np
import pytest

import polyhomocont_b200 as P
from polyhomocont_b200 import _abi
from polyhomocont_b200 import workloads as W

pytestmark = pytest.mark.gpu
TOL = 1e-10


def _call_noalloc(sys, o, g, count, d_out, d_z, d_x, stream, k0=1):
    gamma, b, patch, nstart, st = P.homotopy_init(sys, o.seed)
    assert st == 0
    t, _ = sys.table()
    h, keep = P._homotopy_struct(gamma, b, patch)
    return _abi.lib().phc_solve_paths_noalloc(
        ctypes.byref(t), ctypes.byref(h), ctypes.byref(o), ctypes.byref(g), int(k0), int(count),
        ctypes.c_void_p(d_out), ctypes.c_void_p(d_z), ctypes.c_void_p(d_x),
        ctypes.c_void_p(stream))


SYSTEMS = {"katsura4": lambda: W.katsura(4), "cyclic5": lambda: W.cyclic(5), "cfg2": W.cfg2}


def _assert_same(p, x, ref_p, ref_x, tag):
    for key in ("status", "winding_number", "at_infinity", "singular", "is_real",
                "endgame_status"):
        assert np.array_equal(p[key], ref_p[key]), (tag, key)
    fin = (ref_p["status"] == 0) & (ref_p["at_infinity"] == 0)
    if x is not None and fin.any():
        d = np.max(np.abs(x[fin] - ref_x[fin]), axis=1) / np.maximum(
            1.0, np.max(np.abs(ref_x[fin]), axis=1))
        assert d.max() <= TOL, (tag, d.max())


@pytest.mark.parametrize("name", list(SYSTEMS))
def test_noalloc_matches_allocating_entry_point(name):
    import torch
    if not torch.cuda.is_available():
        pytest.fail("GPU test needs a CUDA device")
    n, eqs = SYSTEMS[name]()
    sys = W.build(P.SparseSystem, n, eqs)
    o = P.default_options()
    g = P.default_gpu_options(P.PHC_PREC_MIXED, P.PHC_SCHED_PERSISTENT)
    npaths = sys.bezout()
    ref_p, ref_z, ref_x, st = P.solve_paths(sys, o, g)
    assert st == 0
    dev = torch.device("cuda", 0)
    d_out = torch.zeros(npaths * P.PATH_DTYPE.itemsize, dtype=torch.uint8, device=dev)
    d_z = torch.zeros(npaths * (n + 1) * 2, dtype=torch.float64, device=dev)
    d_x = torch.zeros(npaths * n * 2, dtype=torch.float64, device=dev)
    stream = torch.cuda.current_stream(dev)
    for call in range(2):
        d_out.fill_(0xFF)  # garbage from a previous use must not leak through
        st = _call_noalloc(sys, o, g, npaths, d_out.data_ptr(), d_z.data_ptr(),
                           d_x.data_ptr(), stream.cuda_stream)
        assert st == 0, (call, _abi.last_error())
        stream.synchronize()
        p = np.frombuffer(d_out.cpu().numpy().tobytes(), dtype=P.PATH_DTYPE)
        x = d_x.cpu().numpy().view(np.complex128).reshape(npaths, n)
        _assert_same(p, x, ref_p, ref_x, (name, call))


@pytest.mark.parametrize("precision", [P.PHC_PREC_FP64, P.PHC_PREC_MIXED])
def test_noalloc_two_systems_back_to_back(precision):
    """Two different systems enqueued on one stream without a
    synchronization between them, twice in a row: the second call of each
    pair finds the other system's table and a used queue counter in the
    shared array. The second system tracks only paths 7..31 (k0 > 1, a
    sub-range) and asks for no x."""
    import torch
    if not torch.cuda.is_available():
        pytest.fail("GPU test needs a CUDA device")
    o = P.default_options()
    g = P.default_gpu_options(precision, P.PHC_SCHED_PERSISTENT)
    dev = torch.device("cuda", 0)
    stream = torch.cuda.current_stream(dev)
    na, eqa = W.katsura(4)
    nb, eqb = W.cyclic(5)
    sa = W.build(P.SparseSystem, na, eqa)
    sb = W.build(P.SparseSystem, nb, eqb)
    pa_ref, _, xa_ref, st = P.solve_paths(sa, o, g)
    assert st == 0
    k0b, countb = 7, 25
    pb_ref, zb_ref, _, st = P.solve_paths(sb, o, g, k0=k0b, count=countb)
    assert st == 0
    npa = sa.bezout()
    oa = torch.zeros(npa * P.PATH_DTYPE.itemsize, dtype=torch.uint8, device=dev)
    za = torch.zeros(npa * (na + 1) * 2, dtype=torch.float64, device=dev)
    xa = torch.zeros(npa * na * 2, dtype=torch.float64, device=dev)
    ob = torch.zeros(countb * P.PATH_DTYPE.itemsize, dtype=torch.uint8, device=dev)
    zb = torch.zeros(countb * (nb + 1) * 2, dtype=torch.float64, device=dev)
    for rep in range(2):
        oa.fill_(0xFF)
        ob.fill_(0xFF)
        st = _call_noalloc(sa, o, g, npa, oa.data_ptr(), za.data_ptr(), xa.data_ptr(),
                           stream.cuda_stream)
        assert st == 0, _abi.last_error()
        st = _call_noalloc(sb, o, g, countb, ob.data_ptr(), zb.data_ptr(), 0,
                           stream.cuda_stream, k0=k0b)
        assert st == 0, _abi.last_error()
        stream.synchronize()
        pa = np.frombuffer(oa.cpu().numpy().tobytes(), dtype=P.PATH_DTYPE)
        x = xa.cpu().numpy().view(np.complex128).reshape(npa, na)
        _assert_same(pa, x, pa_ref, xa_ref, ("katsura4", rep))
        pb = np.frombuffer(ob.cpu().numpy().tobytes(), dtype=P.PATH_DTYPE)
        _assert_same(pb, None, pb_ref, None, ("cyclic5 paths 7..31", rep))
        # without x, compare the projective endpoints z of the finite paths
        z = zb.cpu().numpy().view(np.complex128).reshape(countb, nb + 1)
        fin = (pb_ref["status"] == 0) & (pb_ref["at_infinity"] == 0)
        assert fin.any()
        d = np.max(np.abs(z[fin] - zb_ref[fin]), axis=1) / np.maximum(
            1.0, np.max(np.abs(zb_ref[fin]), axis=1))
        assert d.max() <= TOL, ("cyclic5 z", rep, d.max())


def test_noalloc_rejects_oversize_table():
    """A system whose compiled table exceeds the 256 KiB scratch array is
    refused with PHC_ERR_UNSUPPORTED before anything is launched."""
    import torch
    if not torch.cuda.is_available():
        pytest.fail("GPU test needs a CUDA device")
    n = 24  # all 325 monomials of degree <= 2 per equation: a 359 KiB table
    sys = P.SparseSystem(n)
    mons = W.monomials(n, 2)
    for i in range(n):
        coefs = np.full(len(mons), 1.0 + 0.5j)
        exps = np.array(mons, dtype=np.int32).T
        assert sys.add_equation(coefs, exps) == 0
    o = P.default_options()
    gpu = P.default_gpu_options()
    dev = torch.device("cuda", 0)
    buf = torch.zeros(1024, dtype=torch.float64, device=dev)
    st = _call_noalloc(sys, o, gpu, 4, buf.data_ptr(), buf.data_ptr(), 0, 0)
    assert st == _abi.PHC_ERR_UNSUPPORTED
    assert "256 KiB" in _abi.last_error()
