"""GPU test of phc_solve_paths_noalloc, the entry point for callers that
cannot allocate device memory (graph-capture regions, pre-reserved memory
pools, hosts that forbid allocations after start-up).

It is called twice in a row through the C ABI, writing into device buffers
the test owns, and each result must match phc_solve_paths (which allocates
its own device buffers): identical path status and classification, and
endpoints within the parity tolerance of the tracker tests (1e-10). The
second call checks that the shared scratch array (compiled table, zeroed
queue counter) is reused correctly. Kept in its own file, collected last.
"""
import ctypes

import numpy as np
import pytest

import polyhomocont_b200 as P
from polyhomocont_b200 import _abi
from polyhomocont_b200 import workloads as W

pytestmark = pytest.mark.gpu
TOL = 1e-10


def _call_noalloc(sys, o, g, count, d_out, d_z, d_x, stream):
    gamma, b, patch, nstart, st = P.homotopy_init(sys, o.seed)
    assert st == 0
    t, _ = sys.table()
    h, keep = P._homotopy_struct(gamma, b, patch)
    return _abi.lib().phc_solve_paths_noalloc(
        ctypes.byref(t), ctypes.byref(h), ctypes.byref(o), ctypes.byref(g), 1, int(count),
        ctypes.c_void_p(d_out), ctypes.c_void_p(d_z), ctypes.c_void_p(d_x),
        ctypes.c_void_p(stream))


@pytest.mark.parametrize("name", ["katsura4", "cyclic5", "cfg2"])
def test_noalloc_matches_allocating_entry_point(name):
    import torch
    if not torch.cuda.is_available():
        pytest.fail("GPU test needs a CUDA device")
    n, eqs = {"katsura4": lambda: W.katsura(4), "cyclic5": lambda: W.cyclic(5),
              "cfg2": W.cfg2}[name]()
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
        for key in ("status", "winding_number", "at_infinity", "singular", "is_real",
                    "endgame_status"):
            assert np.array_equal(p[key], ref_p[key]), (call, key)
        fin = (ref_p["status"] == 0) & (ref_p["at_infinity"] == 0)
        d = np.max(np.abs(x[fin] - ref_x[fin]), axis=1) / np.maximum(
            1.0, np.max(np.abs(ref_x[fin]), axis=1))
        assert d.max() <= TOL, (call, d.max())


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
