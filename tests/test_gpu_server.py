"""Serving loop (continuous batching) on the GPU: every request's result is
the same alone (phc_solve_sparse) and in the mix of concurrently served
requests; oversize and invalid requests are refused on the host without
affecting the others."""
import numpy as np
import pytest

import polyhomocont_b200 as P
from polyhomocont_b200 import _abi
from polyhomocont_b200 import workloads as W

pytestmark = pytest.mark.gpu
TOL = 1e-10


@pytest.fixture(scope="module", autouse=True)
def need_gpu():
    import torch
    if not torch.cuda.is_available():
        pytest.fail("GPU tests need a CUDA device")


def test_results_same_alone_and_in_the_mix():
    systems = [W.build(P.SparseSystem, *W.stream_system(i)) for i in range(24)]
    srv = P.Server(nslots=4, max_batch_systems=5)
    try:
        tickets = []
        for s in systems:
            t, st = srv.submit(s)
            assert st == 0
            tickets.append(t)
        for t in tickets:
            assert srv.wait(t, 120000) == 0
        mixed = [srv.result(t) for t in tickets]
        stats = srv.stats()
    finally:
        srv.close()
    assert stats["completed"] == 24 and stats["batches"] >= 5
    for s, (res, st, lat) in zip(systems, mixed):
        alone, st2 = P.solve(s)
        assert st == st2 == 0 and lat > 0
        for key in ("npaths", "nsolutions", "nreal", "nsingular", "ninfinite", "nfailed",
                    "nduplicates"):
            assert getattr(res, key) == getattr(alone, key), key
        for key in ("status", "winding_number", "at_infinity", "singular", "is_real",
                    "solution_index", "singular_index"):
            assert np.array_equal(res.paths[key], alone.paths[key]), key
        fin = alone.paths["solution_index"] > 0
        if fin.any():
            d = np.max(np.abs(res.x[fin] - alone.x[fin]))
            assert d <= TOL * max(1.0, np.max(np.abs(alone.x[fin])))


def test_admission_and_invalid_requests():
    srv = P.Server(nslots=2, mem_budget_bytes=64 * 1024)
    try:
        big = W.build(P.SparseSystem, *W.cfg2())          # 1024 paths: over the budget
        t, st = srv.submit(big)
        assert t is None and st == _abi.PHC_ERR_ADMISSION
        bad = P.SparseSystem(2)
        bad.add_equation([1, -1], [[2, 0], [0, 0]])        # one equation for two unknowns
        t, st = srv.submit(bad)
        assert t is None and st == P.ERR_INVALID_INPUT
        ok = W.build(P.SparseSystem, *W.katsura(3))
        t, st = srv.submit(ok)
        assert st == 0 and srv.wait(t, 60000) == 0
        res, st, lat = srv.result(t)
        assert st == 0 and res.nsolutions == 8
    finally:
        srv.close()


def test_shutdown_with_requests_in_flight():
    """Destroying the server while requests are queued or running returns
    without hanging; in-flight batches finish, queued ones are dropped."""
    srv = P.Server(nslots=1, max_batch_systems=1)
    for i in range(8):
        srv.submit(W.build(P.SparseSystem, *W.stream_system(100 + i)))
    srv.close()


def test_compact_requests_give_the_same_results():
    """A request submitted in the compact wire format is solved exactly
    like the same system submitted as a table."""
    systems = [W.build(P.SparseSystem, *W.stream_system(200 + i)) for i in range(6)]
    srv = P.Server(nslots=2)
    try:
        pairs = []
        for s in systems:
            t1, st1 = srv.submit(s)
            t2, st2 = srv.submit_request(P.encode_request(s, P.default_options()), s.nvars())
            assert st1 == 0 and st2 == 0
            pairs.append((t1, t2))
        for t1, t2 in pairs:
            assert srv.wait(t1, 120000) == 0 and srv.wait(t2, 120000) == 0
            r1, s1, _ = srv.result(t1)
            r2, s2, _ = srv.result(t2)
            assert s1 == s2 == 0
            assert r1.nsolutions == r2.nsolutions and r1.ninfinite == r2.ninfinite
            for key in ("status", "winding_number", "at_infinity", "singular", "is_real",
                        "solution_index"):
                assert np.array_equal(r1.paths[key], r2.paths[key]), key
            assert np.array_equal(r1.x, r2.x)
        bad = b"PHCR" + bytes(20)
        t, st = srv.submit_request(bad, 1)
        assert t is None and st == P.ERR_INVALID_INPUT
    finally:
        srv.close()
