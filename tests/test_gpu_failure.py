"""Failure handling on the device without any GPU fault: the per-path unit
budget (phc_gpu_options.unit_budget_log2) ends paths that would run longer
with the reference's max-steps failure status, the launch returns normally,
and the host counts the failures like the reference's solve() does."""
import numpy as np
import pytest

import polyhomocont_b200 as P
from polyhomocont_b200 import workloads as W

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module", autouse=True)
def need_gpu():
    import torch
    if not torch.cuda.is_available():
        pytest.fail("GPU tests need a CUDA device")


@pytest.mark.parametrize("precision", [P.PHC_PREC_FP64, P.PHC_PREC_MIXED])
def test_unit_budget_ends_paths_with_max_steps_status(precision):
    s = W.build(P.SparseSystem, *W.katsura(3))
    g = P.default_gpu_options(precision)
    g.unit_budget_log2 = 4  # 16 units: far too few for any path
    res, st = P.solve(s, gpu=g)
    assert st == 0
    assert res.npaths == 8 and res.nfailed == 8 and res.nsolutions == 0
    assert (res.paths["status"] == 2).all()          # path_failed_max_steps
    assert (res.paths["n_tangent"] + res.paths["n_newton"] <= 16 + 16).all()  # one step past
    # the default budget leaves every path alone
    ok, st = P.solve(s, gpu=P.default_gpu_options(precision))
    assert st == 0 and ok.nfailed == 0 and ok.nsolutions == 8


def test_unit_budget_in_the_serving_loop():
    """A budget-limited request fails on its own; the requests around it in
    the same batch are unaffected."""
    g = P.default_gpu_options()
    g.unit_budget_log2 = 4
    systems = [W.build(P.SparseSystem, *W.stream_system(300 + i)) for i in range(4)]
    srv_limited = P.Server(nslots=1, gpu=g)
    srv = P.Server(nslots=1)
    try:
        t0, _ = srv_limited.submit(systems[0])
        tickets = [srv.submit(s)[0] for s in systems]
        assert srv_limited.wait(t0, 60000) == 0
        r0, st0, _ = srv_limited.result(t0)
        assert st0 == 0 and r0.nfailed == r0.npaths
        for t in tickets:
            assert srv.wait(t, 120000) == 0
            r, st, _ = srv.result(t)
            assert st == 0 and r.nfailed < r.npaths
    finally:
        srv_limited.close()
        srv.close()
