"""CUDA graphs of plan launches (phc_graph_*): a replayed graph produces
exactly what the direct launch produces, on repeated replays, for both
schedules (the persistent schedule's queue reset is part of the graph)."""
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


@pytest.mark.parametrize("schedule", [P.PHC_SCHED_PERSISTENT, P.PHC_SCHED_GRID])
@pytest.mark.parametrize("precision", [P.PHC_PREC_FP64, P.PHC_PREC_MIXED])
def test_graph_replay_matches_direct_launch(schedule, precision):
    import torch
    n, eqs = W.katsura(4)
    s = W.build(P.SparseSystem, n, eqs)
    npaths = s.bezout()
    plan = P.Plan(s, gpu=P.default_gpu_options(precision, schedule))
    dev = torch.device("cuda", 0)
    out_a = torch.zeros(npaths * 96, dtype=torch.uint8, device=dev)
    z_a = torch.zeros(npaths * (n + 1) * 2, dtype=torch.float64, device=dev)
    out_b = torch.zeros_like(out_a)
    z_b = torch.full_like(z_a, float("nan"))
    stream = torch.cuda.current_stream(dev)
    try:
        plan.launch(1, npaths, out_a.data_ptr(), z_a.data_ptr(), stream.cuda_stream)
        g = plan.graph(1, npaths, out_b.data_ptr(), z_b.data_ptr())
        try:
            for _ in range(2):
                out_b.zero_()
                z_b.fill_(float("nan"))
                g.launch(stream.cuda_stream)
                torch.cuda.synchronize()
                assert torch.equal(out_a, out_b)
                assert torch.equal(z_a, z_b)
        finally:
            g.close()
    finally:
        plan.close()
    p = np.frombuffer(out_a.cpu().numpy().tobytes(), dtype=P.PATH_DTYPE)
    assert (p["status"] == 0).all()
