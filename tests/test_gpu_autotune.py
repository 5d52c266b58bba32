"""The launch-configuration autotuner (phc_autotune): it times every
candidate on a sample of paths, returns the fastest, and the tuned values
are picked up by later plans that leave warps_per_block and chunk at 0.
The launch configuration never changes a path's arithmetic, so results
with the tuned options equal the results with the defaults."""
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
def test_autotune_picks_the_fastest_candidate(precision):
    s = W.build(P.SparseSystem, *W.cfg2())
    g, rep = P.autotune(s, gpu=P.default_gpu_options(precision), sample_paths=256)
    cands = rep["candidates"]
    assert len(cands) >= 6 and rep["sample_paths"] == 256
    assert {c["schedule"] for c in cands} == {P.PHC_SCHED_GRID, P.PHC_SCHED_PERSISTENT}
    assert all(c["ms"] > 0 for c in cands)
    best = cands[rep["best"]]
    assert best["ms"] == min(c["ms"] for c in cands)
    assert (g.schedule, g.warps_per_block, g.chunk) == (best["schedule"],
                                                        best["warps_per_block"], best["chunk"])
    # a plan that leaves warps_per_block at 0 gets the tuned value
    g0 = P.default_gpu_options(precision, best["schedule"])
    plan = P.Plan(s, gpu=g0)
    try:
        assert plan.config()["warps_per_block"] == best["warps_per_block"]
    finally:
        plan.close()


def test_tuned_options_give_the_same_results():
    s = W.build(P.SparseSystem, *W.dense_quadratic())
    ref, st = P.solve(s)
    assert st == 0
    g, _ = P.autotune(s, sample_paths=16)
    res, st2 = P.solve(s, gpu=g)
    assert st2 == 0
    for key in ("nsolutions", "nreal", "nsingular", "ninfinite", "nfailed", "nduplicates"):
        assert getattr(res, key) == getattr(ref, key), key
    for key in ("status", "winding_number", "at_infinity", "singular", "is_real",
                "naccepted", "nrejected", "solution_index"):
        assert np.array_equal(res.paths[key], ref.paths[key]), key
    assert np.array_equal(res.x, ref.x)  # same arithmetic per path: bit-identical
