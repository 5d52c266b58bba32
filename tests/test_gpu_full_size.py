"""The two large benchmark workloads at their full sizes, checked through
properties that do not need the restatement to finish every path:

- n=10, degrees 2, 20 of 66 monomials per equation, 1024 paths;
- n=16, degrees 2, 24 of 153 monomials per equation, 65536 paths.

For each: the mixed FP32/FP64 tracker and the plain FP64 tracker classify
every path identically and agree on every finite regular endpoint within
1e-10 (max norm relative to max(1, |x|)); the counts add up (every path is
regular, singular, at infinity or failed; duplicates and multiplicities
account for the paths that found an earlier solution); every regular
solution has a residual at the reference's refine level; and windows of
paths at the start, middle and end of the path range match the
restatement path by path."""
import numpy as np
import pytest

import polyhomocont_b200 as P
from polyhomocont_b200 import workloads as W

pytestmark = pytest.mark.gpu

TOL = 1e-10


@pytest.fixture(scope="module", autouse=True)
def need_gpu():
    import torch
    if not torch.cuda.is_available():
        pytest.fail("GPU tests need a CUDA device")


WORKLOADS = {"n10_1024paths": W.cfg2, "n16_65536paths": W.cfg5}


def check_counts(res):
    p = res.paths
    regular = (p["status"] == 0) & (p["at_infinity"] == 0) & (p["singular"] == 0)
    singular = (p["status"] == 0) & (p["at_infinity"] == 0) & (p["singular"] != 0)
    infinite = (p["status"] == 0) & (p["at_infinity"] != 0)
    failed = p["status"] != 0
    assert regular.sum() + singular.sum() + infinite.sum() + failed.sum() == res.npaths
    assert res.ninfinite == infinite.sum() and res.nfailed == failed.sum()
    # each regular path either starts a solution or repeats an earlier one
    assert res.nsolutions + res.nduplicates == regular.sum()
    assert np.all(p["solution_index"][regular] >= 1)
    assert np.all(p["solution_index"][regular] <= res.nsolutions)
    assert np.all(p["solution_index"][~regular] == 0)
    # multiplicities count the singular paths per singular solution
    assert int(np.sum(res.multiplicities)) == singular.sum()
    assert res.nreal <= res.nsolutions
    return regular


@pytest.mark.parametrize("name", list(WORKLOADS))
def test_mixed_and_fp64_agree_at_full_size(name):
    n, eqs = WORKLOADS[name]()
    s = W.build(P.SparseSystem, n, eqs)
    r64, st1 = P.solve(s, gpu=P.default_gpu_options(precision=P.PHC_PREC_FP64))
    rmx, st2 = P.solve(s, gpu=P.default_gpu_options(precision=P.PHC_PREC_MIXED))
    assert st1 == st2 == 0
    assert r64.npaths == rmx.npaths == s.bezout()
    for key in ("status", "winding_number", "at_infinity", "singular", "is_real",
                "solution_index", "singular_index"):
        assert np.array_equal(r64.paths[key], rmx.paths[key]), key
    for key in ("nsolutions", "nreal", "nsingular", "ninfinite", "nfailed", "nduplicates"):
        assert getattr(r64, key) == getattr(rmx, key), key
    regular = check_counts(r64)
    check_counts(rmx)
    if regular.any():
        d = np.max(np.abs(rmx.x[regular] - r64.x[regular]), axis=1) / np.maximum(
            1.0, np.max(np.abs(r64.x[regular]), axis=1))
        assert d.max() <= TOL, d.max()
        # the refine stage ends at a backward error near machine precision
        assert np.max(r64.paths["residual"][regular]) <= 1e-12
        assert np.max(rmx.paths["residual"][regular]) <= 1e-12


@pytest.mark.parametrize("name", list(WORKLOADS))
def test_path_windows_match_the_restatement(orc, name):
    n, eqs = WORKLOADS[name]()
    so = W.build(orc.SparseSystem, n, eqs)
    sp = W.build(P.SparseSystem, n, eqs)
    npaths = sp.bezout()
    for k0 in (1, npaths // 2 - 7, npaths - 15):
        pr, zr, xr, st = orc.solve_paths(so, k0=k0, count=16, nthreads=8)
        assert st == 0
        for prec in (P.PHC_PREC_FP64, P.PHC_PREC_MIXED):
            pg, zg, xg, st2 = P.solve_paths(sp, gpu=P.default_gpu_options(precision=prec),
                                            k0=k0, count=16)
            assert st2 == 0
            for key in ("status", "winding_number", "at_infinity", "singular", "is_real"):
                assert np.array_equal(pg[key], pr[key]), (key, k0, prec)
            fin = (pr["status"] == 0) & (pr["at_infinity"] == 0)
            if fin.any():
                d = np.max(np.abs(xg[fin] - xr[fin]), axis=1) / np.maximum(
                    1.0, np.max(np.abs(xr[fin]), axis=1))
                assert d.max() <= TOL, (d.max(), k0, prec)
