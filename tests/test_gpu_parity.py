"""Parity of the CUDA path (through the C ABI) with the CPU restatement of
the reference's solve(), on the reference's own cases and the benchmark
configurations, in both precision modes.

Parity criteria (from the reference's solve() contract): identical status,
winding number, at-infinity/singular/real classification and solution
indices per path; identical counts of regular, real, singular
(multiplicities), infinite, failed and duplicate paths; finite regular
endpoints within 1e-10 relative (max-norm, relative to max(1, |x|));
singular endpoints within 1e-6 relative (the reference's
singular_dedup_tol, since such endpoints are less accurate)."""
import json
import os

import numpy as np
import pytest

import polyhomocont_b200 as P
from polyhomocont_b200 import workloads as W
from tests.helpers import TOL_REGULAR, assert_parity, set_distance

pytestmark = pytest.mark.gpu

GOLDEN = os.path.join(os.path.dirname(__file__), "golden")


@pytest.fixture(scope="module", autouse=True)
def need_gpu():
    import torch
    if not torch.cuda.is_available():
        pytest.fail("GPU tests need a CUDA device")


def cases():
    out = {}
    out["univariate5"] = (1, [(np.poly([0.5, -3j, 3j, -2, 1])[::-1], np.array([[0, 1, 2, 3, 4, 5]]))])
    out["2x2"] = (2, [([1, 1, -5], [[2, 0, 0], [0, 2, 0]]), ([1, -2], [[1, 0], [1, 0]])])
    out["infinity"] = (2, [([1, -1], [[1, 0], [1, 0]]), ([1, -4], [[2, 0], [0, 0]])])
    out["double_root"] = (1, [([1, -1, -1, 1], [[3, 2, 1, 0]])])
    out["mixed"] = (2, [([1, -1], [[1, 0], [1, 0]]), ([1, -3, 2], [[3, 1, 0], [0, 0, 0]])])
    out["multiplicity4"] = (2, [([1], [[2], [0]]), ([1, 1], [[0, 1], [2, 1]])])
    out["triple_root"] = (1, [([1, -1, -3, 5, -2], [[4, 3, 2, 1, 0]])])
    out["katsura3"] = W.katsura(3)
    out["katsura4"] = W.katsura(4)
    out["cyclic5"] = W.cyclic(5)
    out["cfg1"] = W.dense_quadratic()
    out["cfg3"] = W.singular_cubic()[:2]
    return out


CASES = cases()


def solve_both(orc, name, precision, options=None, schedule=P.PHC_SCHED_PERSISTENT):
    n, eqs = CASES[name] if isinstance(name, str) else name
    so = W.build(orc.SparseSystem, n, eqs)
    sp = W.build(P.SparseSystem, n, eqs)
    oo = orc.default_options()
    po = P.default_options()
    if options:
        for k, v in options.items():
            setattr(oo, k, v)
            setattr(po, k, v)
    ref, st1 = orc.solve(so, oo, nthreads=4)
    g = P.default_gpu_options(precision=precision, schedule=schedule)
    got, st2 = P.solve(sp, po, g)
    assert st1 == st2 == 0
    return n, ref, got


@pytest.mark.parametrize("precision", [P.PHC_PREC_FP64, P.PHC_PREC_MIXED])
@pytest.mark.parametrize("name", list(CASES))
def test_parity_reference_cases(orc, name, precision):
    n, ref, got = solve_both(orc, name, precision)
    assert_parity(n, ref, got)


@pytest.mark.parametrize("precision", [P.PHC_PREC_FP64, P.PHC_PREC_MIXED])
def test_known_answers_on_gpu(orc, precision):
    """The reference's own expected values (test/solve.f90, test/katsura.f90)
    on the GPU path directly."""
    g = P.default_gpu_options(precision=precision)
    n, eqs = CASES["mixed"]
    res, st = P.solve(W.build(P.SparseSystem, n, eqs), gpu=g)
    assert st == 0 and res.npaths == 6 and res.nsolutions == 1 and res.ninfinite == 3
    assert np.max(np.abs(res.solutions[0] - [-2, -0.5])) <= 1e-12
    assert res.nsingular == 1 and res.multiplicities[0] == 2
    assert np.max(np.abs(res.singular_solutions[0] - 1)) <= 1e-10
    gold = json.load(open(os.path.join(GOLDEN, "katsura.json")))["katsura4"]
    refs = np.array([[complex(a, b) for a, b in s] for s in gold["solutions"]])
    res, st = P.solve(W.build(P.SparseSystem, *W.katsura(4)), gpu=g)
    assert res.nsolutions == 16 and res.nreal == 12 and res.nfailed == 0
    assert set_distance(res.solutions, refs) <= 1e-12
    assert np.max(res.paths["residual"]) <= 1e-14


@pytest.mark.parametrize("schedule", [P.PHC_SCHED_GRID, P.PHC_SCHED_PERSISTENT])
def test_schedules_agree(orc, schedule):
    n, ref, got = solve_both(orc, "cyclic5", P.PHC_PREC_FP64, schedule=schedule)
    assert_parity(n, ref, got)


def test_without_endgame(orc):
    n, ref, got = solve_both(orc, "2x2", P.PHC_PREC_FP64, options={"use_endgame": 0})
    assert_parity(n, ref, got)
    assert got.nsolutions == 4


def test_seeds(orc):
    for seed in (2, 3, 4):
        n, ref, got = solve_both(orc, "katsura3", P.PHC_PREC_MIXED, options={"seed": seed})
        assert_parity(n, ref, got)


def test_singular_config_exact_root(orc):
    """cfg3: the 16 singular paths end at the exactly known root r."""
    n, eqs, r = W.singular_cubic()
    for prec in (P.PHC_PREC_FP64, P.PHC_PREC_MIXED):
        res, st = P.solve(W.build(P.SparseSystem, n, eqs), gpu=P.default_gpu_options(precision=prec))
        assert res.nsingular == 1 and res.multiplicities[0] == 16
        err = np.max(np.abs(res.singular_solutions[0] - r)) / max(1.0, np.max(np.abs(r)))
        assert err <= 1e-6


def test_cfg2_parity_sample(orc):
    """cfg2 (n = 10, 1024 paths), first 128 paths, mixed precision."""
    n, eqs = W.cfg2()
    so = W.build(orc.SparseSystem, n, eqs)
    sp = W.build(P.SparseSystem, n, eqs)
    pr, zr, xr, st = orc.solve_paths(so, count=128, nthreads=8)
    for prec in (P.PHC_PREC_FP64, P.PHC_PREC_MIXED):
        pg, zg, xg, st2 = P.solve_paths(sp, gpu=P.default_gpu_options(precision=prec), count=128)
        for key in ("status", "winding_number", "at_infinity", "singular", "is_real"):
            assert np.array_equal(pg[key], pr[key]), key
        d = np.max(np.abs(xg - xr), axis=1) / np.maximum(1.0, np.max(np.abs(xr), axis=1))
        assert d.max() <= TOL_REGULAR


@pytest.mark.parametrize("n", [12, 16, 17, 20, 28, 31])
def test_wide_rows_parity_sample(orc, n):
    """Random sparse quadratic systems of every register-row width above the
    benchmark systems' (12, 16, 18, 24 and 32 columns), up to the maximum
    N = n + 1 = 32 unknowns; first 24 paths, both precisions, against the
    restatement."""
    n_, eqs = W.sparse_quadratic(n, 24, W.seed_for(5, 100 + n))
    if n == 31:
        # 2^31 paths exceed the reference's integer bound (src/homotopy.f90:128-132):
        # the last equation is linear, for 2^30 paths
        g = W.Rng(W.seed_for(5, 231))
        eqs[-1] = W.random_sparse(n, 1, 12, g)
    so = W.build(orc.SparseSystem, n_, eqs)
    sp = W.build(P.SparseSystem, n_, eqs)
    pr, zr, xr, st = orc.solve_paths(so, count=24, nthreads=8)
    assert st == 0
    for prec in (P.PHC_PREC_FP64, P.PHC_PREC_MIXED):
        pg, zg, xg, st2 = P.solve_paths(sp, gpu=P.default_gpu_options(precision=prec), count=24)
        assert st2 == 0
        for key in ("status", "winding_number", "at_infinity", "singular", "is_real"):
            assert np.array_equal(pg[key], pr[key]), (key, prec)
        fin = (pr["status"] == 0) & (pr["at_infinity"] == 0)
        if fin.any():
            d = np.max(np.abs(xg[fin] - xr[fin]), axis=1) / np.maximum(
                1.0, np.max(np.abs(xr[fin]), axis=1))
            assert d.max() <= TOL_REGULAR, (d.max(), prec)


@pytest.mark.parametrize("precision", [P.PHC_PREC_FP64, P.PHC_PREC_MIXED])
@pytest.mark.parametrize("name", ["cyclic5", "cfg3", "cfg2", "multiplicity4"])
def test_streamed_solve_equals_tracking_then_bookkeeping(name, precision):
    """phc_solve_sparse overlaps the bookkeeping with the tracking (the
    kernel writes each path into mapped host memory and flags it); its
    result must be byte-identical to tracking every path first
    (phc_solve_paths) and running the bookkeeping afterwards
    (phc_finish_solve), in both precisions and twice in a row (the second
    call reuses the mapped buffers)."""
    n, eqs = W.cfg2() if name == "cfg2" else CASES[name]
    s = W.build(P.SparseSystem, n, eqs)
    g = P.default_gpu_options(precision=precision)
    pg, zg, xg, st = P.solve_paths(s, gpu=g)
    assert st == 0
    ref = P.result_from_arrays(n, pg, xg)
    for _ in range(2):
        got, st = P.solve(s, gpu=g)
        assert st == 0
        assert got.paths.tobytes() == ref.paths.tobytes()
        assert np.array_equal(got.z.view(np.float64), np.asarray(zg).reshape(got.z.shape).view(np.float64))
        assert np.array_equal(got.x.view(np.float64), np.asarray(xg).reshape(got.x.shape).view(np.float64))
        for key in ("nsolutions", "nreal", "nsingular", "ninfinite", "nfailed", "nduplicates"):
            assert getattr(got, key) == getattr(ref, key), key
        for key in ("solutions", "real_solutions", "singular_solutions", "multiplicities"):
            assert np.array_equal(getattr(got, key), getattr(ref, key)), key
