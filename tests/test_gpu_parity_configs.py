"""Parity of the CUDA path with the CPU restatement of the reference's
solve() on every benchmark configuration, path by path, in both precision
modes:

  - the serving stream: the first 10 systems of each size n = 2..8 of the
    request stream (degrees 2 and 3, 6-30 monomials per equation), each a whole
    solve() (src/solve.f90:154-215) on both sides, bookkeeping included,
    once solved one by one and once submitted together to the serving loop;
  - n = 10 with 1024 paths: every path, and the whole solve();
  - cyclic-6 (test/cyclic.f90:26, check_cyclic(6, 156)): 720 paths, 156
    finite solutions, winding numbers up to 16 at infinity;
  - n = 16 with 65,536 paths: 1024 paths in eight windows of 128 spread
    over the whole range of path indices (the restatement's solve of all
    65,536 paths takes minutes; the rest of the range is covered by the
    full-size property tests).

Criteria are those of the reference's solve() contract: identical status,
winding number, at-infinity / singular / real classification and solution
indices per path; identical counts; finite regular endpoints within 1e-10
relative (max norm), singular solution sets within 1e-6 (the reference's
singular_dedup_tol). The end game status is identical too, except on
paths at infinity whose end game errors on both sides are at most 1e-7: the
flag compares them with 1e-11, and rounding decides it there (a few
cyclic-6 paths, with every form of the kernel). No path may take
pathologically more steps than the restatement's."""
import os

import numpy as np
import pytest

import polyhomocont_b200 as P
from polyhomocont_b200 import workloads as W
from tests.helpers import (TOL_REGULAR, assert_parity, assert_steps_comparable,
                           endgame_status_agrees)

pytestmark = pytest.mark.gpu

PRECISIONS = [P.PHC_PREC_FP64, P.PHC_PREC_MIXED]
NT = os.cpu_count() or 4
STREAM_PER_SIZE = 10
CFG5_WINDOWS = 8
CFG5_WINDOW = 128
PATH_KEYS = ("status", "winding_number", "at_infinity", "singular", "is_real")


@pytest.fixture(scope="module", autouse=True)
def need_gpu():
    import torch
    if not torch.cuda.is_available():
        pytest.fail("GPU tests need a CUDA device")


def stream_indices(per_size=STREAM_PER_SIZE):
    """The first per_size systems of each size n = 2..8 of the stream."""
    picked = {n: [] for n in range(2, 9)}
    i = 0
    while any(len(v) < per_size for v in picked.values()):
        n, _ = W.stream_system(i)
        if len(picked[n]) < per_size:
            picked[n].append(i)
        i += 1
    return sorted(j for v in picked.values() for j in v)


@pytest.fixture(scope="module")
def stream_refs(orc):
    out = []
    for i in stream_indices():
        n, eqs = W.stream_system(i)
        ref, st = orc.solve(W.build(orc.SparseSystem, n, eqs), nthreads=NT)
        assert st == 0
        out.append((i, n, eqs, ref))
    return out


@pytest.mark.parametrize("precision", PRECISIONS)
def test_serving_stream_systems(stream_refs, precision):
    g = P.default_gpu_options(precision=precision)
    sizes = set()
    for i, n, eqs, ref in stream_refs:
        got, st = P.solve(W.build(P.SparseSystem, n, eqs), gpu=g)
        assert st == 0, i
        try:
            assert_parity(n, ref, got)
        except AssertionError as e:
            raise AssertionError(f"stream system {i} (n={n}): {e}") from e
        sizes.add(n)
    assert sizes == set(range(2, 9))  # every size of the stream is covered


@pytest.mark.parametrize("precision", PRECISIONS)
def test_serving_stream_through_the_server(stream_refs, precision):
    """The same systems submitted together to the serving loop (batched
    with each other, several slots in flight): every result equals the
    restatement's solve()."""
    srv = P.Server(nslots=4, max_batch_systems=16,
                   gpu=P.default_gpu_options(precision=precision))
    try:
        tickets = []
        for i, n, eqs, ref in stream_refs:
            t, st = srv.submit(W.build(P.SparseSystem, n, eqs))
            assert st == 0
            tickets.append(t)
        for (i, n, eqs, ref), t in zip(stream_refs, tickets):
            assert srv.wait(t, 600000) == 0
            got, st, _ = srv.result(t)
            assert st == 0, i
            try:
                assert_parity(n, ref, got)
            except AssertionError as e:
                raise AssertionError(f"stream system {i} (n={n}): {e}") from e
    finally:
        srv.close()


@pytest.fixture(scope="module")
def cfg2_ref(orc):
    n, eqs = W.cfg2()
    ref, st = orc.solve(W.build(orc.SparseSystem, n, eqs), nthreads=NT)
    assert st == 0
    return n, eqs, ref


@pytest.mark.parametrize("precision", PRECISIONS)
def test_batched_paths_all(cfg2_ref, precision):
    n, eqs, ref = cfg2_ref
    assert ref.npaths == 1024
    got, st = P.solve(W.build(P.SparseSystem, n, eqs),
                      gpu=P.default_gpu_options(precision=precision))
    assert st == 0
    assert_parity(n, ref, got)


@pytest.fixture(scope="module")
def cyclic6_ref(orc):
    n, eqs = W.cyclic(6)
    ref, st = orc.solve(W.build(orc.SparseSystem, n, eqs), nthreads=NT)
    assert st == 0
    assert ref.npaths == 720 and ref.nsolutions == 156  # test/cyclic.f90:26
    return n, eqs, ref


@pytest.mark.parametrize("precision", PRECISIONS)
def test_cyclic6(cyclic6_ref, precision):
    n, eqs, ref = cyclic6_ref
    got, st = P.solve(W.build(P.SparseSystem, n, eqs),
                      gpu=P.default_gpu_options(precision=precision))
    assert st == 0
    assert_parity(n, ref, got)
    assert got.nsolutions == 156 and got.ninfinite == 720 - 156
    assert int(got.paths["winding_number"].max()) > 1


def cfg5_windows(npaths):
    step = npaths // CFG5_WINDOWS
    return [1 + w * step + (step - CFG5_WINDOW) * w // (CFG5_WINDOWS - 1)
            for w in range(CFG5_WINDOWS)]


@pytest.fixture(scope="module")
def cfg5_ref(orc):
    n, eqs = W.cfg5()
    so = W.build(orc.SparseSystem, n, eqs)
    npaths = int(orc.lib().orc_bezout(so.h))
    assert npaths == 65536
    wins = []
    for k0 in cfg5_windows(npaths):
        pr, zr, xr, st = orc.solve_paths(so, k0=k0, count=CFG5_WINDOW, nthreads=NT)
        assert st == 0
        wins.append((k0, pr, xr))
    return n, eqs, wins


def test_cfg5_windows_cover_the_range():
    ks = cfg5_windows(65536)
    assert ks[0] == 1 and ks[-1] + CFG5_WINDOW - 1 == 65536
    assert all(b >= a + CFG5_WINDOW for a, b in zip(ks, ks[1:]))


@pytest.mark.parametrize("precision", PRECISIONS)
def test_large_system_windows(cfg5_ref, precision):
    n, eqs, wins = cfg5_ref
    sp = W.build(P.SparseSystem, n, eqs)
    g = P.default_gpu_options(precision=precision)
    for k0, pr, xr in wins:
        pg, zg, xg, st = P.solve_paths(sp, gpu=g, k0=k0, count=CFG5_WINDOW)
        assert st == 0
        for key in PATH_KEYS:
            bad = np.nonzero(pg[key] != pr[key])[0]
            assert bad.size == 0, (k0, key, (bad + k0)[:10])
        ok = endgame_status_agrees(pr, pg)
        assert ok.all(), (k0, "endgame_status", (np.nonzero(~ok)[0] + k0)[:10])
        assert_steps_comparable(pr, pg)
        fin = (pr["status"] == 0) & (pr["at_infinity"] == 0) & (pr["singular"] == 0)
        assert fin.any()
        d = np.max(np.abs(xg[fin] - xr[fin]), axis=1) / np.maximum(
            1.0, np.max(np.abs(xr[fin]), axis=1))
        assert d.max() <= TOL_REGULAR, (k0, d.max())


def test_stream_indices_cover_every_size():
    idx = stream_indices()
    assert len(idx) == 7 * STREAM_PER_SIZE
    assert {W.stream_system(i)[0] for i in idx} == set(range(2, 9))
