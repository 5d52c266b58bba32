"""The library's host bookkeeping (phc_finish_solve: add_solution,
add_singular, find, collect_real; src/solve.f90:330-426) against a direct
restatement of the reference's rules, on endpoints placed at the decision
boundaries: duplicates at tol * max(1, ||x||_inf) * (1 + k eps), norms
around 1 (where max(1, .) bends), magnitudes from 1e-150 to 1e150, and
imaginary parts at the real-solution threshold. The library decides with
hashed buckets and squared moduli and falls back to hypot near a
threshold; every decision must be the reference's, bit for bit."""
import numpy as np
import pytest

import polyhomocont_b200 as P
from tests.helpers import reference_bookkeeping


def boundary_case(g, o):
    n = int(g.integers(1, 7))
    npaths = int(g.integers(1, 80))
    mode = int(g.integers(0, 4))
    if mode == 0:
        scale = 10.0 ** int(g.integers(-150, 151))
    elif mode == 1:
        scale = 1.0 + 1e-16 * int(g.integers(-8, 9))
    else:
        scale = 10.0 ** float(g.uniform(-3, 3))
    base = []
    for _ in range(int(g.integers(1, 5))):
        re = scale * g.normal(size=n)
        kind = int(g.integers(0, 3))
        if kind == 0:
            im = np.zeros(n)
        elif kind == 1:  # at the real-solution threshold
            im = o.real_tol * max(1.0, float(np.max(np.abs(re)))) * (1 + 1e-16 * g.integers(-6, 7, size=n))
        else:
            im = scale * g.normal(size=n)
        base.append(re + 1j * im)
    paths = np.zeros(npaths, dtype=P.PATH_DTYPE)
    x = np.zeros((npaths, n), dtype=np.complex128)
    for k in range(npaths):
        paths["status"][k] = 1 if g.integers(0, 12) == 0 else 0
        paths["at_infinity"][k] = 1 if g.integers(0, 10) == 0 else 0
        paths["singular"][k] = 1 if g.integers(0, 5) == 0 else 0
        b = base[int(g.integers(0, len(base)))].copy()
        tol = o.singular_dedup_tol if paths["singular"][k] else o.dedup_tol
        if g.integers(0, 4):
            off = tol * max(1.0, float(np.max(np.abs(b)))) * (1 + 1e-16 * int(g.integers(-6, 7)))
            j = int(g.integers(0, n))
            b[j] += off if g.integers(0, 2) else off * np.exp(1j * g.uniform(0, 2 * np.pi))
        x[k] = b
    return n, paths, x


@pytest.mark.parametrize("seed", range(6))
def test_bookkeeping_decisions_at_the_boundaries(seed):
    o = P.default_options()
    g = np.random.default_rng(1000 + seed)
    for _ in range(40):
        n, paths, x = boundary_case(g, o)
        got = P.result_from_arrays(n, paths, x, o)
        ref = reference_bookkeeping(n, paths, x, o)
        assert got.nfailed == ref["nfailed"] and got.ninfinite == ref["ninfinite"]
        assert got.nduplicates == ref["nduplicates"]
        assert np.array_equal(got.paths["solution_index"], ref["solution_index"])
        assert np.array_equal(got.paths["singular_index"], ref["singular_index"])
        assert np.array_equal(got.solutions, ref["solutions"])
        assert np.array_equal(got.singular_solutions, ref["singular_solutions"])
        assert np.array_equal(got.multiplicities, ref["multiplicities"])
        assert np.array_equal(got.real_solutions, ref["real_solutions"])
