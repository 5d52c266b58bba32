"""sys%evaluate and sys%evaluate_homogeneous of type(sparse_system)
(src/sparse.f90:197-221) through the library's host entry points, pinned
by the reference's check_small_system (test/sparse.f90:32-110) and against
the restatement on random systems."""
import numpy as np
import pytest

import polyhomocont_b200 as P
from polyhomocont_b200 import workloads as W


def small_system():
    """test/sparse.f90:46-53: F_1 = x1^2 + x2^2 - 5, F_2 = x1 x2^2 - 2 x2 + x1
    with an extra zero term in F_2."""
    s = P.SparseSystem(2)
    assert s.add_equation([1, 1, -5], np.array([[2, 0], [0, 2], [0, 0]]).T) == 0
    assert s.add_equation([1, -2, 0, 1], np.array([[1, 2], [0, 1], [5, 5], [1, 0]]).T) == 0
    return s


def test_check_small_system():
    s = small_system()
    assert s.nvars() == 2 and s.nequations() == 2
    assert s.nterms(2) == 3  # the zero term is dropped
    assert list(s.degrees()) == [2, 3]
    x = np.array([0.3 - 1.2j, 2.1 + 0.4j])
    f, jac = s.evaluate(x)
    fref = np.array([x[0] ** 2 + x[1] ** 2 - 5, x[0] * x[1] ** 2 - 2 * x[1] + x[0]])
    jref = np.array([[2 * x[0], 2 * x[1]], [x[1] ** 2 + 1, 2 * x[0] * x[1] - 2]])
    assert np.max(np.abs(f - fref)) <= 1e-14
    assert np.max(np.abs(jac - jref)) <= 1e-14
    # the homogenized system at a finite point and exactly at infinity
    for w in (0.7 + 0.2j, 0.0):
        z = np.array([0.3 - 1.2j, 2.1 + 0.4j, w])
        fh, jh = s.evaluate_homogeneous(z)
        fhref = np.array([z[0] ** 2 + z[1] ** 2 - 5 * z[2] ** 2,
                          z[0] * z[1] ** 2 - 2 * z[1] * z[2] ** 2 + z[0] * z[2] ** 2])
        jhref = np.array([[2 * z[0], 2 * z[1], -10 * z[2]],
                          [z[1] ** 2 + z[2] ** 2, 2 * z[0] * z[1] - 2 * z[2] ** 2,
                           -4 * z[1] * z[2] + 2 * z[0] * z[2]]])
        assert np.max(np.abs(fh - fhref)) <= 1e-14
        assert np.max(np.abs(jh - jhref)) <= 1e-14
    # points with zero coordinates: finite differences, and the exact Jacobian at 0
    x = np.array([0.0, 1.5 - 0.5j])
    _, jac = s.evaluate(x)
    err = 0.0
    for j in range(2):
        h = 1e-5 * max(1.0, abs(x[j]))
        xp, xm = x.copy(), x.copy()
        xp[j] += h
        xm[j] -= h
        err = max(err, np.max(np.abs((s.evaluate(xp)[0] - s.evaluate(xm)[0]) / (2 * h) - jac[:, j])))
    assert err / max(1.0, np.max(np.abs(jac))) <= 1e-8
    _, jac = s.evaluate(np.zeros(2, dtype=complex))
    assert np.array_equal(jac, np.array([[0, 0], [1, -2]], dtype=complex))


@pytest.mark.parametrize("name", ["katsura4", "cyclic5", "cfg3"])
def test_matches_the_restatement(orc, name):
    n, eqs = {"katsura4": lambda: W.katsura(4), "cyclic5": lambda: W.cyclic(5),
              "cfg3": lambda: W.singular_cubic()[:2]}[name]()
    s = W.build(P.SparseSystem, n, eqs)
    so = W.build(orc.SparseSystem, n, eqs)
    g = np.random.default_rng(5)
    for _ in range(5):
        x = g.normal(size=n) + 1j * g.normal(size=n)
        z = np.append(x, g.normal() + 1j * g.normal())
        for got, ref in ((s.evaluate(x), so.evaluate(x)),
                         (s.evaluate_homogeneous(z), so.evaluate_homogeneous(z))):
            scale = max(1.0, np.max(np.abs(ref[1])))
            assert np.max(np.abs(got[0] - ref[0])) <= 1e-13 * scale
            assert np.max(np.abs(got[1] - ref[1])) <= 1e-13 * scale


def test_a_sparse_system_samples_to_itself():
    """A SparseSystem is a PolySystem too (nvars, degrees, evaluate): sampling
    it reproduces its own table."""
    n, eqs = W.katsura(3)
    s = W.build(P.SparseSystem, n, eqs)
    t, st, err = P.sample_system(s)
    assert st == 0 and err <= 1e-13
    assert t.total_terms() <= s.total_terms()
    assert list(t.degrees()) == list(s.degrees())
