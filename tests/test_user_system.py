"""User-evaluator systems (class(poly_system), src/system.f90:27-67) on CPU:
the sampler that turns them into sparse tables (phc_sparse_sample, host
code of the library) and the restatement's default homogenization
(src/system.f90:71-119), pinned by the reference's own check_user_system
(test/solve.f90:320-365)."""
import numpy as np
import pytest

import polyhomocont_b200 as P
from polyhomocont_b200 import _abi
from polyhomocont_b200 import workloads as W
from tests.helpers import CircleCubic, ClosedForm, TermEvaluator, set_distance


def table_dict(s):
    """{homogenized exponents: coefficient} per equation of a SparseSystem"""
    t, st = s.table()
    assert st == 0
    n, T = s.nvars(), s.total_terms()
    first = np.ctypeslib.as_array(t.first, shape=(n + 1,))
    hexps = np.ctypeslib.as_array(t.hexps, shape=((n + 1) * T,)).reshape(T, n + 1)
    coefs = np.ctypeslib.as_array(t.coefs, shape=(2 * T,)).view(np.complex128)
    out = []
    for i in range(n):
        d = {}
        for k in range(first[i], first[i + 1]):  # a table may repeat a monomial: sum
            d[tuple(hexps[k])] = d.get(tuple(hexps[k]), 0) + coefs[k]
        out.append({k: v for k, v in d.items() if v != 0})
    return out


def assert_same_table(got, ref, rtol):
    assert len(got) == len(ref)
    for g, r in zip(got, ref):
        assert set(g) == set(r)
        scale = max(abs(v) for v in r.values())
        for k in r:
            assert abs(g[k] - r[k]) <= rtol * scale, (k, g[k], r[k])


def test_closed_form_table():
    s, st, err = P.sample_system(ClosedForm())
    assert st == 0 and err <= 1e-13
    ref = P.SparseSystem(2)
    ref.add_equation([1, 1, -5], [[2, 0, 0], [0, 2, 0]])
    ref.add_equation([1, -2, 1], [[1, 0, 1], [2, 1, 0]])
    assert list(s.degrees()) == [2, 3]
    assert_same_table(table_dict(s), table_dict(ref), 1e-14)


@pytest.mark.parametrize("name", ["katsura4", "cyclic5", "cfg1", "cfg2", "cfg3", "stream"])
def test_tables_of_known_systems(name):
    """The sampled table has exactly the terms of the system the evaluator
    computes, with the same coefficients to rounding."""
    n, eqs = {"katsura4": lambda: W.katsura(4), "cyclic5": lambda: W.cyclic(5),
              "cfg1": W.dense_quadratic, "cfg2": W.cfg2, "cfg3": lambda: W.singular_cubic()[:2],
              "stream": lambda: W.stream_system(W.seed_for(4, 7))}[name]()
    s, st, err = P.sample_system(TermEvaluator(n, eqs))
    assert st == 0, st
    assert err <= 1e-12
    assert_same_table(table_dict(s), table_dict(W.build(P.SparseSystem, n, eqs)), 1e-12)


def test_user_systems_reject_what_the_reference_forbids():
    class Lower(ClosedForm):  # F_2 has degree 3, not 2
        def degrees(self):
            return [2, 2]

    class Higher(ClosedForm):  # degree 4 stated, top part zero: not exact
        def degrees(self):
            return [2, 4]

    class BadJacobian(ClosedForm):
        def evaluate(self, x):
            f, jac = super().evaluate(x)
            jac[0, 0] += 1e-3
            return f, jac

    class NotPolynomial(ClosedForm):
        def evaluate(self, x):
            f, jac = super().evaluate(x)
            f[0] = np.exp(x[0])
            return f, jac

    class WrongCount(ClosedForm):
        def degrees(self):
            return [2]

    for bad in (Lower(), Higher(), BadJacobian(), NotPolynomial(), WrongCount()):
        s, st, err = P.sample_system(bad)
        assert st == P.ERR_INVALID_INPUT, type(bad).__name__
        t, tst = s.table()
        assert tst != 0  # nothing half-built is left in the builder


def test_evaluator_exception_is_raised_again():
    class Raises(ClosedForm):
        def evaluate(self, x):
            raise ValueError("user evaluator failed")

    with pytest.raises(ValueError, match="user evaluator failed"):
        P.sample_system(Raises())


def test_too_many_monomials_is_unsupported():
    class Big:
        def nvars(self):
            return 30

        def degrees(self):
            return [3] * 30

        def evaluate(self, x):
            raise AssertionError("not sampled")

    s, st, err = P.sample_system(Big())
    assert st == _abi.PHC_ERR_UNSUPPORTED


def test_sampling_is_reproducible():
    a, st1, _ = P.sample_system(TermEvaluator(*W.katsura(4)), seed=3)
    b, st2, _ = P.sample_system(TermEvaluator(*W.katsura(4)), seed=3)
    assert st1 == st2 == 0
    ta, tb = table_dict(a), table_dict(b)
    assert all(x == y for x, y in zip(ta, tb))


def test_check_user_system_on_the_restatement(orc):
    """check_user_system (test/solve.f90:320-365) on the restatement: the
    user system through the default homogenization and its sparse form give
    the same solutions, which solve the system."""
    ru, st = orc.solve(orc.UserSystem(ClosedForm()))
    assert st == 0
    s = orc.SparseSystem(2)
    s.add_equation([1, 1, -5], [[2, 0, 0], [0, 2, 0]])
    s.add_equation([1, -2, 1], [[1, 0, 1], [2, 1, 0]])
    rs, st = orc.solve(s)
    assert st == 0
    assert ru.nsolutions > 0 and ru.nsolutions == rs.nsolutions
    assert set_distance(ru.solutions, rs.solutions) <= 1e-11
    resid = max(np.max(np.abs(ClosedForm().evaluate(x)[0])) / max(1.0, np.max(np.abs(x))) ** 3
                for x in ru.solutions)
    assert resid <= 1e-13
    assert ru.nduplicates == 0


def _by_hand(z):
    """homogenized_by_hand, test/system.f90:65-80"""
    w = z[2]
    f = np.array([z[0] ** 2 + z[1] ** 2 - 5 * w ** 2,
                  z[0] * z[1] ** 2 - 2 * z[1] * w ** 2 + z[0] * w ** 2])
    jac = np.array([[2 * z[0], 2 * z[1], -10 * w],
                    [z[1] ** 2 + w ** 2, 2 * z[0] * z[1] - 2 * w ** 2,
                     -4 * z[1] * w + 2 * z[0] * w]])
    return f, jac


def test_default_homogenization_matches_by_hand(orc):
    """test/system.f90:104-138 on the restatement's default homogenization:
    against the system homogenized by hand, by finite differences and by
    homogeneity at a generic point, and against the hand-written system
    close to infinity (w = 1e-6 - 2e-6 i, where dF^h/dw loses about
    eps/|w| to cancellation), with the reference's tolerances."""
    u = orc.UserSystem(ClosedForm())
    z = np.array([0.3 - 1.2j, 2.1 + 0.4j, 0.7 + 0.2j])
    f, jac = u.evaluate_homogeneous(z)
    fr, jr = _by_hand(z)
    assert np.max(np.abs(f - fr)) <= 1e-13
    assert np.max(np.abs(jac - jr)) <= 1e-13
    # homogeneous_jacobian_fd_error, test/testing.f90:158-188
    err = 0.0
    for j in range(3):
        h = 1e-5 * max(1.0, abs(z[j]))
        zp, zm = z.copy(), z.copy()
        zp[j] += h
        zm[j] -= h
        err = max(err, np.max(np.abs((u.evaluate_homogeneous(zp)[0] -
                                      u.evaluate_homogeneous(zm)[0]) / (2 * h) - jac[:, j])))
    assert err / max(1.0, np.max(np.abs(jac))) <= 1e-8
    # homogeneity_error, test/testing.f90:190-215, lambda = 0.6 - 1.3 i
    lam, d = 0.6 - 1.3j, np.array([2, 3])
    fl, _ = u.evaluate_homogeneous(lam * z)
    fa, _ = ClosedForm().evaluate(z[:2] / z[2])
    herr = max(np.max(np.abs(fl - lam ** d * f)) / max(1.0, np.max(np.abs(fl))),
               np.max(np.abs(f - z[2] ** d * fa)) / max(1.0, np.max(np.abs(f))))
    assert herr <= 1e-13
    z[2] = 1e-6 - 2e-6j
    f, jac = u.evaluate_homogeneous(z)
    fr, jr = _by_hand(z)
    assert np.max(np.abs(f - fr)) / np.max(np.abs(fr)) <= 1e-9
    assert np.max(np.abs(jac - jr)) / np.max(np.abs(jr)) <= 1e-8


def test_circle_cubic_example_on_the_restatement(orc):
    """app/example.f90: six finite solutions, each with a tiny residual."""
    r, st = orc.solve(orc.UserSystem(CircleCubic()))
    assert st == 0 and r.npaths == 6 and r.nsolutions == 6 and r.nfailed == 0
    for x in r.solutions:
        assert np.max(np.abs(CircleCubic().evaluate(x)[0])) <= 1e-12 * max(1, np.max(np.abs(x))) ** 3
