"""Pins the CPU restatement (oracle/) against the reference's unit tests:
test/random.f90, test/linalg.f90, test/sparse.f90, test/homotopy.f90.
Tolerances are the reference's."""
import numpy as np
import pytest

from tests.helpers import jacobian_fd_error, norm_inf


# ---- test/random.f90 -------------------------------------------------
def test_random_moments(orc):
    g = orc.Rng(42)
    u = np.array([g.uniform() for _ in range(200000)])
    assert u.min() > 0.0 and u.max() < 1.0                      # :44-45
    assert abs(u.mean() - 0.5) <= 5e-3                           # :46
    assert abs(u.var() - 1.0 / 12.0) <= 5e-3                     # :47-48


def test_random_reproducible(orc):
    a, b = orc.Rng(7), orc.Rng(7)
    assert all(a.uniform() == b.uniform() for _ in range(100))   # :51-57
    a, b = orc.Rng(7), orc.Rng(8)
    assert any(a.uniform() != b.uniform() for _ in range(100))   # :58-65


def test_random_complex(orc):
    g = orc.Rng(1)
    z = np.array([g.unit_complex() for _ in range(200000)])
    assert np.max(np.abs(np.abs(z) - 1.0)) <= 1e-14             # :76
    assert abs(z.mean()) <= 1e-2                                 # :77
    z = np.array([g.normal_complex() for _ in range(200000)])
    assert abs(z.mean()) <= 1e-2                                 # :88
    assert abs(np.mean(np.abs(z) ** 2) - 1.0) <= 1e-2            # :90


def test_host_rng_matches_oracle(orc):
    """The product's host generator (input synthesis) draws the same
    sequence as the restatement of src/random.f90."""
    from polyhomocont_b200.rng import Rng
    for seed in (1, 5, 2026, 20261403, -17):
        a, b = Rng(seed), orc.Rng(seed)
        for _ in range(50):
            assert a.uniform() == b.uniform()
        assert a.unit_complex() == b.unit_complex()
        assert a.normal_complex() == b.normal_complex()


# ---- test/linalg.f90 -------------------------------------------------
def test_linalg_random_solves(orc):
    g = orc.Rng(2026)
    for n in range(1, 21, 3):                                    # :41-43
        a = np.zeros((n, n), dtype=complex)
        xref = np.zeros(n, dtype=complex)
        for j in range(n):
            for i in range(n):
                a[i, j] = g.normal_complex()
            xref[j] = g.normal_complex()
        x, st = orc.solve_linear(a, a @ xref)
        assert st == 0
        assert norm_inf(x - xref) / norm_inf(xref) <= 1e-11      # :79-80


def test_linalg_pivoting(orc):
    a = np.array([[0, 1 - 1j, 4], [2 + 1j, 0, 1 + 1j], [1, 3, 2j]], dtype=complex)
    lu, ipiv, st = orc.lu_factor(a)                              # :95-101
    assert st == 0
    for xref in ([1, 1j, -2 + 0.5j], [0.5 + 0.5j, 3, -1j]):
        xref = np.array(xref, dtype=complex)
        b = orc.lu_solve(lu, ipiv, a @ xref)
        assert norm_inf(b - xref) <= 1e-14                       # :106-113


def test_linalg_singular(orc):
    a = np.array([[1, 2, 3j], [1, 2, 3j], [1j, 1, 5]], dtype=complex)
    x, st = orc.solve_linear(a, np.ones(3, dtype=complex))
    assert st == orc.ERR_SINGULAR_MATRIX                         # :132
    assert orc.cond1(a) == np.finfo(float).max                   # :133


def test_linalg_cond(orc):
    d = np.diag([1e3, -2j, 0.3 + 0.4j])
    assert abs(orc.cond1(d) - 1e3 / 0.5) <= 1e-13 * 2e3          # :149-150
    eps = 1e-6
    a = np.array([[1, 1], [1, 1 + eps]], dtype=complex)
    ref = (2 + eps) ** 2 / eps
    assert abs(orc.cond1(a) - ref) <= 1e-8 * ref                 # :157-158


# ---- test/sparse.f90 -------------------------------------------------
def small_system(orc):
    s = orc.SparseSystem(2)
    assert s.add_equation([1, 1, -5], [[2, 0, 0], [0, 2, 0]]) == 0
    assert s.add_equation([1, -2, 0, 1], [[1, 0, 5, 1], [2, 1, 5, 0]]) == 0
    return s


def test_sparse_small(orc):
    s = small_system(orc)
    assert s.nvars() == 2 and s.nequations() == 2                # :57-58
    assert s.nterms(2) == 3                                      # zero term dropped
    assert list(s.degrees()) == [2, 3]
    x = np.array([0.3 - 1.2j, 2.1 + 0.4j])
    f, jac = s.evaluate(x)
    fref = [x[0] ** 2 + x[1] ** 2 - 5, x[0] * x[1] ** 2 - 2 * x[1] + x[0]]
    jref = [[2 * x[0], 2 * x[1]], [x[1] ** 2 + 1, 2 * x[0] * x[1] - 2]]
    assert norm_inf(f - fref) <= 1e-14
    assert np.max(np.abs(jac - jref)) <= 1e-14
    for z in (np.array([0.3 - 1.2j, 2.1 + 0.4j, 0.7 + 0.2j]),
              np.array([0.3 - 1.2j, 2.1 + 0.4j, 0.0])):          # :168-171
        f, jh = s.evaluate_homogeneous(z)
        fr = [z[0] ** 2 + z[1] ** 2 - 5 * z[2] ** 2,
              z[0] * z[1] ** 2 - 2 * z[1] * z[2] ** 2 + z[0] * z[2] ** 2]
        jr = [[2 * z[0], 2 * z[1], -10 * z[2]],
              [z[1] ** 2 + z[2] ** 2, 2 * z[0] * z[1] - 2 * z[2] ** 2,
               -4 * z[1] * z[2] + 2 * z[0] * z[2]]]
        assert norm_inf(f - fr) <= 1e-14
        assert np.max(np.abs(jh - jr)) <= 1e-14
    assert jacobian_fd_error(s.evaluate, [0, 1.5 - 0.5j]) <= 1e-8
    f, jac = s.evaluate(np.zeros(2, dtype=complex))
    assert np.max(np.abs(jac - np.array([[0, 0], [1, -2]]))) == 0.0   # exact


def test_sparse_random_fd_and_homogeneity(orc):
    g = orc.Rng(11)
    small_system(orc)  # the reference draws nothing for the small system
    n, nt = 4, 6
    err_j = err_jh = err_h = 0.0
    for _ in range(5):                                           # :236-256
        s = orc.SparseSystem(n)
        for _ in range(n):
            coefs = np.zeros(nt, dtype=complex)
            exps = np.zeros((n, nt), dtype=np.int32)
            for k in range(nt):
                coefs[k] = g.normal_complex()
                for j in range(n):
                    exps[j, k] = int(4.0 * g.uniform())
            assert s.add_equation(coefs, exps) == 0
        x = np.zeros(n, dtype=complex)
        z = np.zeros(n + 1, dtype=complex)
        for j in range(n):
            x[j] = g.normal_complex()
            z[j] = g.normal_complex()
        z[n] = g.normal_complex()
        lam = g.normal_complex()
        err_j = max(err_j, jacobian_fd_error(s.evaluate, x))
        err_jh = max(err_jh, jacobian_fd_error(s.evaluate_homogeneous, z))
        d = s.degrees()
        f, _ = s.evaluate_homogeneous(z)
        fl, _ = s.evaluate_homogeneous(lam * z)
        fa, _ = s.evaluate(z[:n] / z[n])
        e = np.max(np.abs(fl - lam ** d * f)) / max(1.0, np.max(np.abs(fl)))
        e = max(e, np.max(np.abs(f - z[n] ** d * fa)) / max(1.0, np.max(np.abs(f))))
        err_h = max(err_h, e)
    assert err_j <= 1e-7 and err_jh <= 1e-7                      # :257-260
    assert err_h <= 1e-12                                        # :261


def test_sparse_validation(orc):
    s = orc.SparseSystem(2)                                      # :271-297
    assert s.add_equation([1, 2], np.array([[1], [0], [0]])) == orc.ERR_INVALID_INPUT
    assert s.add_equation([1, 2], np.array([[1], [0]])) == orc.ERR_INVALID_INPUT
    assert s.add_equation([1], np.array([[1], [-1]])) == orc.ERR_INVALID_INPUT
    assert s.add_equation([3, 0], np.array([[0, 1], [0, 1]])) == orc.ERR_INVALID_INPUT
    assert s.nequations() == 0
    assert s.add_equation([1], np.array([[1], [0]])) == 0
    assert s.add_equation([1], np.array([[0], [1]])) == 0
    assert s.add_equation([1], np.array([[1], [1]])) == orc.ERR_INVALID_INPUT


# ---- test/homotopy.f90 -----------------------------------------------
def test_homotopy(orc):
    s = orc.SparseSystem(2)
    s.add_equation([1, 1, -5], [[2, 0, 0], [0, 2, 0]])
    s.add_equation([1, -2, 1], [[1, 0, 1], [2, 1, 0]])
    g = orc.Rng(5)
    hom = orc.Homotopy()
    assert hom.init(s, g) == 0
    assert hom.nunknowns() == 3 and hom.nstart == 6              # :336-337
    gamma, b, a = hom.constants()
    assert abs(abs(gamma) - 1.0) <= 1e-15

    def check_start():
        zs = [hom.start_solution(k) for k in range(1, hom.nstart + 1)]
        res = 0.0
        for z in zs:
            h, hz, ht = hom.evaluate(z, 1.0)
            res = max(res, norm_inf(h) / max(1.0, norm_inf(z)) ** 3)
        assert res <= 1e-14                                      # :383-384
        dmin = min(norm_inf(zs[k] - zs[l]) for k in range(len(zs))
                   for l in range(k + 1, len(zs)))
        assert dmin > 1e-3                                       # :392

    check_start()
    assert hom.init(s, g) == 0                                   # re-init
    check_start()
    step = 1e-5
    for t in (0.37, 1.0, 0.0, 0.02 - 0.05j):                     # :346-349
        z = np.array([g.normal_complex() for _ in range(3)])
        h, hz, ht = hom.evaluate(z, t)
        err = 0.0
        for j in range(3):
            zp = z.copy()
            zp[j] = z[j] + step
            hp, _, _ = hom.evaluate(zp, t)
            zp[j] = z[j] - step
            hm, _, _ = hom.evaluate(zp, t)
            err = max(err, norm_inf((hp - hm) / (2 * step) - hz[:, j]))
        assert err / np.max(np.abs(hz)) <= 1e-8                  # :431
        hp, _, _ = hom.evaluate(z, t + step)
        hm, _, _ = hom.evaluate(z, t - step)
        err = norm_inf((hp - hm) / (2 * step) - ht)
        assert err / max(1.0, norm_inf(ht)) <= 1e-8              # :437-438
    inc = orc.SparseSystem(2)
    inc.add_equation([1, -1], [[2, 0], [0, 0]])
    assert hom.init(inc, g) == orc.ERR_INVALID_INPUT             # :351-357
