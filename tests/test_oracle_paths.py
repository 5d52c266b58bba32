"""Pins the CPU restatement (oracle/) against the reference's path-level
tests: test/tracker.f90, test/endgame.f90, test/solve.f90,
test/katsura.f90 (golden vectors from reference/ref_katsura.py, see
tests/golden/make_katsura.py) and test/cyclic.f90."""
import json
import os

import numpy as np
import pytest

from polyhomocont_b200 import workloads as W
from tests.helpers import norm_inf, set_distance

GOLDEN = os.path.join(os.path.dirname(__file__), "golden")


def sparse(orc, n, eqs):
    return W.build(orc.SparseSystem, n, eqs)


# ---- test/tracker.f90 ------------------------------------------------
def test_tracker(orc):
    g = orc.Rng(3)
    # cubic x^3 - 2x + 1, :38-74
    s = orc.SparseSystem(1)
    s.add_equation([1, -2, 1], [[3, 1, 0]])
    hom = orc.Homotopy()
    assert hom.init(s, g) == 0
    roots = np.array([1.0, (-1 + 5 ** 0.5) / 2, (-1 - 5 ** 0.5) / 2])
    found, err = set(), 0.0
    for k in range(1, hom.nstart + 1):
        z, info = orc.track_path(hom, hom.start_solution(k), 1.0, 0.0)
        assert info.status == orc.PATH_SUCCESS
        r = int(np.argmin(np.abs(z[0] / z[1] - roots)))
        found.add(r)
        err = max(err, abs(z[0] / z[1] - roots[r]))
    assert found == {0, 1, 2} and err <= 1e-10
    # 2x2 x^2 + y^2 = 5, xy = 2, :76-131
    s = orc.SparseSystem(2)
    s.add_equation([1, 1, -5], [[2, 0, 0], [0, 2, 0]])
    s.add_equation([1, -2], [[1, 0], [1, 0]])
    hom = orc.Homotopy()
    assert hom.init(s, g) == 0
    sols = np.array([[1, 2], [2, 1], [-1, -2], [-2, -1]], dtype=float)
    found, err, err_split = set(), 0.0, 0.0
    for k in range(1, hom.nstart + 1):
        z0 = hom.start_solution(k)
        z, info = orc.track_path(hom, z0, 1.0, 0.0)
        assert info.status == orc.PATH_SUCCESS
        d = [norm_inf(z[:2] / z[2] - sr) for sr in sols]
        r = int(np.argmin(d))
        found.add(r)
        err = max(err, d[r])
        z2, _ = orc.track_path(hom, z0, 1.0, 0.5)
        z2, _ = orc.track_path(hom, z2, 0.5, 0.0)
        err_split = max(err_split, norm_inf(z2 - z) / norm_inf(z))
    assert found == {0, 1, 2, 3}
    assert err <= 1e-10 and err_split <= 1e-9
    assert info.naccepted > 0
    # max steps, :133-158
    s = orc.SparseSystem(1)
    s.add_equation([1, -2], [[2, 0]])
    hom = orc.Homotopy()
    hom.init(s, g)
    o = orc.default_tracker_options()
    o.step_max = o.step_init = 1e-3
    o.max_steps = 10
    z, info = orc.track_path(hom, hom.start_solution(1), 1.0, 0.0, o)
    assert info.status == orc.PATH_FAILED_MAX_STEPS
    assert 0.0 < info.t.real < 1.0
    # loops around t = 0 for (x - 1)^2 (x + 1), :160-216
    s = orc.SparseSystem(1)
    s.add_equation([1, -1, -1, 1], [[3, 2, 1, 0]])
    hom = orc.Homotopy()
    hom.init(s, g)
    o = orc.default_tracker_options()
    o.step_init = o.step_max = 1.0 / 8.0
    r, twopi = 1e-3, 8.0 * np.arctan(1.0)
    nsimple = ndouble = 0
    for k in range(1, hom.nstart + 1):
        z0, info = orc.track_path(hom, hom.start_solution(k), 1.0, r)
        assert info.status == orc.PATH_SUCCESS
        z1, info = orc.track_arc(hom, z0, r, 0.0, twopi, o)
        assert info.status == orc.PATH_SUCCESS
        if abs(z0[0] / z0[1] + 1.0) < 0.1:
            nsimple += 1
            assert norm_inf(z1 - z0) / norm_inf(z0) <= 1e-9
        else:
            ndouble += 1
            assert norm_inf(z1 - z0) / norm_inf(z0) > 1e-3
            z2, info = orc.track_arc(hom, z1, r, 0.0, twopi, o)
            assert norm_inf(z2 - z0) / norm_inf(z0) <= 1e-9
    assert nsimple == 1 and ndouble == 2


# ---- test/endgame.f90 ------------------------------------------------
def _run_endgame_paths(orc, s, g):
    hom = orc.Homotopy()
    hom.init(s, g)
    eo = orc.default_endgame_options()
    zs, egs = [], []
    for k in range(1, hom.nstart + 1):
        z, info = orc.track_path(hom, hom.start_solution(k), 1.0, eo.t_start)
        assert info.status == orc.PATH_SUCCESS
        _, zr, r = orc.cauchy_endgame(hom, z, eo)
        zs.append(zr)
        egs.append(r)
    return zs, egs


def test_endgame(orc):
    g = orc.Rng(17)
    for coefs, root, mult, other in (([1, -1, -1, 1], 1.0, 2, -1.0),
                                     ([1, -1, -3, 5, -2], 1.0, 3, -2.0)):
        deg = len(coefs) - 1
        s = orc.SparseSystem(1)
        s.add_equation(coefs, [[deg - k for k in range(deg + 1)]])
        zs, egs = _run_endgame_paths(orc, s, g)
        nmult, err_mult, err_other = 0, 0.0, 0.0
        for z, r in zip(zs, egs):
            assert r.status == orc.ENDGAME_CONVERGED             # :321
            x = z[0] / z[1]
            if abs(x - root) < 0.1:
                nmult += 1
                err_mult = max(err_mult, abs(x - root))
                assert r.winding_number == mult
            else:
                err_other = max(err_other, abs(x - other))
                assert r.winding_number == 1
        assert nmult == mult                                     # :331
        assert err_mult <= 1e-9 and err_other <= 1e-12           # :334-337
    # endpoints at infinity: x y = 1, x^2 = 4, :341-374
    s = orc.SparseSystem(2)
    s.add_equation([1, -1], [[1, 0], [1, 0]])
    s.add_equation([1, -4], [[2, 0], [0, 0]])
    zs, egs = _run_endgame_paths(orc, s, g)
    ninf, wmax = 0, 0.0
    for z in zs:
        if abs(z[2]) < 1e-3 * np.max(np.abs(z)):
            ninf += 1
            wmax = max(wmax, abs(z[2]) / np.max(np.abs(z)), abs(z[0]) / np.max(np.abs(z)))
    assert ninf == 2 and wmax <= 1e-9


# ---- test/solve.f90 --------------------------------------------------
def univariate_system(orc):
    roots = np.array([1, -2, 3j, -3j, 0.5])
    c = np.zeros(6, dtype=complex)
    c[0] = 1
    for k in range(1, 6):
        c[1:k + 1] = c[0:k] - roots[k - 1] * c[1:k + 1]
        c[0] = -roots[k - 1] * c[0]
    s = orc.SparseSystem(1)
    s.add_equation(c, [[0, 1, 2, 3, 4, 5]])
    return s, roots


def test_solve_cases(orc):
    s, roots = univariate_system(orc)                            # :98-130
    res, st = orc.solve(s)
    assert st == 0 and res.npaths == 5 and res.nsolutions == 5 and res.nreal == 3
    assert res.nfailed == 0 and res.nduplicates == 0
    assert set_distance(res.solutions, roots.reshape(5, 1)) <= 1e-12
    # 2x2 for seeds 1..10, :132-173
    s = orc.SparseSystem(2)
    s.add_equation([1, 1, -5], [[2, 0, 0], [0, 2, 0]])
    s.add_equation([1, -2], [[1, 0], [1, 0]])
    sols = np.array([[1, 2], [2, 1], [-1, -2], [-2, -1]], dtype=complex)
    o = orc.default_options()
    for seed in range(1, 11):
        o.seed = seed
        res, st = orc.solve(s, o)
        assert res.nsolutions == 4 and res.nreal == 4
        assert set_distance(res.solutions, sols) <= 1e-12
    assert np.max(np.abs(res.solutions.imag)) <= 1e-12
    # infinity, :175-202
    s = orc.SparseSystem(2)
    s.add_equation([1, -1], [[1, 0], [1, 0]])
    s.add_equation([1, -4], [[2, 0], [0, 0]])
    res, st = orc.solve(s)
    assert st == 0 and res.npaths == 4 and res.nsolutions == 2
    assert set_distance(res.solutions, [[2, 0.5], [-2, -0.5]]) <= 1e-12
    assert res.ninfinite == 2 and res.nfailed == 0 and res.nsingular == 0
    # double root, :204-228
    s = orc.SparseSystem(1)
    s.add_equation([1, -1, -1, 1], [[3, 2, 1, 0]])
    res, st = orc.solve(s)
    assert res.nsolutions == 1 and abs(res.solutions[0, 0] + 1) <= 1e-12
    assert res.nsingular == 1 and res.multiplicities[0] == 2
    assert abs(res.singular_solutions[0, 0] - 1) <= 1e-10 and res.nfailed == 0
    # mixed, :230-273
    s = orc.SparseSystem(2)
    s.add_equation([1, -1], [[1, 0], [1, 0]])
    s.add_equation([1, -3, 2], [[3, 1, 0], [0, 0, 0]])
    res, st = orc.solve(s)
    assert res.npaths == 6 and res.nsolutions == 1
    assert np.max(np.abs(res.solutions[0] - [-2, -0.5])) <= 1e-12
    assert res.nsingular == 1 and res.multiplicities[0] == 2
    assert np.max(np.abs(res.singular_solutions[0] - 1)) <= 1e-10
    assert res.ninfinite == 3 and res.nfailed == 0
    assert np.all(res.paths["endgame_status"] == orc.ENDGAME_CONVERGED)
    for p in res.paths:
        if p["solution_index"] > 0:
            assert p["winding_number"] == 1
        elif p["singular_index"] > 0:
            assert p["winding_number"] == 2
    # multiplicity 4, :275-299
    s = orc.SparseSystem(2)
    s.add_equation([1], [[2], [0]])
    s.add_equation([1, 1], [[0, 1], [2, 1]])
    res, st = orc.solve(s)
    assert res.nsolutions == 0 and res.nsingular == 1 and res.multiplicities[0] == 4
    assert np.max(np.abs(res.singular_solutions[0])) <= 1e-8 and res.nfailed == 0
    # without end game, :301-319
    s = orc.SparseSystem(2)
    s.add_equation([1, 1, -5], [[2, 0, 0], [0, 2, 0]])
    s.add_equation([1, -2], [[1, 0], [1, 0]])
    o = orc.default_options()
    o.use_endgame = 0
    res, st = orc.solve(s, o)
    assert st == 0 and res.nsolutions == 4
    # invalid, :364-377
    s = orc.SparseSystem(2)
    s.add_equation([1, -1], [[2, 0], [0, 0]])
    res, st = orc.solve(s)
    assert st == orc.ERR_INVALID_INPUT


# ---- test/katsura.f90 ------------------------------------------------
@pytest.mark.parametrize("n", [3, 4])
def test_katsura_golden(orc, n):
    gold = json.load(open(os.path.join(GOLDEN, "katsura.json")))[f"katsura{n}"]
    ref = np.array([[complex(a, b) for a, b in s] for s in gold["solutions"]])
    s = sparse(orc, *W.katsura(n))
    res, st = orc.solve(s)
    assert st == 0
    assert res.npaths == 2 ** n and res.nsolutions == 2 ** n     # :220-221
    assert res.nreal == gold["nreal"]                            # :222
    assert res.nfailed == 0 and res.nduplicates == 0
    assert set_distance(res.solutions, ref) <= 1e-12             # :225-226
    assert np.max(res.paths["residual"]) <= 1e-14               # :227-228


# ---- test/cyclic.f90 -------------------------------------------------
@pytest.mark.parametrize("n,nsols", [(5, 70), (6, 156)])
def test_cyclic(orc, n, nsols):
    s = sparse(orc, *W.cyclic(n))
    res, st = orc.solve(s, nthreads=4)
    assert st == 0
    assert res.nsolutions == nsols and res.nsingular == 0        # :307-308
    assert res.ninfinite == res.npaths - nsols                   # :309-310
    assert res.nfailed == 0 and res.nduplicates == 0
    mask = res.paths["solution_index"] > 0
    assert np.max(res.paths["residual"][mask]) <= 1e-13          # :313-316
    sols = res.solutions
    assert set_distance(sols, np.roll(sols, -1, axis=1)) <= 1e-10
    omega = np.exp(2j * np.pi / n)
    assert set_distance(sols, omega * sols) <= 1e-10


# ---- benchmark configurations: properties known exactly ---------------
def test_singular_config_root(orc):
    """cfg3: the 16 paths to the exact root r are singular with winding
    numbers > 1 and cluster into one singular solution of multiplicity
    16 close to r."""
    n, eqs, r = W.singular_cubic()
    s = sparse(orc, n, eqs)
    res, st = orc.solve(s, nthreads=4)
    assert st == 0 and res.npaths == 81 and res.nfailed == 0
    assert res.nsingular == 1 and res.multiplicities[0] == 16
    assert norm_inf(res.singular_solutions[0] - r) / max(1.0, norm_inf(r)) <= 1e-6
    sing = res.paths["singular_index"] > 0
    assert np.all(res.paths["winding_number"][sing] > 1)
