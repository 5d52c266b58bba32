"""CPU tests of the C ABI boundary: the library loads, exports every entry
point include/polyhomocont_b200.h declares, and its host logic (sparse
builder, homotopy set-up, option validation) agrees with the restatement of
the reference. No kernel is launched here."""
import ctypes
import os
import re

import numpy as np
import pytest

import polyhomocont_b200 as P
from polyhomocont_b200 import _abi
from polyhomocont_b200 import workloads as W

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def header_functions():
    names = set()
    for fn in os.listdir(os.path.join(ROOT, "include")):
        if fn.endswith(".h"):
            text = open(os.path.join(ROOT, "include", fn)).read()
            text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
            names |= set(re.findall(r"\b(phc_[a-z0-9_]+)\s*\(", text))
    return sorted(names)


@pytest.fixture(scope="module")
def lib():
    from polyhomocont_b200 import build
    build.build()
    return _abi.lib()


def test_exports_every_declared_symbol(lib):
    raw = ctypes.CDLL(_abi.LIB_PATH)
    names = header_functions()
    assert len(names) >= 30
    missing = [n for n in names if not hasattr(raw, n)]
    assert not missing, missing
    bound = {s[0] for s in _abi.SIGNATURES}
    assert set(names) <= bound, set(names) - bound


def test_sparse_builder_validation(lib):
    s = P.SparseSystem(2)  # test/sparse.f90:271-297
    assert s.add_equation([1, 2], np.array([[1], [0], [0]])) == P.ERR_INVALID_INPUT
    assert s.add_equation([1, 2], np.array([[1], [0]])) == P.ERR_INVALID_INPUT
    assert s.add_equation([1], np.array([[1], [-1]])) == P.ERR_INVALID_INPUT
    assert s.add_equation([3, 0], np.array([[0, 1], [0, 1]])) == P.ERR_INVALID_INPUT
    assert s.nequations() == 0
    assert s.add_equation([1], np.array([[1], [0]])) == 0
    t, st = s.table()
    assert st == P.ERR_INVALID_INPUT  # fewer equations than variables
    assert s.add_equation([1], np.array([[0], [1]])) == 0
    assert s.add_equation([1], np.array([[1], [1]])) == P.ERR_INVALID_INPUT
    t, st = s.table()
    assert st == 0 and s.bezout() == 1


@pytest.mark.parametrize("name", ["cfg1", "cfg2", "cfg3", "katsura4", "cyclic5"])
def test_tables_and_homotopy_match_oracle(lib, orc, name):
    gen = {"cfg1": W.dense_quadratic, "cfg2": W.cfg2,
           "cfg3": lambda: W.singular_cubic()[:2], "katsura4": lambda: W.katsura(4),
           "cyclic5": lambda: W.cyclic(5)}[name]
    n, eqs = gen()
    sp = W.build(P.SparseSystem, n, eqs)
    so = W.build(orc.SparseSystem, n, eqs)
    assert list(sp.degrees()) == list(so.degrees())
    t, st = sp.table()
    assert st == 0
    T = sp.total_terms()
    assert T == so.total_terms()
    first, hexps, coefs = so.table()
    assert np.array_equal(np.ctypeslib.as_array(t.first, shape=(n + 1,)), first)
    assert np.array_equal(np.ctypeslib.as_array(t.hexps, shape=(T * (n + 1),)).reshape(T, n + 1),
                          hexps)
    assert np.array_equal(np.ctypeslib.as_array(t.coefs, shape=(2 * T,)).view(complex), coefs)
    for seed in (1, 2, 12345):
        g, b, a, ns, st = P.homotopy_init(sp, seed)
        h = orc.Homotopy()
        assert h.init(so, orc.Rng(seed)) == 0
        g2, b2, a2 = h.constants()
        assert st == 0 and ns == h.nstart
        assert g == g2 and np.array_equal(b, b2) and np.array_equal(a, a2)   # bit-exact


def test_option_validation_without_device(lib):
    n, eqs = W.katsura(3)
    s = W.build(P.SparseSystem, n, eqs)
    o = P.default_options()
    o.endgame.radius_factor = 1.5  # would never reach radius_min
    res, st = P.solve(s, o)
    assert st == P.ERR_INVALID_INPUT
    o = P.default_options()
    o.endgame.nsamples = 0
    res, st = P.solve(s, o)
    assert st == P.ERR_INVALID_INPUT


def test_defaults_mirror_reference(lib):
    o = P.default_options()
    t, e = o.tracker, o.endgame
    assert (t.step_init, t.step_max, t.step_min, t.corrector_tol) == (0.05, 0.1, 1e-14, 1e-10)
    assert (t.corrector_maxit, t.contraction, t.grow_after, t.max_steps) == (3, 0.5, 5, 20000)
    assert (e.t_start, e.nsamples, e.radius_factor, e.radius_min) == (0.1, 8, 0.25, 1e-13)
    assert (e.max_winding, e.loop_radius, e.winding_agreement) == (16, 1e-5, 0.2)
    assert (e.tol, e.residual_tol, e.closure_factor) == (1e-11, 1e-8, 0.1)
    assert (o.use_endgame, o.seed, o.refine_maxit) == (1, 1, 5)
    assert (o.infinity_tol, o.singular_cond, o.real_tol) == (1e-8, 1e10, 1e-8)
    assert (o.dedup_tol, o.singular_dedup_tol) == (1e-8, 1e-6)


def test_no_cpu_fallback(lib):
    """Without a usable CUDA device the solver raises; it never computes the
    paths on the host."""
    import torch
    if torch.cuda.is_available():
        pytest.skip("a GPU is present")
    n, eqs = W.katsura(3)
    s = W.build(P.SparseSystem, n, eqs)
    with pytest.raises(P.PhcError) as ei:
        P.solve(s)
    assert ei.value.code == _abi.PHC_ERR_NO_DEVICE


def test_host_bookkeeping_matches_reference_rules():
    """result_from_arrays follows add_solution/add_singular/find: first match
    within the relative tolerance, in path order."""
    n = 1
    paths = np.zeros(5, dtype=P.PATH_DTYPE)
    paths["singular"] = [0, 0, 1, 1, 0]
    paths["at_infinity"] = [0, 0, 0, 0, 1]
    x = np.array([[1.0], [1.0 + 5e-9], [2.0], [2.0 + 5e-7], [0.0]], dtype=complex)
    res = P.result_from_arrays(n, paths, x)
    assert res.nsolutions == 1 and res.nduplicates == 1
    assert res.nsingular == 1 and list(res.multiplicities) == [2]
    assert res.ninfinite == 1
    assert list(res.paths["solution_index"]) == [1, 1, 0, 0, 0]
    assert list(res.paths["singular_index"]) == [0, 0, 1, 1, 0]
    assert res.nreal == 1
