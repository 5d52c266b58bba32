"""User-evaluator systems on the GPU: solve() samples a PolySystem into a
sparse table and tracks that. Checked with the reference's own
check_user_system (test/solve.f90:320-365) and per path against the
restatement of the reference's path for user systems, the default
homogenization through the affine evaluator (src/system.f90:71-119).

Both paths track the same homotopy (gamma, b and the patch come from the
degrees and the seed alone); they differ in how F^h is evaluated, so
endpoints agree to the parity tolerance, not bit for bit."""
import numpy as np
import pytest

import polyhomocont_b200 as P
from polyhomocont_b200 import workloads as W
from tests.helpers import CircleCubic, ClosedForm, TermEvaluator, set_distance

pytestmark = pytest.mark.gpu

TOL_REGULAR = 1e-10
TOL_SINGULAR = 1e-6


@pytest.fixture(scope="module", autouse=True)
def need_gpu():
    import torch
    if not torch.cuda.is_available():
        pytest.fail("GPU tests need a CUDA device")


@pytest.mark.parametrize("precision", [P.PHC_PREC_FP64, P.PHC_PREC_MIXED])
def test_check_user_system(precision):
    """test/solve.f90:320-365 on the GPU path."""
    g = P.default_gpu_options(precision=precision)
    ru, st = P.solve(ClosedForm(), gpu=g)
    assert st == 0
    s = P.SparseSystem(2)
    s.add_equation([1, 1, -5], [[2, 0, 0], [0, 2, 0]])
    s.add_equation([1, -2, 1], [[1, 0, 1], [2, 1, 0]])
    rs, st = P.solve(s, gpu=g)
    assert st == 0
    assert ru.nsolutions > 0 and ru.nsolutions == rs.nsolutions
    assert set_distance(ru.solutions, rs.solutions) <= 1e-11
    resid = max(np.max(np.abs(ClosedForm().evaluate(x)[0])) / max(1.0, np.max(np.abs(x))) ** 3
                for x in ru.solutions)
    assert resid <= 1e-13
    assert ru.nduplicates == 0


def user_cases():
    return {
        "closed_form": ClosedForm(),
        "circle_cubic": CircleCubic(),
        "mixed": TermEvaluator(2, [([1, -1], [[1, 0], [1, 0]]), ([1, -3, 2], [[3, 1, 0], [0, 0, 0]])]),
        "katsura3": TermEvaluator(*W.katsura(3)),
        "cyclic5": TermEvaluator(*W.cyclic(5)),
    }


_REF = {}


@pytest.mark.parametrize("precision", [P.PHC_PREC_FP64, P.PHC_PREC_MIXED])
@pytest.mark.parametrize("name", list(user_cases()))
def test_user_system_parity(orc, name, precision):
    """Per path against the restatement's user-system path: identical
    statuses, windings, classification and solution indices; counts equal;
    regular endpoints within 1e-10, singular ones within 1e-6."""
    usys = user_cases()[name]
    if name not in _REF:  # the restatement's side does not depend on the precision
        _REF[name] = orc.solve(orc.UserSystem(usys))
    ref, st1 = _REF[name]
    got, st2 = P.solve(usys, gpu=P.default_gpu_options(precision=precision))
    assert st1 == st2 == 0
    assert got.npaths == ref.npaths
    for key in ("nsolutions", "nreal", "nsingular", "ninfinite", "nfailed", "nduplicates"):
        assert getattr(got, key) == getattr(ref, key), key
    for key in ("status", "winding_number", "at_infinity", "singular", "is_real",
                "solution_index", "singular_index"):
        assert np.array_equal(got.paths[key], ref.paths[key]), key
    if ref.nsolutions:
        assert set_distance(got.solutions, ref.solutions) <= TOL_REGULAR
    if ref.nsingular:
        assert set_distance(got.singular_solutions, ref.singular_solutions) <= TOL_SINGULAR


def test_user_systems_through_the_server():
    """A user system submitted to the serving loop gives the same result as
    solve() on it, also when mixed with sparse systems in one batch."""
    users = [ClosedForm(), CircleCubic(), TermEvaluator(*W.katsura(3))]
    others = [W.build(P.SparseSystem, *W.stream_system(400 + i)) for i in range(3)]
    srv = P.Server(nslots=2, max_batch_systems=6)
    try:
        tickets = []
        for u, o in zip(users, others):
            for s in (u, o):
                t, st = srv.submit(s)
                assert st == 0
                tickets.append((s, t))
        for _, t in tickets:
            assert srv.wait(t, 120000) == 0
        got = [(s, srv.result(t)) for s, t in tickets]
    finally:
        srv.close()
    for s, (res, st, _lat) in got:
        alone, st2 = P.solve(s)
        assert st == st2 == 0
        for key in ("npaths", "nsolutions", "nreal", "nsingular", "ninfinite", "nfailed",
                    "nduplicates"):
            assert getattr(res, key) == getattr(alone, key), key
        for key in ("status", "winding_number", "at_infinity", "singular", "is_real",
                    "solution_index"):
            assert np.array_equal(res.paths[key], alone.paths[key]), key
        if alone.nsolutions:
            assert set_distance(res.solutions, alone.solutions) <= TOL_REGULAR
