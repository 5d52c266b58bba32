"""Helpers mirroring the reference's test/testing.f90, and the parity
check of a GPU solve() against the restatement's."""
import numpy as np

# finite regular endpoints: relative max-norm error (the tracker's
# corrector tolerance is 1e-10); singular endpoints: the reference's
# singular_dedup_tol, since such endpoints are less accurate
TOL_REGULAR = 1e-10
TOL_SINGULAR = 1e-6


def set_distance(a, b):
    """set_distance, test/testing.f90:219-261: rows of a and b are points;
    largest relative distance of a point of either set to its nearest
    point in the other set; huge if the counts differ."""
    a = np.atleast_2d(np.asarray(a, dtype=np.complex128))
    b = np.atleast_2d(np.asarray(b, dtype=np.complex128))
    if a.shape[0] != b.shape[0]:
        return np.finfo(float).max

    def nearest(x, pts):
        return min(np.max(np.abs(x - p)) / max(1.0, np.max(np.abs(x))) for p in pts)

    d = 0.0
    for x in a:
        d = max(d, nearest(x, b))
    for x in b:
        d = max(d, nearest(x, a))
    return d


def norm_inf(z):
    z = np.asarray(z)
    return float(np.max(np.abs(z))) if z.size else 0.0


def jacobian_fd_error(evaluate, x):
    """jacobian_fd_error, test/testing.f90:124-156, for evaluate(x) ->
    (f, jac)."""
    x = np.asarray(x, dtype=np.complex128)
    f, jac = evaluate(x)
    err = 0.0
    for j in range(x.size):
        h = 1.0e-5 * max(1.0, abs(x[j]))
        xp = x.copy()
        xp[j] = x[j] + h
        fp, _ = evaluate(xp)
        xp[j] = x[j] - h
        fm, _ = evaluate(xp)
        err = max(err, np.max(np.abs((fp - fm) / (2 * h) - jac[:, j])))
    return err / max(1.0, np.max(np.abs(jac)))


class ClosedForm:
    """The user system of test/solve.f90:16-57 and test/system.f90:18-63:
    F_1 = x1^2 + x2^2 - 5, F_2 = x1 x2^2 - 2 x2 + x1, degrees (2, 3)."""

    def nvars(self):
        return 2

    def degrees(self):
        return [2, 3]

    def evaluate(self, x):
        f = np.array([x[0] ** 2 + x[1] ** 2 - 5.0, x[0] * x[1] ** 2 - 2.0 * x[1] + x[0]])
        jac = np.array([[2.0 * x[0], 2.0 * x[1]], [x[1] ** 2 + 1.0, 2.0 * x[0] * x[1] - 2.0]])
        return f, jac


class CircleCubic:
    """The user system of app/example.f90:15-54: x^2 + y^2 = 4 and
    y = x^3 - 2x + 1/2, degrees (2, 3)."""

    def nvars(self):
        return 2

    def degrees(self):
        return [2, 3]

    def evaluate(self, x):
        f = np.array([x[0] ** 2 + x[1] ** 2 - 4.0, x[0] ** 3 - 2.0 * x[0] + 0.5 - x[1]])
        jac = np.array([[2.0 * x[0], 2.0 * x[1]], [3.0 * x[0] ** 2 - 2.0, -1.0]])
        return f, jac


class TermEvaluator:
    """A user system that evaluates a term list (n, [(coefs, exps), ...]) in
    closed form, as user code would: F_i = sum_k c_k x^a_k and its
    derivatives, vectorized over the terms."""

    def __init__(self, n, eqs):
        self.n = n
        self.eqs = [(np.asarray(c, dtype=np.complex128), np.asarray(e, dtype=np.int64).reshape(n, -1))
                    for c, e in eqs]

    def nvars(self):
        return self.n

    def degrees(self):
        return [int(np.max(np.sum(e[:, c != 0], axis=0))) for c, e in self.eqs]

    def evaluate(self, x):
        n = self.n
        f = np.zeros(n, dtype=np.complex128)
        jac = np.zeros((n, n), dtype=np.complex128)
        for i, (c, e) in enumerate(self.eqs):
            f[i] = np.sum(c * np.prod(x[:, None] ** e, axis=0))
            for j in range(n):
                d = e.copy()
                d[j] = np.maximum(d[j] - 1, 0)
                jac[i, j] = np.sum(c * e[j] * np.prod(x[:, None] ** d, axis=0))
        return f, jac


def reference_bookkeeping(n, paths, x, o):
    """add_solution, add_singular, find and collect_real of the reference
    (src/solve.f90:330-426), restated directly in path order: the first
    stored point within tol * max(1, ||x||_inf) of x by max-norm distance
    (moduli as hypot). Returns a dict of the counts, per-path indices,
    solution arrays and multiplicities. Moduli come from np.hypot on the
    real and imaginary parts, which matches the C library's hypot (the
    modulus of Fortran's abs); numpy's complex abs is off by one ulp for
    some inputs, which flips decisions that sit exactly at a threshold."""
    def norm_inf(v):
        return float(np.max(np.hypot(v.real, v.imag))) if len(v) else 0.0

    def find(v, pts, tol):
        scale = max(1.0, norm_inf(v))
        for j, p in enumerate(pts):
            if norm_inf(v - p) <= tol * scale:
                return j + 1
        return 0

    sols, ssols, mult = [], [], []
    sol_idx = np.zeros(len(paths), dtype=np.int32)
    sing_idx = np.zeros(len(paths), dtype=np.int32)
    nfailed = ninfinite = nduplicates = 0
    for k in range(len(paths)):
        p = paths[k]
        if p["status"] != 0:
            nfailed += 1
        elif p["at_infinity"]:
            ninfinite += 1
        elif p["singular"]:
            j = find(x[k], ssols, o.singular_dedup_tol)
            if j > 0:
                mult[j - 1] += 1
            else:
                ssols.append(x[k].copy())
                mult.append(1)
                j = len(ssols)
            sing_idx[k] = j
        else:
            j = find(x[k], sols, o.dedup_tol)
            if j > 0:
                nduplicates += 1
            else:
                sols.append(x[k].copy())
                j = len(sols)
            sol_idx[k] = j
    reals = [s.real for s in sols if np.max(np.abs(s.imag)) <= o.real_tol * max(1.0, norm_inf(s))]
    return dict(nfailed=nfailed, ninfinite=ninfinite, nduplicates=nduplicates,
                solution_index=sol_idx, singular_index=sing_idx,
                solutions=np.array(sols, dtype=np.complex128).reshape(len(sols), n),
                singular_solutions=np.array(ssols, dtype=np.complex128).reshape(len(ssols), n),
                multiplicities=np.array(mult, dtype=np.int32),
                real_solutions=np.array(reals).reshape(len(reals), n))


# The end game's convergence flag compares the relative change of its last
# two estimates with endgame tol = 1e-11. For paths at infinity those
# changes sit anywhere between 1e-12 and 1e-8, and rounding decides the flag
# (the reference's own LU and the GPU's elimination round differently; the
# classification, winding number and counts do not depend on the flag).
ENDGAME_FLAG_BAND = 1e-7


def endgame_status_agrees(ref_paths, got_paths):
    """Per path: the end game status is identical, or the path ends at
    infinity on both sides with both end game errors at most
    ENDGAME_FLAG_BAND (a flag that rounding decides)."""
    same = ref_paths["endgame_status"] == got_paths["endgame_status"]
    free = ((ref_paths["at_infinity"] != 0) & (got_paths["at_infinity"] != 0) &
            (ref_paths["endgame_error"] <= ENDGAME_FLAG_BAND) &
            (got_paths["endgame_error"] <= ENDGAME_FLAG_BAND))
    return same | free


def assert_steps_comparable(ref_paths, got_paths):
    """No path takes pathologically more steps than the restatement's: at
    most twice its steps plus 1000; on the paths at infinity whose end game
    flag rounding decides (endgame_status_agrees), where one side may
    converge early and the other continue down to the smallest radius, at
    most 8 times plus 5000. The total stays within 10 %."""
    rs = ref_paths["naccepted"].astype(np.int64) + ref_paths["nrejected"]
    gs = got_paths["naccepted"].astype(np.int64) + got_paths["nrejected"]
    band = ((ref_paths["at_infinity"] != 0) & (got_paths["at_infinity"] != 0) &
            (ref_paths["endgame_error"] <= ENDGAME_FLAG_BAND) &
            (got_paths["endgame_error"] <= ENDGAME_FLAG_BAND))
    limit = np.where(band, 8 * rs + 5000, 2 * rs + 1000)
    bad = np.nonzero(gs > limit)[0]
    assert bad.size == 0, ("steps", bad[:10], gs[bad[:10]], rs[bad[:10]])
    assert gs.sum() <= 1.1 * rs.sum() + 1000, (gs.sum(), rs.sum())


def assert_parity(n, ref, got):
    """Parity of a GPU solve() result with the restatement's: identical
    counts, multiplicities and per-path status, winding number,
    classification and solution/singular indices; end game status
    identical up to endgame_status_agrees; finite regular endpoints within
    TOL_REGULAR (relative, max norm) and the singular solution sets within
    TOL_SINGULAR; step counts comparable."""
    assert got.npaths == ref.npaths
    for key in ("nsolutions", "nreal", "nsingular", "ninfinite", "nfailed", "nduplicates"):
        assert getattr(got, key) == getattr(ref, key), key
    assert list(got.multiplicities) == list(ref.multiplicities)
    for key in ("status", "winding_number", "at_infinity", "singular", "is_real",
                "solution_index", "singular_index"):
        assert np.array_equal(got.paths[key], ref.paths[key]), (
            key, np.nonzero(got.paths[key] != ref.paths[key])[0][:10])
    ok = endgame_status_agrees(ref.paths, got.paths)
    assert ok.all(), ("endgame_status", np.nonzero(~ok)[0][:10])
    assert_steps_comparable(ref.paths, got.paths)
    reg = (ref.paths["solution_index"] > 0)
    if reg.any():
        d = np.max(np.abs(got.x[reg] - ref.x[reg]), axis=1) / np.maximum(
            1.0, np.max(np.abs(ref.x[reg]), axis=1))
        assert d.max() <= TOL_REGULAR, d.max()
        assert set_distance(got.solutions, ref.solutions) <= TOL_REGULAR
    sing = (ref.paths["singular_index"] > 0)
    if sing.any():
        assert set_distance(got.singular_solutions, ref.singular_solutions) <= TOL_SINGULAR
