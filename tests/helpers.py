"""Helpers mirroring the reference's test/testing.f90."""
import numpy as np


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
