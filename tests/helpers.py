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
