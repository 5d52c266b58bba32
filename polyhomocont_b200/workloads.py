"""Synthetic polynomial systems for the benchmark configurations and the
reference's benchmark families.

Every generator is deterministic: coefficients and monomial choices come
from the reference generator (polyhomocont_b200.rng.Rng, a restatement of
src/random.f90) seeded with 20261203 + 100*cfg + sys_index. A system is
returned as (n, equations), each equation a pair (coefs[T], exps[n, T]) in
the layout of sparse_system%add_equation (src/sparse.f90:83-141): column k
of exps is the exponent vector of term k.

Configurations (one GPU):
  cfg1  n=4, degrees 2, all 15 monomials of degree <= 2, 16 paths
  cfg2  n=10, degrees 2, 20 distinct monomials (of 66) per equation, at
        least one of degree 2, 1024 paths (many end at infinity)
  cfg3  n=4, F_i = sum_j A_ij (x_j - r_j)^2 + B_ij (x_j - r_j)^3, 81 paths,
        16 of them end at the known singular root r
  cfg4  stream of random sparse systems: n ~ U{2..8}, d_i ~ U{2,3} with
        prod d_i <= 2048, 6-30 monomials per equation (one of degree d_i)
  cfg5  n=16, degrees 2, 24 distinct monomials (of 153), 65536 paths
"""
import itertools

import numpy as np

from .rng import Rng

BASE_SEED = 20261203


def seed_for(cfg, sys_index=0):
    return BASE_SEED + 100 * cfg + sys_index


def monomials(n, dmax):
    """All exponent vectors of total degree <= dmax in n variables, in
    ascending lexicographic order of the exponent tuples."""
    out = []
    for d in range(dmax + 1):
        for combo in itertools.combinations_with_replacement(range(n), d):
            e = [0] * n
            for j in combo:
                e[j] += 1
            out.append(tuple(e))
    out.sort()
    return out


def _equation(coefs, exps_list, n):
    exps = np.zeros((n, len(exps_list)), dtype=np.int32)
    for k, e in enumerate(exps_list):
        exps[:, k] = e
    return (np.asarray(coefs, dtype=np.complex128), exps)


def dense_quadratic(n=4, seed=None):
    """cfg1: every equation has all monomials of degree <= 2."""
    g = Rng(seed if seed is not None else seed_for(1))
    mons = monomials(n, 2)
    eqs = []
    for _ in range(n):
        coefs = [g.normal_complex() for _ in mons]
        eqs.append(_equation(coefs, mons, n))
    return n, eqs


def random_sparse(n, d, nterms, g, exact_degree=True):
    """One equation: nterms distinct monomials drawn uniformly from those
    of degree <= d (index floor(M*u), repeats rejected), resampled until
    one has degree exactly d; complex normal coefficients in the order of
    the monomial list."""
    mons = monomials(n, d)
    M = len(mons)
    if nterms > M:
        raise ValueError("more terms than monomials")
    while True:
        chosen = []
        seen = set()
        while len(chosen) < nterms:
            idx = min(int(M * g.uniform()), M - 1)
            if idx in seen:
                continue
            seen.add(idx)
            chosen.append(idx)
        if not exact_degree or any(sum(mons[i]) == d for i in chosen):
            break
    chosen.sort()
    coefs = [g.normal_complex() for _ in chosen]
    return _equation(coefs, [mons[i] for i in chosen], n)


def sparse_quadratic(n, nterms, seed):
    g = Rng(seed)
    return n, [random_sparse(n, 2, nterms, g) for _ in range(n)]


def cfg2(seed=None):
    """n=10, 20 of 66 monomials per equation, 1024 paths."""
    return sparse_quadratic(10, 20, seed if seed is not None else seed_for(2))


def cfg5(seed=None):
    """n=16, 24 of 153 monomials per equation, 65536 paths."""
    return sparse_quadratic(16, 24, seed if seed is not None else seed_for(5))


def singular_cubic(n=4, seed=None):
    """cfg3: F_i = sum_j A_ij (x_j - r_j)^2 + B_ij (x_j - r_j)^3, expanded
    into the monomials 1, x_j, x_j^2, x_j^3. Draw order: r, then A and B
    row by row. Returns (n, eqs, r)."""
    g = Rng(seed if seed is not None else seed_for(3))
    r = [g.normal_complex() for _ in range(n)]
    A = [[g.normal_complex() for _ in range(n)] for _ in range(n)]
    B = [[g.normal_complex() for _ in range(n)] for _ in range(n)]
    eqs = []
    for i in range(n):
        const = 0j
        coefs, exps = [], []
        for j in range(n):
            a, b, rj = A[i][j], B[i][j], r[j]
            const += a * rj * rj - b * rj * rj * rj
            for p, c in ((1, -2 * a * rj + 3 * b * rj * rj),
                         (2, a - 3 * b * rj),
                         (3, b)):
                e = [0] * n
                e[j] = p
                coefs.append(c)
                exps.append(tuple(e))
        coefs.insert(0, const)
        exps.insert(0, tuple([0] * n))
        eqs.append(_equation(coefs, exps, n))
    return n, eqs, np.asarray(r, dtype=np.complex128)


def stream_system(sys_index, nmin=2, nmax=8, max_paths=2048):
    """cfg4: one system of the serving stream."""
    g = Rng(seed_for(4, sys_index))
    while True:
        n = nmin + min(int((nmax - nmin + 1) * g.uniform()), nmax - nmin)
        degs = [2 + min(int(2 * g.uniform()), 1) for _ in range(n)]
        if int(np.prod(degs)) <= max_paths:
            break
    eqs = []
    for i in range(n):
        d = degs[i]
        M = len(monomials(n, d))
        lo, hi = 6, min(30, M)
        nt = lo + min(int((hi - lo + 1) * g.uniform()), hi - lo)
        eqs.append(random_sparse(n, d, nt, g))
    return n, eqs


def poisson_arrivals(count, rate, seed=None):
    """Arrival times (s) of a Poisson process with the given rate."""
    g = Rng(seed if seed is not None else seed_for(4, 999999))
    t = 0.0
    out = []
    for _ in range(count):
        t += -np.log(g.uniform()) / rate
        out.append(t)
    return np.asarray(out)


def katsura(n):
    """Katsura-n (test/katsura.f90:145-202): unknowns u_0..u_n,
    u_0 + 2 sum u_k - 1 = 0 and sum_l u_|l| u_|m-l| - u_m = 0 for
    m = 0..n-1, repeated monomials kept as separate terms."""
    N = n + 1
    eqs = []
    coefs = [1.0] + [2.0] * n + [-1.0]
    exps = []
    e = [0] * N
    e[0] = 1
    exps.append(tuple(e))
    for k in range(1, n + 1):
        e = [0] * N
        e[k] = 1
        exps.append(tuple(e))
    exps.append(tuple([0] * N))
    eqs.append(_equation(coefs, exps, N))
    for m in range(n):
        coefs, exps = [], []
        for l in range(-n, n + 1):
            if abs(m - l) > n:
                continue
            e = [0] * N
            e[abs(l)] += 1
            e[abs(m - l)] += 1
            coefs.append(1.0)
            exps.append(tuple(e))
        e = [0] * N
        e[m] = 1
        coefs.append(-1.0)
        exps.append(tuple(e))
        eqs.append(_equation(coefs, exps, N))
    return N, eqs


def cyclic(n):
    """Cyclic-n (test/cyclic.f90:263-289)."""
    eqs = []
    for k in range(1, n):
        exps = np.zeros((n, n), dtype=np.int32)
        for i in range(n):
            for j in range(k):
                exps[(i + j) % n, i] = 1
        eqs.append((np.ones(n, dtype=np.complex128), exps))
    exps = np.zeros((n, 2), dtype=np.int32)
    exps[:, 0] = 1
    eqs.append((np.array([1.0, -1.0], dtype=np.complex128), exps))
    return n, eqs


def build(system_cls, n, eqs):
    """Builds a sparse system object of the given class (anything with
    init(n) and add_equation(coefs, exps))."""
    s = system_cls()
    s.init(n)
    for c, e in eqs:
        st = s.add_equation(c, e)
        if st != 0:
            raise ValueError(f"add_equation failed with status {st}")
    return s
