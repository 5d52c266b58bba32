"""Generates tests/golden/katsura.json from the reference's own Python
script (reference/ref_katsura.py: lex Groebner basis with sympy, roots with
mpmath at 40 digits), imported from the reference checkout. Run once in a
container that has the reference mounted:

    python tests/golden/make_katsura.py /path/to/reference

The JSON holds, for n = 3 and 4, the 2^n solutions (u_0..u_n) as
[re, im] pairs and the number of real solutions. The same values are
printed as Fortran constants in the reference's test/katsura.f90:23-137.
"""
import json
import os
import sys


def main():
    ref_root = sys.argv[1] if len(sys.argv) > 1 else None
    if ref_root is None:
        raise SystemExit("usage: make_katsura.py <reference checkout>")
    sys.path.insert(0, os.path.join(ref_root, "reference"))
    import mpmath
    import ref_katsura as rk  # the reference's generator

    out = {}
    for n in (3, 4):
        u, eqs = rk.katsura(n)
        sols, deg = rk.solve_shape_position(u, eqs)
        assert deg == 2 ** n and len(sols) == 2 ** n
        nreal = sum(all(abs(mpmath.mpc(c).imag) < mpmath.mpf("1e-30") for c in s)
                    for s in sols)
        out[f"katsura{n}"] = {
            "n": n,
            "nreal": int(nreal),
            "solutions": [[[float(mpmath.mpc(c).real), float(mpmath.mpc(c).imag)]
                           for c in s] for s in sols],
        }
    path = os.path.join(os.path.dirname(os.path.abspath(__file__)), "katsura.json")
    with open(path, "w") as f:
        json.dump(out, f, indent=1)
    print("wrote", path)


if __name__ == "__main__":
    main()
