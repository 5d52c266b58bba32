"""Host-side restatement of polyhomocont's seeded generator (type(rng),
src/random.f90:1-111): L'Ecuyer's combined multiplicative linear
congruential generator with the reference's seeding (16 discarded draws),
unit_complex and normal_complex (Box-Muller, variance 1/2 per part).

Used to generate the synthetic benchmark systems deterministically. The
same generator, in C++, draws gamma, b and the patch inside the library
(phc_homotopy_init), so a seed gives the same homotopy as the reference.
"""
import math

_M1 = 2147483563
_M2 = 2147483399
_A1 = 40014
_A2 = 40692
_PI = 3.14159265358979323846


class Rng:
    def __init__(self, seed=None):
        self.s1 = 1234567
        self.s2 = 7654321
        if seed is not None:
            self.seed(seed)

    def seed(self, seed):
        """rng_seed, src/random.f90:43-62"""
        s = abs(int(seed))
        self.s1 = s % (_M1 - 1) + 1
        self.s2 = (s * 7919 + 104729) % (_M2 - 1) + 1
        for _ in range(16):
            self.uniform()

    def uniform(self):
        """rng_uniform, src/random.f90:64-78: deviate in (0, 1)"""
        self.s1 = (_A1 * self.s1) % _M1
        self.s2 = (_A2 * self.s2) % _M2
        z = self.s1 - self.s2
        if z < 1:
            z += _M1 - 1
        return float(z) / float(_M1)

    def unit_complex(self):
        """rng_unit_complex, src/random.f90:80-91"""
        phi = 2.0 * _PI * self.uniform()
        return complex(math.cos(phi), math.sin(phi))

    def normal_complex(self):
        """rng_normal_complex, src/random.f90:93-109"""
        r = math.sqrt(-math.log(self.uniform()))
        phi = 2.0 * _PI * self.uniform()
        return complex(r * math.cos(phi), r * math.sin(phi))
