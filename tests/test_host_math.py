"""CPU: integer identities the kernels rely on."""
import numpy as np


def test_rans_reciprocal_division_is_exact():
    """floor(x / f) == (x * ceil(2^(31+s)/f)) >> (31+s), s = ceil(log2 f), for x < 2^31 (encoder state bound)."""
    rng = np.random.default_rng(0)
    for f in range(1, 4097):
        s = (f - 1).bit_length()
        M = ((1 << (31 + s)) + f - 1) // f
        assert M < 2 ** 32
        xs = np.concatenate([rng.integers(0, 2 ** 31, 64), np.arange(1, 33) * f - 1, [2 ** 31 - 1, 0, f, 2 ** 31 - f]])
        for x in xs:
            x = int(x)
            if 0 <= x < 2 ** 31:
                assert (x * M) >> (31 + s) == x // f, (f, x)


def test_morton_neighbour_arithmetic():
    """+-1 along one axis on the interleaved code, as decode.cu / encode.cu do it, equals re-encoding."""
    def mort(x, y, z):
        r = 0
        for i in range(10):
            r |= ((x >> i) & 1) << (3 * i) | ((y >> i) & 1) << (3 * i + 1) | ((z >> i) & 1) << (3 * i + 2)
        return r

    rng = np.random.default_rng(1)
    for lc in range(1, 7):
        size = 1 << lc
        lvl = (1 << (3 * lc)) - 1
        for _ in range(300):
            c = [int(v) for v in rng.integers(0, size, 3)]
            n = mort(*c)
            for a in range(3):
                m = (0x09249249 << a) & lvl
                bit = 1 << a
                if c[a] + 1 < size:
                    N = (((n | ~m) + bit) & m) | (n & ~m)
                    d = list(c); d[a] += 1
                    assert N & 0xFFFFFFFF == mort(*d)
                else:
                    assert (n & m) == m
                if c[a] > 0:
                    N = (((n & m) - bit) & m) | (n & ~m)
                    d = list(c); d[a] -= 1
                    assert N == mort(*d)
                else:
                    assert (n & m) == 0
