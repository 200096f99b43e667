"""The multiply-high division by an invariant divisor that splits cell indices on the
device (Granlund & Montgomery 1994, fig. 4.1), restated in Python with the same 32-bit
arithmetic as make_fastdiv/fast_div in csrc/mcs_internal.h, checked exhaustively on edges
and randomly elsewhere; the device path is checked end to end by the mesh parity tests."""
import random


def _magic(d):
    l = (d - 1).bit_length()
    return ((1 << 32) * ((1 << l) - d) // d + 1) & 0xFFFFFFFF, min(l, 1), max(l - 1, 0)


def _div(n, d):
    m, s1, s2 = _magic(d)
    t = (m * n) >> 32
    return (t + ((n - t) >> s1)) >> s2


def test_fast_division_is_exact():
    rng = random.Random(7)
    ds = [1, 2, 3, 7, 128, 129, 255, 256, 512, 1000, 1024, 65537, 2**31 - 1, 2**31, 2**32 - 1]
    ds += [rng.randrange(1, 2**32) for _ in range(500)]
    for d in ds:
        ns = [0, 1, d - 1, d, d + 1, 2**32 - 1, 2**31] + [rng.randrange(0, 2**32) for _ in range(200)]
        for n in ns:
            if 0 <= n < 2**32:
                assert _div(n, d) == n // d, (n, d)
