"""Seeded synthetic inputs (splitmix64 stream, reproducible on any machine).

u01(seed, n)     i.i.d. U[0, 1) doubles: top 53 bits of splitmix64 outputs.
uniform(seed, n) i.i.d. U[-1, 1).
normal(seed, n)  i.i.d. N(0, 1) by Box-Muller on consecutive U pairs.
The i-th output of splitmix64 is mix(seed + (i + 1) * 0x9E3779B97F4A7C15).
"""
import numpy as np

_G = np.uint64(0x9E3779B97F4A7C15)
_M1 = np.uint64(0xBF58476D1CE4E5B9)
_M2 = np.uint64(0x94D049BB133111EB)


def splitmix64(seed, n, offset=0):
    with np.errstate(over="ignore"):
        i = np.arange(offset + 1, offset + n + 1, dtype=np.uint64)
        z = np.uint64(seed) + i * _G
        z = (z ^ (z >> np.uint64(30))) * _M1
        z = (z ^ (z >> np.uint64(27))) * _M2
        z = z ^ (z >> np.uint64(31))
    return z


def u01(seed, n, offset=0):
    return (splitmix64(seed, n, offset) >> np.uint64(11)).astype(np.float64) * (1.0 / 9007199254740992.0)


def uniform(seed, n, offset=0):
    return 2.0 * u01(seed, n, offset) - 1.0


def normal(seed, n, offset=0):
    m = (n + 1) // 2
    u = u01(seed, 2 * m, 2 * offset)
    u1 = np.maximum(u[0::2], 2.0 ** -60)
    u2 = u[1::2]
    r = np.sqrt(-2.0 * np.log(u1))
    out = np.empty(2 * m)
    out[0::2] = r * np.cos(2 * np.pi * u2)
    out[1::2] = r * np.sin(2 * np.pi * u2)
    return out[:n]


def complex_uniform(seed, n, dtype=np.complex64):
    """n complex values with re, im i.i.d. U[-1, 1) (interleaved draw order)."""
    v = uniform(seed, 2 * n)
    return (v[0::2] + 1j * v[1::2]).astype(dtype)


def complex_normal(seed, n, dtype=np.complex128):
    v = normal(seed, 2 * n)
    return (v[0::2] + 1j * v[1::2]).astype(dtype)


def _next_pow2(n):
    p = 1
    while p < n:
        p *= 2
    return p


def _smooth7(n):
    for p in (2, 3, 5, 7):
        while n % p == 0:
            n //= p
    return n == 1


def _is_prime(n):
    if n < 2:
        return False
    if n % 2 == 0:
        return n == 2
    f = 3
    while f * f <= n:
        if n % f == 0:
            return False
        f += 2
    return True


def ragged_sizes(seed, count, lo=2, hi=65536):
    """Transform lengths of a ragged batch: N0 = round(exp(u)), u ~ U[ln lo, ln hi],
    then one third each (by a second draw) rounded up to the next power of two,
    the next 7-smooth number, or the next prime, clamped to hi."""
    u = u01(seed, 2 * count)
    out = []
    for i in range(count):
        n0 = int(round(np.exp(np.log(lo) + u[2 * i] * (np.log(hi) - np.log(lo)))))
        n0 = max(lo, min(hi, n0))
        cls = int(u[2 * i + 1] * 3)
        if cls == 0:
            n = _next_pow2(n0)
        elif cls == 1:
            n = n0
            while not _smooth7(n):
                n += 1
        else:
            n = n0
            while not _is_prime(n):
                n += 1
        if n > hi:
            n = hi
            if cls == 2:
                while not _is_prime(n):
                    n -= 1
        out.append(n)
    return out
