"""The seeded input generators behind every parity test and bench workload
(aoclfftz_b200.synthetic), on the CPU: the vectorised splitmix64 stream
against a plain-integer restatement of the published algorithm, the ranges
and moments of the derived draws, and the length classes of the ragged
workload."""
import numpy as np
import pytest

from aoclfftz_b200 import synthetic

MASK = (1 << 64) - 1


def splitmix64_ref(seed, n):
    """Published splitmix64: state += golden gamma, then the two xor-shift-multiply rounds."""
    out, state = [], seed & MASK
    for _ in range(n):
        state = (state + 0x9E3779B97F4A7C15) & MASK
        z = state
        z = ((z ^ (z >> 30)) * 0xBF58476D1CE4E5B9) & MASK
        z = ((z ^ (z >> 27)) * 0x94D049BB133111EB) & MASK
        out.append(z ^ (z >> 31))
    return out


@pytest.mark.parametrize("seed", [0, 1, 1234, (1 << 64) - 5])
def test_splitmix64_matches_the_algorithm(seed):
    got = [int(v) for v in synthetic.splitmix64(seed, 257)]
    assert got == splitmix64_ref(seed, 257)


def test_splitmix64_first_output_and_offsets():
    assert int(synthetic.splitmix64(0, 1)[0]) == 0xE220A8397B1DCDAF
    full = synthetic.splitmix64(99, 100)
    assert np.array_equal(synthetic.splitmix64(99, 40, offset=60), full[60:])


def test_ranges_and_moments():
    u = synthetic.u01(5, 200000)
    assert u.min() >= 0.0 and u.max() < 1.0 and abs(u.mean() - 0.5) < 0.005
    v = synthetic.uniform(6, 200000)
    assert v.min() >= -1.0 and v.max() < 1.0 and abs(v.mean()) < 0.01
    g = synthetic.normal(7, 200001)
    assert g.shape == (200001,) and abs(g.mean()) < 0.01 and abs(g.var() - 1.0) < 0.02
    c = synthetic.complex_uniform(8, 1000)
    assert c.dtype == np.complex64 and np.all(np.abs(c.real) <= 1) and np.all(np.abs(c.imag) <= 1)
    # interleaved draw order: re of element k is draw 2k, im draw 2k + 1
    assert np.allclose(c.real, synthetic.uniform(8, 2000)[0::2].astype(np.float32))


def test_number_classes():
    assert [synthetic._next_pow2(n) for n in (1, 2, 3, 1000, 4096, 4097)] == [1, 2, 4, 1024, 4096, 8192]
    assert [n for n in range(2, 30) if synthetic._smooth7(n)] == [2, 3, 4, 5, 6, 7, 8, 9, 10, 12, 14, 15, 16, 18,
                                                                  20, 21, 24, 25, 27, 28]
    assert [n for n in range(0, 40) if synthetic._is_prime(n)] == [2, 3, 5, 7, 11, 13, 17, 19, 23, 29, 31, 37]
    assert synthetic._is_prime(65521) and not synthetic._is_prime(65535)


def test_ragged_sizes():
    s = synthetic.ragged_sizes(4242, 4096)
    assert s == synthetic.ragged_sizes(4242, 4096) and len(s) == 4096
    assert min(s) >= 2 and max(s) <= 65536
    pow2 = sum(1 for n in s if n & (n - 1) == 0)
    prime = sum(1 for n in s if synthetic._is_prime(n) and n & (n - 1))
    assert all((n & (n - 1)) == 0 or synthetic._smooth7(n) or synthetic._is_prime(n) for n in s)
    # one third each by a uniform draw (pow2 also catches the smooth class's powers of two
    # and the prime 2), so the counts sit near 4096 / 3
    assert 1200 < pow2 < 1750 and 1050 < prime < 1500
