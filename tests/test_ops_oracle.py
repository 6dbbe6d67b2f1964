"""CPU checks of the oracle's restatement of the ops beside the NTT (src/ops_complex.rs).

Each expectation is the reference's own test's (src/ops_complex.rs:1366-1670):
powers of a domain generator compared with generator^i, powers of a base
with base^i, the omega shift with x_i * w^(shift * i), and the bit reversal
with dst[reverse_bits(i)] = src[i] -- computed here in pure Python, so the C
oracle is pinned independently of itself.
"""
import numpy as np
import pytest

import oracle
from conftest import P, uniform


def brev(x: int, bits: int) -> int:
    return int(format(x, f"0{bits}b")[::-1], 2) if bits else 0


def test_bit_reverse_matches_definition_and_is_an_involution():
    rng = np.random.default_rng(1)
    for log_rows in (0, 1, 3, 8, 11):
        rows, cols = 1 << log_rows, 3
        x = uniform(rng, cols * rows)
        y = oracle.bit_reverse(x, log_rows, cols)
        for c in range(cols):
            for i in range(rows):
                assert y[c * rows + brev(i, log_rows)] == x[c * rows + i]
        np.testing.assert_array_equal(oracle.bit_reverse(y, log_rows, cols), x)


@pytest.mark.parametrize("inverse", [False, True])
@pytest.mark.parametrize("of_g", [False, True])
def test_powers_of_w_and_g(inverse, of_g):
    """src/ops_complex.rs:1366-1437: 2^16 powers in two halves (offset 0, n/2) equal generator^i, where the
    generator is w_{2^16} or 7^(2^(24-16)), inverted when inverse."""
    log_degree = 16
    n = 1 << log_degree
    gen = pow(7, 1 << (24 - log_degree), P) if of_g else oracle.root_of_unity(log_degree)
    if inverse:
        gen = pow(gen, P - 2, P)
    got = np.concatenate([oracle.powers_of(log_degree, 0, inverse, False, of_g, n // 2),
                          oracle.powers_of(log_degree, n // 2, inverse, False, of_g, n // 2)])
    acc = 1
    for i in range(0, n, 257):
        assert int(got[i]) == pow(gen, i, P), i
    for i in range(n):
        assert int(got[i]) == acc
        acc = acc * gen % P


def test_powers_of_index_conventions():
    """bit_reverse reverses log_degree bits of i + offset; the exponent is (idx << (24 - log_degree)) mod 2^24."""
    w24 = oracle.root_of_unity(24)
    for log_degree, offset, bitrev in ((5, 7, True), (24, 2**32 - 3, False), (0, 9, True), (3, 2**31, False)):
        got = oracle.powers_of(log_degree, offset, False, bitrev, False, 12)
        for i in range(12):
            r = (i + offset) % 2**32
            idx = brev(r % (1 << log_degree), log_degree) if bitrev else r
            e = ((idx << (24 - log_degree)) % 2**32) % 2**24
            assert int(got[i]) == pow(w24, e, P)


def ext_mul(a, b):
    return ((a[0] * b[0] + 7 * a[1] * b[1]) % P, (a[0] * b[1] + a[1] * b[0]) % P)


def test_powers_by_base_field_and_extension():
    """src/ops_complex.rs:1438-1533: base 42 (and 42 + 42x) to the powers i, two halves."""
    n = 1 << 12
    got = np.concatenate([oracle.powers_by(42, 0, False, n // 2), oracle.powers_by(42, n // 2, False, n // 2)])
    assert all(int(got[i]) == pow(42, i, P) for i in range(n))
    ext = oracle.powers_by((42, 42), 0, False, n)
    acc = (1, 0)
    for i in range(n):
        assert (int(ext[i]), int(ext[n + i])) == acc, i
        acc = ext_mul(acc, (42, 42))
    # bit_reverse reverses all 32 bits of i; the u32 exponent wraps
    got = oracle.powers_by(3, 2**32 - 5, True, 8)
    for i in range(8):
        assert int(got[i]) == pow(3, (brev(i, 32) + 2**32 - 5) % 2**32, P)
    got = oracle.powers_by(P + 5, 2**32 - 2, False, 4)  # a non-canonical base reads mod p
    assert [int(v) for v in got] == [pow(5, (i + 2**32 - 2) % 2**32, P) for i in range(4)]


@pytest.mark.parametrize("inverse", [False, True])
def test_omega_shift(inverse):
    """src/ops_complex.rs:1534-1618: x_i * w^(42 i) with w = w_{2^16} (inverse: w^-1), two halves."""
    rng = np.random.default_rng(2)
    log_degree, n, shift = 16, 1 << 10, 42
    x = uniform(rng, n)
    w = oracle.root_of_unity(log_degree)
    if inverse:
        w = pow(w, P - 2, P)
    got = np.concatenate([oracle.omega_shift(x[: n // 2], log_degree, 0, inverse, shift),
                          oracle.omega_shift(x[n // 2:], log_degree, n // 2, inverse, shift)])
    for i in range(n):
        assert int(got[i]) == int(x[i]) * pow(w, shift * i, P) % P
    # u32 wrap of shift * (i + offset) before the reduction mod 2^24
    got = oracle.omega_shift(x[:4], 20, 2**31 + 1, False, 2**30 + 3)
    w24 = oracle.root_of_unity(24)
    for i in range(4):
        e = (((2**30 + 3) * (i + 2**31 + 1)) % 2**32 << 4) % 2**32 % 2**24
        assert int(got[i]) == int(x[i]) * pow(w24, e, P) % P
