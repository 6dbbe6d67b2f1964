"""CPU checks of the oracle itself (no GPU): the checker has to be right first.

* the fast oracle against an independent pure-Python DFT written from the
  definition, for every variant of batch_ntt_internal (src/ntt.rs:179-191)
  at tiny sizes;
* algebraic identities at larger sizes (inverse round trip, convolution
  theorem, linearity, LDE restriction);
* the root-of-unity convention (generator 7, two-adicity 32).
"""
import numpy as np
import pytest

import oracle
from conftest import P, raw_u64, uniform


def _brev(i, bits):
    return int(format(i, f"0{bits}b")[::-1], 2) if bits else 0


def _py_transform(x, log_n, bitrev_inputs, inverse, log_ext, coset_idx):
    """Pure-Python restatement of one column, straight from the definition."""
    n = 1 << log_n
    w32 = pow(7, (P - 1) >> 32, P)
    w = pow(w32, 1 << (32 - log_n), P)
    c = 1
    if log_ext:
        c = 7 * pow(pow(w32, 1 << (32 - log_n - log_ext), P), coset_idx, P) % P
    nat = [int(x[_brev(i, log_n)] if bitrev_inputs else x[i]) % P for i in range(n)]
    if inverse:
        wi = pow(w, P - 2, P)
        ninv = pow(n, P - 2, P)
        ci = pow(c, P - 2, P)
        y = [ninv * pow(ci, i, P) * sum(nat[m] * pow(wi, i * m, P) for m in range(n)) % P for i in range(n)]
    else:
        xs = [nat[i] * pow(c, i, P) % P for i in range(n)]
        y = [sum(xs[i] * pow(w, i * m, P) for i in range(n)) % P for m in range(n)]
    out = [0] * n
    for m in range(n):
        out[m if bitrev_inputs else _brev(m, log_n)] = y[m]
    return out


def test_root_of_unity():
    w32 = oracle.root_of_unity(32)
    assert w32 == pow(7, (P - 1) >> 32, P) == 0x185629DCDA58878C
    assert pow(w32, 1 << 31, P) == P - 1  # primitive 2^32-th root
    for k in range(1, 33):
        wk = oracle.root_of_unity(k)
        assert pow(wk, 1 << k, P) == 1 and pow(wk, 1 << (k - 1), P) == P - 1


@pytest.mark.parametrize("log_n", [1, 2, 3, 4, 5, 6])
@pytest.mark.parametrize("bitrev_inputs", [False, True])
@pytest.mark.parametrize("inverse", [False, True])
@pytest.mark.parametrize("log_ext,coset_idx", [(0, 0), (1, 1), (3, 3), (2, 0)])
def test_oracle_vs_definition(log_n, bitrev_inputs, inverse, log_ext, coset_idx):
    rng = np.random.default_rng(log_n * 100 + log_ext * 10 + coset_idx)
    n = 1 << log_n
    num = 3
    stride_in, stride_out = n + 2, n + 5
    x = raw_u64(rng, num * stride_in)
    got = oracle.batch_ntt(x, log_n, num, stride_in, stride_out, bitrev_inputs, inverse, log_ext, coset_idx)
    for c in range(num):
        exp = _py_transform(x[c * stride_in:c * stride_in + n], log_n, bitrev_inputs, inverse, log_ext, coset_idx)
        assert [int(v) for v in got[c * stride_out:c * stride_out + n]] == exp


def test_naive_dft_matches():
    """The C definition-based DFT agrees with the fast path (natural order; inverse without 1/n)."""
    rng = np.random.default_rng(3)
    for log_n in range(1, 9):
        n = 1 << log_n
        x = uniform(rng, n)
        for inverse in (False, True):
            y = oracle.dft_naive(x, log_n, inverse)
            if inverse:
                y = np.array([int(v) * pow(n, P - 2, P) % P for v in y], dtype=np.uint64)
            z = oracle.batch_ntt(x, log_n, 1, n, n, False, inverse, 0, 0)  # bit-reversed output
            np.testing.assert_array_equal(oracle.bitrev_permute(z, log_n), y)


@pytest.mark.parametrize("log_n", [10, 14, 17])
def test_roundtrip_and_linearity(log_n):
    rng = np.random.default_rng(log_n)
    n = 1 << log_n
    x = raw_u64(rng, 4 * n)
    for e, k in ((0, 0), (2, 3), (3, 7)):
        y = oracle.batch_ntt(x, log_n, 4, n, n, False, False, e, k, threads=4)
        z = oracle.batch_ntt(y, log_n, 4, n, n, True, True, e, k, threads=4)
        np.testing.assert_array_equal(z, oracle.canon(x))
    a = uniform(rng, n)
    b = uniform(rng, n)
    s = np.array([(int(u) + int(v)) % P for u, v in zip(a, b)], dtype=np.uint64)
    fa, fb, fs = (oracle.batch_ntt(t, log_n, 1, n, n, False, False, 1, 1) for t in (a, b, s))
    np.testing.assert_array_equal(fs, np.array([(int(u) + int(v)) % P for u, v in zip(fa, fb)], dtype=np.uint64))


def test_convolution_theorem():
    """NTT(a * b cyclic) = NTT(a) . NTT(b) for small n."""
    rng = np.random.default_rng(9)
    log_n = 6
    n = 1 << log_n
    a = uniform(rng, n)
    b = uniform(rng, n)
    conv = [0] * n
    for i in range(n):
        for j in range(n):
            conv[(i + j) % n] = (conv[(i + j) % n] + int(a[i]) * int(b[j])) % P
    fa = oracle.batch_ntt(a, log_n, 1, n, n, False, False)
    fb = oracle.batch_ntt(b, log_n, 1, n, n, False, False)
    fc = oracle.batch_ntt(np.array(conv, dtype=np.uint64), log_n, 1, n, n, False, False)
    np.testing.assert_array_equal(fc, np.array([int(u) * int(v) % P for u, v in zip(fa, fb)], dtype=np.uint64))


def test_lde_restricts_to_original_domain():
    """Coset LDE of evaluations: evaluating the interpolant on c_k H agrees with a direct DFT of size B*n."""
    rng = np.random.default_rng(4)
    log_n, log_b, cols = 7, 2, 3
    n, B = 1 << log_n, 1 << log_b
    ev = uniform(rng, cols * n)  # bit-reversed evaluations on H
    out = oracle.lde(ev, log_n, cols, n, log_b).reshape(B, cols, n)
    coef = oracle.batch_ntt(ev, log_n, cols, n, n, True, True).reshape(cols, n)
    # g * H_{Bn}: zero-padded coefficients scaled by g^i, DFT of size B*n, natural order
    for c in range(cols):
        padded = np.zeros(B * n, dtype=np.uint64)
        padded[:n] = coef[c]
        big = oracle.batch_ntt(padded, log_n + log_b, 1, B * n, B * n, False, False, log_b, 0)
        # coset k of size n is {g w_{Bn}^(k + B m)}: natural index k + B m of the big evaluation
        big_nat = oracle.bitrev_permute(big, log_n + log_b)
        # big used coset 7 * w_{(Bn) 2^b}^0 = 7: evaluations at 7 * w_{Bn}^j
        for k in range(B):
            exp = big_nat[k::B]  # natural order over m
            np.testing.assert_array_equal(oracle.bitrev_permute(out[k, c], log_n), exp)
