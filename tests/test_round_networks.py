"""The algebra behind the radix-16 round networks of
era-boojum-cuda_b200/csrc/ntt_pass.cuh (cstage / cnet), in exact arithmetic
mod p.

The kernels compute an inverse (DIF) round's network with Cooley-Tukey
butterflies: stage qq multiplies by w_{2^(qq+1)}^(-+j) (ct_tw_exp in
csrc/tables.cuh) before the sum and difference.  That is only correct because
the stage-by-stage inverse of the forward (DIT) network -- sum-then-twiddle
butterflies with the bit-reversed small twiddles T[u] (small_tw_exp) -- equals
the in-place Cooley-Tukey iteration on the same registers.  These tests pin
that identity for every round width V = 1..4 and both directions, and pin the
two twiddle-exponent helpers against the roots of unity they stand for.
"""
import random
import re
import os

import pytest

HERE = os.path.dirname(os.path.abspath(__file__))
TABLES = os.path.join(HERE, "..", "era-boojum-cuda_b200", "csrc", "tables.cuh")
P = (1 << 64) - (1 << 32) + 1


def _fwd_exponents():
    src = open(TABLES).read()
    m = re.search(r"constexpr int fwd\[8\] = \{([^}]*)\}", src)
    return [int(v) for v in m.group(1).split(",")]


FWD = _fwd_exponents()


def small_tw_exp(inv, u):
    return (192 - FWD[u]) % 192 if inv else FWD[u]


def ct_tw_exp(inv, qq, j):
    e = (156 * (j << (3 - qq))) % 192
    return (192 - e) % 192 if inv else e


def w(e):
    return pow(2, e, P)


def gs_network(x, v, inv):
    """Sum-then-twiddle butterflies, bottom bit first: the stage-by-stage inverse of the DIT network."""
    x = list(x)
    for qq in range(v):
        for j0 in range(1 << v):
            if j0 & (1 << qq):
                continue
            e = small_tw_exp(inv, j0 >> (qq + 1))
            a, b = x[j0], x[j0 | (1 << qq)]
            x[j0], x[j0 | (1 << qq)] = (a + b) % P, (a - b) * w(e) % P
    return x


def ct_network(x, v, inv, dif):
    """Twiddle-then-sum butterflies, as cstage computes them."""
    x = list(x)
    stages = range(v) if dif else reversed(range(v))
    for qq in stages:
        for j0 in range(1 << v):
            if j0 & (1 << qq):
                continue
            e = ct_tw_exp(inv, qq, j0 & ((1 << qq) - 1)) if dif else small_tw_exp(inv, j0 >> (qq + 1))
            a, b = x[j0], x[j0 | (1 << qq)] * w(e) % P
            x[j0], x[j0 | (1 << qq)] = (a + b) % P, (a - b) % P
    return x


def brev(i, bits):
    return int(format(i, f"0{bits}b")[::-1], 2) if bits else 0


def test_small_twiddles_are_bit_reversed_16th_roots():
    w16 = pow(7, (P - 1) >> 4, P)
    assert w16 == w(156)
    for u in range(8):
        assert w(small_tw_exp(False, u)) == pow(w16, brev(u, 3), P)
        assert w(small_tw_exp(True, u)) * w(small_tw_exp(False, u)) % P == 1


@pytest.mark.parametrize("v", [1, 2, 3, 4])
@pytest.mark.parametrize("inv", [False, True])
def test_dif_network_equals_cooley_tukey(v, inv):
    rnd = random.Random(100 * v + inv)
    for _ in range(100):
        x = [rnd.randrange(P) for _ in range(1 << v)]
        assert ct_network(x, v, inv, dif=True) == gs_network(x, v, inv)


@pytest.mark.parametrize("v", [1, 2, 3, 4])
@pytest.mark.parametrize("inv", [False, True])
def test_dif_network_inverts_dit_network(v, inv):
    # DIF (this direction's table) after DIT (the other table) is 2^v times the identity
    rnd = random.Random(7 + 10 * v + inv)
    for _ in range(50):
        x = [rnd.randrange(P) for _ in range(1 << v)]
        y = ct_network(x, v, not inv, dif=False)
        assert ct_network(y, v, inv, dif=True) == [(xi << v) % P for xi in x]


@pytest.mark.parametrize("v", [1, 2, 3, 4])
def test_dit_network_is_dft_with_bit_reversed_output(v):
    n = 1 << v
    root = pow(7, (P - 1) >> v, P)
    rnd = random.Random(v)
    x = [rnd.randrange(P) for _ in range(n)]
    y = ct_network(x, v, False, dif=False)
    for k in range(n):
        f = brev(k, v)
        assert y[k] == sum(x[j] * pow(root, j * f, P) for j in range(n)) % P
