"""The Goldilocks field arithmetic's inline PTX (era-boojum-cuda_b200/csrc/gl.cuh),
executed on the CPU by tests/ptx_model.py and compared with exact arithmetic
mod p = 2^64 - 2^32 + 1.

Each asm block is driven with the operands the C++ around it computes (the
split of x << s into 32-bit words for mul_pow2, for example), over the edge
values of the carry chains (0, 1, EPS, 2^32, p - 1, p, p + 1, 2^63, 2^64 - 1
and words that are all ones or all zeros) and seeded random inputs.  A block
added to the header without a driver here fails `test_every_block_is_driven`.
The same functions are checked on the GPU, through the transforms, by the
parity tests.
"""
import os
import random

import pytest

import ptx_model as pm

HERE = os.path.dirname(os.path.abspath(__file__))
GL = os.path.join(HERE, "..", "era-boojum-cuda_b200", "csrc", "gl.cuh")
P = (1 << 64) - (1 << 32) + 1
EPS = (1 << 32) - 1
M32 = (1 << 32) - 1
M64 = (1 << 64) - 1

BLOCKS = {k: pm.compile_block(v) for k, v in pm.asm_blocks(GL).items()}

EDGE = sorted(
    {0, 1, 2, EPS - 1, EPS, 1 << 32, (1 << 32) + 1, P - 2, P - 1, P, P + 1, (1 << 63) - 1, 1 << 63, M64 - 1, M64,
     M64 - EPS, 0xFFFFFFFF00000000, 0x00000000FFFFFFFF, 0x8000000080000000, 0x7FFFFFFF7FFFFFFF}
)


def samples(n=1500, seed=7):
    rnd = random.Random(seed)
    xs = list(EDGE)
    xs += [rnd.getrandbits(64) for _ in range(n)]
    # sparse patterns: a run of ones at a random place, the carry chains' hard cases
    for _ in range(n // 3):
        w = rnd.randint(1, 64)
        xs.append((((1 << w) - 1) << rnd.randint(0, 64 - w)) & M64)
    return xs


def pairs(n=1500, seed=11):
    rnd = random.Random(seed)
    out = [(a, b) for a in EDGE for b in EDGE]
    out += [(rnd.getrandbits(64), rnd.getrandbits(64)) for _ in range(n)]
    return out


DRIVEN = set()


def block(name, k=0):
    DRIVEN.add((name, k))
    return BLOCKS[(name, k)]


def test_add_any_operands():
    b = block("add")
    for x, y in pairs():
        r = pm.run(b, [x, y])
        assert r <= M64 and r % P == (x + y) % P, (hex(x), hex(y), hex(r))


def test_sub_any_operands():
    b = block("sub")
    for x, y in pairs():
        r = pm.run(b, [x, y])
        assert r <= M64 and r % P == (x - y) % P, (hex(x), hex(y), hex(r))


def test_add_bc_sub_bc_canonical_second_operand():
    ba, bs = block("add_bc"), block("sub_bc")
    for x, y in pairs():
        y %= P
        ra, rs = pm.run(ba, [x, y]), pm.run(bs, [x, y])
        assert ra % P == (x + y) % P, (hex(x), hex(y), hex(ra))
        assert rs % P == (x - y) % P, (hex(x), hex(y), hex(rs))


@pytest.mark.parametrize("name", ["reduce128", "reduce128_chain", "reduce128_canon"])
def test_reduce128(name):
    b = block(name)
    for lo, hi in pairs(seed=13):
        r = pm.run(b, [lo, hi])
        want = (lo + (hi << 64)) % P
        if name == "reduce128_canon":
            assert r == want, (hex(lo), hex(hi), hex(r))
        else:
            assert r <= M64 and r % P == want, (hex(lo), hex(hi), hex(r))


def test_mul128_chain_is_the_full_product():
    b = block("mul128_chain")
    for x, y in pairs(seed=17):
        lo, hi = pm.run(b, [x, y], outputs=2)
        assert lo + (hi << 64) == x * y, (hex(x), hex(y))


@pytest.mark.parametrize("canon", [True, False])
def test_add_h_eps(canon):
    # add_h_eps<CANON>(lo, h) is called by mul_pow2<E < 32> with lo = x << E, h = x >> (64 - E)
    b = block("add_h_eps", 0 if canon else 1)
    for x in samples():
        for e in (1, 12, 24, 31):
            lo, h = (x << e) & M64, x >> (64 - e)
            r = pm.run(b, [lo, h])
            want = x * pow(2, e, P) % P
            if canon:
                assert r == want, (hex(x), e, hex(r))
            else:
                assert r <= M64 and r % P == want, (hex(x), e, hex(r))


@pytest.mark.parametrize("e", [32, 33, 36, 48, 60, 63])
def test_mul_pow2_32_to_64(e):
    b = block("mul_pow2", 0)
    s = e - 32
    for x in samples():
        xs = (x << s) & M64
        v1, v2, v3 = xs & M32, xs >> 32, (x >> (64 - s)) if s else 0
        r = pm.run(b, [v1, v2, v3])
        # canonical without a separate reduction (mul_pow2<E, true> relies on it)
        assert r == x * pow(2, e, P) % P, (hex(x), e, hex(r))


@pytest.mark.parametrize("e", [64, 65, 72, 84, 95])
def test_mul_pow2_64_to_96(e):
    b = block("mul_pow2", 1)
    s = e - 64
    for x in samples():
        y0 = (x << s) & M32
        t, big_y = y0 * EPS, x >> (32 - s)
        r = pm.run(b, [t, big_y])
        assert r == x * pow(2, e, P) % P, (hex(x), e, hex(r))


def test_every_block_is_driven():
    # runs last in this file: every asm block of the header has a driver above
    missing = set(BLOCKS) - DRIVEN
    assert not missing, f"asm blocks without a model test: {sorted(missing)}"
