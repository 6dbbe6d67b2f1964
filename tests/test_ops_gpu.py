"""GPU parity of the ops beside the NTT (include/bc_ops.h) against the CPU oracle and the reference's kernels.

The cases start from the reference's own tests (src/ops_complex.rs:1366-1670:
2^16 elements, split in two calls at offset n/2; bit reversal of 16 columns x
2^16 rows, in place and out of place) and add the edges its kernels cover:
every log_rows of the naive and the tiled bit-reversal paths, odd row counts,
strided and in-place matrices, exponents that wrap in u32, bit-reversed
indexes, non-canonical bases.  Results must be bit-exact (canonical).
"""
import os

import numpy as np
import pytest

import oracle
from conftest import P, raw_u64, to_dev, to_host, uniform

pytestmark = pytest.mark.gpu


def _ref():
    if not os.path.exists(oracle.REF_LIB):
        pytest.skip("oracle/_ref/libref_ntt.so not built")
    return oracle.RefKernels()


def _stream():
    import torch

    return torch.cuda.current_stream().cuda_stream


def _zeros(n):
    import torch

    return torch.zeros(n, dtype=torch.int64, device="cuda")


@pytest.mark.parametrize("in_place", [False, True])
def test_bit_reverse_reference_case(gpu_ctx, in_place):
    """src/ops_complex.rs:1620-1670: 16 columns x 2^16 rows."""
    import bc_ntt

    rng = np.random.default_rng(3)
    log_rows, cols = 16, 16
    x = uniform(rng, cols << log_rows)
    exp = oracle.bit_reverse(x, log_rows, cols)
    d = to_dev(x)
    if in_place:
        bc_ntt.bit_reverse_in_place(d, log_rows, cols)
        got = to_host(d)
    else:
        out = _zeros(cols << log_rows)
        bc_ntt.bit_reverse(d, out, log_rows, cols)
        got = to_host(out)
        np.testing.assert_array_equal(to_host(d), x)
    np.testing.assert_array_equal(got, exp)


@pytest.mark.parametrize("gap", [5, 6])
def test_bit_reverse_every_size_strided(gpu_ctx, gap):
    """log_rows 0..23 (swap path below 10, tiles from 10, odd and even), 3 columns in strided matrices whose
    gaps must stay untouched; out of place and in place agree with the oracle.  An odd gap leaves the columns
    8-byte aligned (8-byte tile accesses), an even one 16-byte aligned (16-byte accesses)."""
    import bc_ntt

    rng = np.random.default_rng(4 + gap)
    sentinel = np.uint64(0x5EED5EED5EED5EED)
    for log_rows in range(0, 24):
        rows, cols = 1 << log_rows, 3
        stride = rows + gap
        buf = raw_u64(rng, cols * stride)
        x = np.ascontiguousarray(buf.reshape(cols, stride)[:, :rows]).reshape(-1)
        exp = oracle.bit_reverse(x, log_rows, cols).reshape(cols, rows)
        d_in = to_dev(buf)
        d_out = to_dev(np.full(cols * stride, sentinel, dtype=np.uint64))
        bc_ntt.bit_reverse(d_in, d_out, log_rows, cols, stride, stride)
        got = to_host(d_out).reshape(cols, stride)
        np.testing.assert_array_equal(got[:, :rows], exp, err_msg=f"log_rows={log_rows}")
        assert np.all(got[:, rows:] == sentinel), f"write outside the columns, log_rows={log_rows}"
        bc_ntt.bit_reverse_in_place(d_in, log_rows, cols, stride)
        got = to_host(d_in).reshape(cols, stride)
        np.testing.assert_array_equal(got[:, :rows], exp, err_msg=f"in place, log_rows={log_rows}")
        np.testing.assert_array_equal(got[:, rows:], buf.reshape(cols, stride)[:, rows:])


def test_bit_reverse_vs_reference_kernels(gpu_ctx):
    import bc_ntt

    ref = _ref()
    rng = np.random.default_rng(5)
    for log_rows in (1, 4, 9, 10, 11, 15, 20, 23):
        rows, cols = 1 << log_rows, 2
        x = raw_u64(rng, cols * rows)
        d = to_dev(x)
        a, b = _zeros(cols * rows), _zeros(cols * rows)
        ref.bit_reverse(d.data_ptr(), rows, a.data_ptr(), rows, log_rows, cols, _stream())
        bc_ntt.bit_reverse(d, b, log_rows, cols)
        np.testing.assert_array_equal(to_host(b), to_host(a), err_msg=f"log_rows={log_rows}")


def test_bit_reverse_involution_large(gpu_ctx):
    """Size-independent property at 2 columns x 2^27 rows (2 GiB): applying it twice is the identity."""
    import bc_ntt
    import torch

    log_rows, cols = 27, 2
    g = torch.Generator(device="cuda").manual_seed(9)
    x = torch.randint(-(2**63), 2**63 - 1, (cols << log_rows,), dtype=torch.int64, device="cuda", generator=g)
    y = x.clone()
    bc_ntt.bit_reverse_in_place(y, log_rows, cols)
    assert not torch.equal(x, y)
    idx = torch.tensor([1, 2, 3, 12345, (1 << log_rows) - 2], device="cuda")
    rev = torch.tensor([int(format(int(i), f"0{log_rows}b")[::-1], 2) for i in idx.tolist()], device="cuda")
    assert torch.equal(y[rev], x[idx])
    bc_ntt.bit_reverse_in_place(y, log_rows, cols)
    assert torch.equal(x, y)


@pytest.mark.parametrize("of_g", [False, True])
@pytest.mark.parametrize("inverse", [False, True])
def test_powers_of_reference_case(gpu_ctx, of_g, inverse):
    """src/ops_complex.rs:1366-1437: log_degree 16, two halves."""
    import bc_ntt

    n = 1 << 16
    d = _zeros(n)
    fn = bc_ntt.get_powers_of_g if of_g else bc_ntt.get_powers_of_w
    fn(16, 0, inverse, False, d[: n // 2])
    fn(16, n // 2, inverse, False, d[n // 2:])
    np.testing.assert_array_equal(to_host(d), oracle.powers_of(16, 0, inverse, False, of_g, n))


def test_powers_of_edges_and_reference_kernels(gpu_ctx):
    import bc_ntt

    ref = _ref()
    cases = [(0, 0, 5), (1, 0, 2), (12, 77, 4096 + 13), (24, 0, 1 << 20), (24, 2**32 - 300, 1000), (20, 5, 3)]
    for log_degree, offset, count in cases:
        for of_g in (False, True):
            for inverse in (False, True):
                for bitrev in (False, True):
                    exp = oracle.powers_of(log_degree, offset, inverse, bitrev, of_g, count)
                    d = _zeros(count)
                    (bc_ntt.get_powers_of_g if of_g else bc_ntt.get_powers_of_w)(log_degree, offset, inverse, bitrev,
                                                                                   d)
                    msg = f"log_degree={log_degree} offset={offset} g={of_g} inv={inverse} brev={bitrev}"
                    np.testing.assert_array_equal(to_host(d), exp, err_msg=msg)
                    r = _zeros(count)
                    ref.get_powers_of(log_degree, offset, inverse, bitrev, of_g, r.data_ptr(), count, _stream())
                    np.testing.assert_array_equal(oracle.canon(to_host(r)), exp, err_msg="reference " + msg)
    with pytest.raises(ValueError):
        bc_ntt.get_powers_of_w(25, 0, False, False, _zeros(4))


@pytest.mark.parametrize("by_ref", [False, True])
def test_powers_by_reference_case(gpu_ctx, by_ref):
    """src/ops_complex.rs:1438-1533: base 42 over 2^16 (two halves) and 42 + 42x over 2 x 2^16."""
    import bc_ntt

    n = 1 << 16
    d = _zeros(n)
    base = to_dev(np.array([42], dtype=np.uint64))
    for half, off in ((d[: n // 2], 0), (d[n // 2:], n // 2)):
        if by_ref:
            bc_ntt.get_powers_by_ref(base, off, False, half)
        else:
            bc_ntt.get_powers_by_val(42, off, False, half)
    np.testing.assert_array_equal(to_host(d), oracle.powers_by(42, 0, False, n))
    ebase = to_dev(np.array([42, 42], dtype=np.uint64))
    for off in (0, n):
        e = _zeros(2 * n)
        if by_ref:
            bc_ntt.get_powers_by_ref(ebase, off, False, e, ext=True)
        else:
            bc_ntt.get_powers_by_val((42, 42), off, False, e)
        exp = oracle.powers_by((42, 42), off, False, n)
        np.testing.assert_array_equal(to_host(e), exp, err_msg=f"extension offset={off}")


def test_powers_by_edges_and_reference_kernels(gpu_ctx):
    """Wrapping u32 exponents (inside one thread's run), 32-bit reversed indexes, non-canonical bases,
    ragged counts; against the oracle and the reference kernels."""
    import bc_ntt

    ref = _ref()
    rng = np.random.default_rng(6)
    b0, b1 = (int(v) for v in raw_u64(rng, 2))
    for base in (42, P + 3, b0, (b0, b1), (P, P + 1)):
        for offset, count, bitrev in ((0, 5000, False), (2**32 - 3000, 7001, False), (17, 4099, True),
                                      (2**32 - 1, 300, True), (123456, 1, False)):
            ext = isinstance(base, tuple)
            exp = oracle.powers_by(base, offset, bitrev, count)
            d = _zeros((2 if ext else 1) * count)
            bc_ntt.get_powers_by_val(base, offset, bitrev, d)
            msg = f"base={base} offset={offset} count={count} brev={bitrev}"
            np.testing.assert_array_equal(to_host(d), exp, err_msg=msg)
            r = _zeros((2 if ext else 1) * count)
            ref.get_powers_by_val(base, offset, bitrev, r.data_ptr(), count, _stream())
            np.testing.assert_array_equal(oracle.canon(to_host(r)), exp, err_msg="reference " + msg)


@pytest.mark.parametrize("in_place", [False, True])
@pytest.mark.parametrize("inverse", [False, True])
def test_omega_shift_reference_case(gpu_ctx, in_place, inverse):
    """src/ops_complex.rs:1534-1618: log_degree 16, shift 42, two halves."""
    import bc_ntt

    rng = np.random.default_rng(7)
    n = 1 << 16
    x = uniform(rng, n)
    exp = oracle.omega_shift(x, 16, 0, inverse, 42)
    d = to_dev(x)
    if in_place:
        bc_ntt.omega_shift_in_place(d[: n // 2], 16, 0, inverse, 42)
        bc_ntt.omega_shift_in_place(d[n // 2:], 16, n // 2, inverse, 42)
        got = to_host(d)
    else:
        out = _zeros(n)
        bc_ntt.omega_shift(d[: n // 2], 16, 0, inverse, 42, out[: n // 2])
        bc_ntt.omega_shift(d[n // 2:], 16, n // 2, inverse, 42, out[n // 2:])
        got = to_host(out)
    np.testing.assert_array_equal(got, exp)


def test_omega_shift_edges_and_reference_kernels(gpu_ctx):
    import bc_ntt

    ref = _ref()
    rng = np.random.default_rng(8)
    for log_degree, offset, shift, count in ((0, 0, 1, 100), (24, 3, 2**31 + 7, 5000), (10, 2**32 - 1000, 3, 4097),
                                             (20, 2**31, 2**30 + 3, 1 << 20), (16, 0, 0, 33)):
        x = raw_u64(rng, count)
        for inverse in (False, True):
            exp = oracle.omega_shift(x, log_degree, offset, inverse, shift)
            d, out = to_dev(x), _zeros(count)
            bc_ntt.omega_shift(d, log_degree, offset, inverse, shift, out)
            msg = f"log_degree={log_degree} offset={offset} shift={shift} inv={inverse}"
            np.testing.assert_array_equal(to_host(out), exp, err_msg=msg)
            r = _zeros(count)
            ref.omega_shift(d.data_ptr(), log_degree, offset, inverse, shift, r.data_ptr(), count, _stream())
            np.testing.assert_array_equal(oracle.canon(to_host(r)), exp, err_msg="reference " + msg)
