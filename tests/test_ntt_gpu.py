"""GPU parity of the plain batched NTT against the CPU oracle and the reference kernels.

The matrix follows the reference's own tests (src/ntt.rs:391-663): for each
log_n, every column sits at offset n inside a stride of 2 * n_max, inputs are
raw u64 words (src/ntt.rs:424), and all four variants run -- natural->bitrev
and bitrev->natural, each in place and out of place -- for forward, inverse,
forward-LDE (log_extension_degree 3, coset 3) and inverse-LDE.  Results must
be bit-exact (canonical) and the words outside each column's window must be
left untouched.
"""
import numpy as np
import pytest

import oracle
from conftest import raw_u64, to_dev, to_host, uniform

pytestmark = pytest.mark.gpu

SENTINEL = np.uint64(0xDEADBEEFCAFEF00D)


def _bitrev_chunks(a: np.ndarray, log_n: int) -> np.ndarray:
    n = 1 << log_n
    return oracle.bitrev_permute(a.reshape(-1, n), log_n).reshape(-1)


def _window(a: np.ndarray, num: int, stride: int, off: int, n: int) -> np.ndarray:
    return a.reshape(num, stride)[:, off:off + n]


def _outside(a: np.ndarray, num: int, stride: int, off: int, n: int) -> np.ndarray:
    m = a.reshape(num, stride).copy()
    m[:, off:off + n] = 0
    return m


def correctness(log_n_range, inverse, log_ext, coset, num_ntts, seed=0):
    import bc_ntt
    import torch

    rng = np.random.default_rng(seed + 1000 * log_ext + 17 * num_ntts + int(inverse))
    n_max = 1 << (log_n_range[-1])
    stride = 2 * n_max
    io = raw_u64(rng, num_ntts * stride)
    for log_n in log_n_range:
        n = 1 << log_n
        off = n
        io_brev = _bitrev_chunks(io, log_n)
        x = np.ascontiguousarray(_window(io, num_ntts, stride, off, n)).reshape(-1)
        xb = np.ascontiguousarray(_window(io_brev, num_ntts, stride, off, n)).reshape(-1)
        exp_n2b = oracle.batch_ntt(x, log_n, num_ntts, n, n, False, inverse, log_ext, coset, threads=8)
        exp_b2n = oracle.batch_ntt(xb, log_n, num_ntts, n, n, True, inverse, log_ext, coset, threads=8)
        for bitrev, src, exp in ((False, io, exp_n2b), (True, io_brev, exp_b2n)):
            exp = exp.reshape(num_ntts, n)
            # in place
            d = to_dev(src)
            bc_ntt.batch_ntt_in_place(d, log_n, num_ntts, off, stride, bitrev, inverse, log_ext, coset)
            got = to_host(d)
            np.testing.assert_array_equal(_window(got, num_ntts, stride, off, n), exp,
                                          err_msg=f"in-place log_n={log_n} bitrev={bitrev}")
            np.testing.assert_array_equal(_outside(got, num_ntts, stride, off, n),
                                          _outside(src, num_ntts, stride, off, n))
            # out of place, output prefilled with a sentinel
            d_in = to_dev(src)
            d_out = to_dev(np.full(num_ntts * stride, SENTINEL, dtype=np.uint64))
            bc_ntt.batch_ntt_out_of_place(d_in, d_out, log_n, num_ntts, off, off, stride, stride, bitrev, inverse,
                                          log_ext, coset)
            got = to_host(d_out)
            np.testing.assert_array_equal(_window(got, num_ntts, stride, off, n), exp,
                                          err_msg=f"out-of-place log_n={log_n} bitrev={bitrev}")
            outside = _outside(got, num_ntts, stride, off, n)
            mask = np.ones_like(outside, dtype=bool)
            mask[:, off:off + n] = False
            assert np.all(outside[mask] == SENTINEL), f"write outside window, log_n={log_n}"
            np.testing.assert_array_equal(to_host(d_in), src)  # input untouched
        torch.cuda.synchronize()


# src/ntt.rs:613-663: NTTS_PER_BLOCK = 8, so 2 * 8 + 3 columns exercise a partial chunk.
def test_fwd(gpu_ctx):
    correctness(list(range(1, 17)), False, 0, 0, 2 * 8 + 3)


def test_lde_fwd(gpu_ctx):
    correctness(list(range(1, 17)), False, 3, 3, 3)


def test_inv(gpu_ctx):
    correctness(list(range(1, 17)), True, 0, 0, 1)


def test_lde_inv(gpu_ctx):
    correctness(list(range(1, 17)), True, 3, 3, 3)


def test_fwd_large(gpu_ctx):
    correctness(list(range(17, 25)), False, 0, 0, 3)


def test_inv_large(gpu_ctx):
    correctness(list(range(17, 25)), True, 0, 0, 1)


def test_lde_fwd_large(gpu_ctx):
    correctness(list(range(17, 22)), False, 3, 3, 3)


def test_lde_inv_large(gpu_ctx):
    correctness(list(range(17, 22)), True, 3, 3, 3)


@pytest.mark.parametrize("log_n", [25, 26])
def test_beyond_reference_limit(gpu_ctx, log_n):
    """Sizes the reference rejects (log_n + e > 24): one column each direction."""
    import bc_ntt

    rng = np.random.default_rng(log_n)
    n = 1 << log_n
    x = uniform(rng, n)
    for bitrev, inverse, e, k in ((False, False, 2, 3), (True, True, 0, 0)):
        exp = oracle.batch_ntt(x, log_n, 1, n, n, bitrev, inverse, e, k)
        d = to_dev(x)
        out = to_dev(np.zeros(n, dtype=np.uint64))
        bc_ntt.batch_ntt_internal(d.data_ptr(), out.data_ptr(), log_n, 1, n, n, bitrev, inverse, e, k)
        np.testing.assert_array_equal(to_host(out), exp)


@pytest.mark.parametrize("fill", [0, 1, 2**64 - 1, 0xFFFFFFFF00000001, 0xFFFFFFFF00000000, 0xFFFFFFFF])
def test_extreme_words(gpu_ctx, fill):
    """Constant and near-p inputs, including every non-canonical word class."""
    import bc_ntt

    for log_n in (3, 11, 16, 20):
        n = 1 << log_n
        x = np.full(4 * n, fill, dtype=np.uint64)
        x[1::7] = np.uint64(2**64 - 1)
        for bitrev in (False, True):
            for inverse, e, k in ((False, 0, 0), (True, 0, 0), (False, 3, 5), (True, 2, 1)):
                exp = oracle.batch_ntt(x, log_n, 4, n, n, bitrev, inverse, e, k)
                d = to_dev(x)
                bc_ntt.batch_ntt_in_place(d, log_n, 4, 0, n, bitrev, inverse, e, k)
                np.testing.assert_array_equal(to_host(d), exp, err_msg=f"log_n={log_n} {bitrev} {inverse}")


def test_odd_stride_unaligned(gpu_ctx):
    """Odd strides and offsets force the 8-byte access path."""
    import bc_ntt

    rng = np.random.default_rng(5)
    for log_n in (5, 13, 18):
        n = 1 << log_n
        stride = n + 3
        num = 5
        src = raw_u64(rng, num * stride + 1)
        x = np.ascontiguousarray(src[1:].reshape(num, stride)[:, :n]).reshape(-1)
        for bitrev, inverse in ((False, False), (True, True)):
            exp = oracle.batch_ntt(x, log_n, num, n, n, bitrev, inverse, 1, 1).reshape(num, n)
            d_in = to_dev(src)
            d_out = to_dev(np.zeros(num * stride + 1, dtype=np.uint64))
            bc_ntt.batch_ntt_out_of_place(d_in, d_out, log_n, num, 1, 1, stride, stride, bitrev, inverse, 1, 1)
            got = to_host(d_out)[1:].reshape(num, stride)[:, :n]
            np.testing.assert_array_equal(got, exp)


def test_roundtrip_large(gpu_ctx):
    """Size-independent property at the LDE benchmark size: iNTT(NTT(x)) == x for 128 x 2^22 columns."""
    import bc_ntt
    import torch

    log_n, num = 22, 128
    n = 1 << log_n
    g = torch.Generator(device="cuda").manual_seed(7)
    x = torch.randint(-(2**63), 2**63 - 1, (num * n,), device="cuda", dtype=torch.int64, generator=g)
    y = torch.empty_like(x)
    z = torch.empty_like(x)
    ptr = lambda t: t.data_ptr()  # noqa: E731
    bc_ntt.batch_ntt_internal(ptr(x), ptr(y), log_n, num, n, n, False, False, 2, 1)
    bc_ntt.batch_ntt_internal(ptr(y), ptr(z), log_n, num, n, n, True, True, 2, 1)
    # canonical x on the device: unsigned words >= p are the signed range [-(2^32 - 1), -1]
    xc = torch.where((x < 0) & (x >= -(2**32 - 1)), x + (2**32 - 1), x)
    assert torch.equal(z, xc)


def test_reference_kernels_parity(gpu_ctx):
    """Against the reference's own kernels (compiled for sm_100a), log_n 1..24, canonicalised."""
    import os

    import bc_ntt
    import torch

    if not os.path.exists(oracle.REF_LIB):
        pytest.skip("oracle/_ref/libref_ntt.so not built")
    ref = oracle.RefKernels()
    rng = np.random.default_rng(11)
    stream = torch.cuda.current_stream().cuda_stream
    for log_n in range(1, 25):
        n = 1 << log_n
        num = 3 if log_n <= 22 else 1
        x = raw_u64(rng, num * n)
        cases = [(False, False, 0, 0), (True, False, 0, 0), (False, True, 0, 0), (True, True, 0, 0)]
        if log_n <= 21:
            cases += [(False, False, 3, 3), (True, False, 3, 5), (False, True, 2, 1), (True, True, 3, 3)]
        for bitrev, inverse, e, k in cases:
            d_in = to_dev(x)
            d_ref = to_dev(np.zeros(num * n, dtype=np.uint64))
            d_new = to_dev(np.zeros(num * n, dtype=np.uint64))
            ref.batch_ntt(d_in.data_ptr(), d_ref.data_ptr(), log_n, num, n, n, bitrev, inverse, e, k, stream)
            bc_ntt.batch_ntt_internal(d_in.data_ptr(), d_new.data_ptr(), log_n, num, n, n, bitrev, inverse, e, k)
            torch.cuda.synchronize()
            np.testing.assert_array_equal(to_host(d_new), oracle.canon(to_host(d_ref)),
                                          err_msg=f"log_n={log_n} bitrev={bitrev} inv={inverse} e={e} k={k}")
