"""GPU parity of barycentric evaluation (include/bc_barycentric.h) against the oracle and the reference kernels.

The cases follow the reference's tests (src/barycentric.rs:307-683):
coefficients at a base or extension point for log_count 0..19 (bit-reversed),
and batch evaluation of 1, 3, 32, 33 polynomials for log_count 0..16 in the
three kinds, checked against Horner evaluation of the polynomials whose coset
values (computed with this library's batch NTT) are evaluated.  Plus the
reference's own kernels on the same inputs, a point inside the domain, and a
2^22-row batch.
"""
import os

import numpy as np
import pytest

import oracle
from conftest import P, to_dev, to_host, uniform

pytestmark = pytest.mark.gpu

KINDS = (oracle.EVAL_BASE_AT_BASE, oracle.EVAL_BASE_AT_EXT, oracle.EVAL_EXT_AT_EXT)


def _ref():
    if not os.path.exists(oracle.REF_LIB):
        pytest.skip("oracle/_ref/libref_ntt.so not built")
    return oracle.RefKernels()


def _stream():
    import torch

    return torch.cuda.current_stream().cuda_stream


def _zeros(n):
    import torch

    return torch.zeros(max(n, 1), dtype=torch.int64, device="cuda")


def _coeffs(x, log_count, bit_reverse=True):
    import bc_ntt

    ext = isinstance(x, tuple)
    w = 2 if ext else 1
    dx = to_dev(np.array(x if ext else [x], dtype=np.uint64))
    cf = _zeros(w)
    out = _zeros(w << log_count)
    bc_ntt.precompute_lagrange_coeffs(dx, cf, 7, out, bit_reverse, ext=ext)
    return out, to_host(out)


@pytest.mark.parametrize("ext", [False, True])
def test_precompute_reference_case(gpu_ctx, ext):
    """src/barycentric.rs:307-395: log_count 0..19, coset 7, bit-reversed; oracle and reference kernels."""
    ref = _ref()
    rng = np.random.default_rng(20 + ext)
    for log_count in range(0, 20):
        x = tuple(int(v) for v in rng.integers(0, 2**64, 2, dtype=np.uint64)) if ext else int(
            rng.integers(0, 2**64, dtype=np.uint64))
        _, got = _coeffs(x, log_count)
        exp = oracle.lagrange_coeffs(x, 7, log_count, True)
        np.testing.assert_array_equal(got, exp, err_msg=f"log_count={log_count}")
        w = 2 if ext else 1
        dx = to_dev(np.array(x if ext else [x], dtype=np.uint64))
        cf, r = _zeros(w), _zeros(w << log_count)
        ref.barycentric_precompute(ext, dx.data_ptr(), cf.data_ptr(), 7, r.data_ptr(), 1 << log_count, True, _stream())
        np.testing.assert_array_equal(oracle.canon(to_host(r)), exp, err_msg=f"reference log_count={log_count}")


def test_precompute_natural_order_and_point_in_domain(gpu_ctx):
    x = 7 * pow(oracle.root_of_unity(10), 37, P) % P
    for pt in (x, (x, 0)):
        _, got = _coeffs(pt, 10, bit_reverse=False)
        assert not got.any()
    rng = np.random.default_rng(3)
    x = int(uniform(rng, 1)[0])
    _, got = _coeffs(x, 12, bit_reverse=False)
    np.testing.assert_array_equal(got, oracle.lagrange_coeffs(x, 7, 12, False))


def _eval(kind, ys_dev, count, num_polys, coeffs_dev):
    import bc_ntt

    words, nbytes = bc_ntt.get_batch_eval_temp_storage_sizes(kind, count, num_polys)
    assert nbytes == 0
    tmp = _zeros(words)
    evals = _zeros((1 if kind == 0 else 2) * num_polys)
    bc_ntt.batch_eval(kind, ys_dev, count, num_polys, coeffs_dev, tmp, None, evals)
    return to_host(evals)[:(1 if kind == 0 else 2) * num_polys]


@pytest.mark.parametrize("kind", KINDS)
def test_batch_eval_reference_case(gpu_ctx, kind):
    """src/barycentric.rs:397-683: random polynomials, coset values by batch_ntt (n2b, e = 1, k = 0), evaluation
    at a random point == Horner, for 1, 3, 32, 33 polynomials and log_count 0..16; reference kernels beside."""
    import bc_ntt

    ref = _ref()
    rng = np.random.default_rng(30 + kind)
    for num_polys in (1, 3, 32, 33):
        for log_count in range(0, 17):
            count = 1 << log_count
            ext_vals = kind == oracle.EVAL_EXT_AT_EXT
            cols = (2 if ext_vals else 1) * num_polys
            a = uniform(rng, cols * count)
            ys = to_dev(a)
            if log_count > 0:
                bc_ntt.batch_ntt_in_place(ys, log_count, cols, 0, count, False, False, 1, 0)
            x = int(uniform(rng, 1)[0]) if kind == oracle.EVAL_BASE_AT_BASE else tuple(
                int(v) for v in uniform(rng, 2))
            cdev, _ = _coeffs(x, log_count)
            got = _eval(kind, ys, count, num_polys, cdev)
            exp = oracle.poly_eval(a, count, num_polys, x, ext_coeffs=ext_vals)
            if kind == oracle.EVAL_BASE_AT_BASE:
                exp = exp[0::2]
            msg = f"num_polys={num_polys} log_count={log_count}"
            np.testing.assert_array_equal(got, exp, err_msg=msg)
            if log_count in (0, 5, 12, 16):
                r = ref.batch_eval(kind, ys.data_ptr(), count, num_polys, cdev.data_ptr(), _stream())
                np.testing.assert_array_equal(oracle.canon(r), exp, err_msg="reference " + msg)


def test_batch_eval_large(gpu_ctx):
    """2^22 rows x 8 polynomials (256 MiB) at an extension point, against the oracle's dot products."""
    import torch

    rng = np.random.default_rng(44)
    log_count, num_polys = 22, 8
    count = 1 << log_count
    g = torch.Generator(device="cuda").manual_seed(4)
    ys = torch.randint(-(2**63), 2**63 - 1, (num_polys * count,), dtype=torch.int64, device="cuda", generator=g)
    x = tuple(int(v) for v in uniform(rng, 2))
    cdev, coeffs = _coeffs(x, log_count)
    got = _eval(oracle.EVAL_BASE_AT_EXT, ys, count, num_polys, cdev)
    exp = oracle.batch_eval(oracle.EVAL_BASE_AT_EXT, to_host(ys), count, num_polys, coeffs)
    np.testing.assert_array_equal(got, exp)


def test_batch_eval_rejects_short_scratch(gpu_ctx):
    import bc_ntt

    count, num_polys = 1 << 14, 5
    words, _ = bc_ntt.get_batch_eval_temp_storage_sizes(0, count, num_polys)
    with pytest.raises(ValueError):
        bc_ntt.batch_eval(0, _zeros(count * num_polys), count, num_polys, _zeros(count), _zeros(words - 1), None,
                          _zeros(num_polys))
    with pytest.raises(ValueError):
        bc_ntt.get_batch_eval_temp_storage_sizes(0, 3 << 10, 1)  # not a power of two
