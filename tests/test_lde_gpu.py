"""GPU parity of the coset LDE (plain composition and fused kernels).

The LDE the reference's callers compose (src/ntt.rs:179-191 called as in
benches/ntt.rs:110-116): inverse b2n, then one forward n2b per coset with
(log_extension_degree = log2 B, coset_index = k).  Checked bit-exact against
the CPU oracle (gl_oracle_lde), against that composition run on the
reference's own kernels, and -- at the 128 x 2^22 benchmark size -- fused
against plain on the device.
"""
import os

import numpy as np
import pytest

import oracle
from conftest import raw_u64, to_dev, to_host, uniform

pytestmark = pytest.mark.gpu


def run_lde(x, log_n, cols, log_b, fused, layout="coset", stride_in=None):
    import bc_ntt

    n, B = 1 << log_n, 1 << log_b
    stride_in = stride_in or n
    if layout == "coset":
        stride_out, coset_stride, size = n, cols * n, B * cols * n
    else:  # column-major: column j holds its B cosets back to back
        stride_out, coset_stride, size = B * n, n, B * cols * n
    d_in = to_dev(x)
    d_out = to_dev(np.full(size, 0x5A5A5A5A5A5A5A5A, dtype=np.uint64))
    bc_ntt.lde(d_in, d_out, log_n, cols, log_b, stride_in=stride_in, stride_out=stride_out,
               coset_stride=coset_stride, fused=fused)
    got = to_host(d_out)
    np.testing.assert_array_equal(to_host(d_in), x)  # input untouched
    if layout == "coset":
        return got.reshape(B, cols, n)
    return got.reshape(cols, B, n).transpose(1, 0, 2)


@pytest.mark.parametrize("fused", [True, False])
@pytest.mark.parametrize("log_b", [1, 2, 3])
def test_lde_small_sizes(gpu_ctx, fused, log_b):
    rng = np.random.default_rng(10 + log_b)
    cols = 3
    for log_n in range(1, 17):
        n = 1 << log_n
        x = raw_u64(rng, cols * n)
        exp = oracle.lde(x, log_n, cols, n, log_b, threads=4).reshape(1 << log_b, cols, n)
        got = run_lde(x, log_n, cols, log_b, fused)
        np.testing.assert_array_equal(got, exp, err_msg=f"log_n={log_n} B={1 << log_b} fused={fused}")


@pytest.mark.parametrize("log_n,cols,log_b", [(17, 5, 1), (20, 3, 2), (22, 2, 1), (23, 1, 2), (21, 9, 3), (22, 2, 3)])
def test_lde_large_sizes(gpu_ctx, log_n, cols, log_b):
    rng = np.random.default_rng(log_n)
    n = 1 << log_n
    x = uniform(rng, cols * n)
    exp = oracle.lde(x, log_n, cols, n, log_b, threads=8).reshape(1 << log_b, cols, n)
    for fused in (True, False):
        np.testing.assert_array_equal(run_lde(x, log_n, cols, log_b, fused), exp)


def test_lde_large_config_two_whole_columns(gpu_ctx):
    """The large configuration at full size -- 64 columns x 2^23, blowup 4 (16 GiB out) -- with two whole
    columns (every coset, every position) checked against the oracle, through the fused and the plain path."""
    import bc_ntt
    import torch

    log_n, cols, log_b = 23, 64, 2
    n, B = 1 << log_n, 1 << log_b
    g = torch.Generator(device="cuda").manual_seed(2023)
    x = torch.randint(-(2**63), 2**63 - 1, (cols * n,), device="cuda", dtype=torch.int64, generator=g)
    picks = [0, 37]
    xs = np.concatenate([to_host(x[j * n:(j + 1) * n]) for j in picks])
    exp = oracle.lde(xs, log_n, len(picks), n, log_b, threads=2).reshape(B, len(picks), n)
    out = torch.empty(B * cols * n, dtype=torch.int64, device="cuda")
    for fused in (True, False):
        out.fill_(0)
        bc_ntt.lde(x, out, log_n, cols, log_b, fused=fused)
        torch.cuda.synchronize()
        got = to_host(out.view(B, cols, n)[:, picks].contiguous())
        np.testing.assert_array_equal(got, exp, err_msg=f"fused={fused}")
    del x, out


@pytest.mark.parametrize("log_n", [5, 12, 13, 18])
def test_lde_column_major_and_strides(gpu_ctx, log_n):
    rng = np.random.default_rng(77 + log_n)
    n, cols, log_b = 1 << log_n, 6, 2
    stride_in = n + 6
    xs = raw_u64(rng, cols * stride_in)
    x = np.ascontiguousarray(xs.reshape(cols, stride_in)[:, :n]).reshape(-1)
    exp = oracle.lde(x, log_n, cols, n, log_b, threads=4).reshape(1 << log_b, cols, n)
    for fused in (True, False):
        got = run_lde(xs, log_n, cols, log_b, fused, layout="column", stride_in=stride_in)
        np.testing.assert_array_equal(got, exp)


def test_lde_invalid_arguments(gpu_ctx):
    import bc_ntt
    import torch

    x = torch.zeros(1 << 10, dtype=torch.int64, device="cuda")
    out = torch.zeros(1 << 12, dtype=torch.int64, device="cuda")
    with pytest.raises(ValueError):
        bc_ntt.lde(x, out, 10, 1, 0)  # blowup 1 is not an extension
    with pytest.raises(ValueError):
        bc_ntt.lde(x, out, 10, 2, 1, stride_out=1 << 10, coset_stride=1 << 9)  # overlapping blocks
    with pytest.raises(ValueError):
        bc_ntt.lde(x, out, 26, 1, 2)  # log_n + log_blowup > 27


def test_lde_matches_reference_kernels(gpu_ctx):
    """Fused LDE == the reference kernels run as its callers compose an LDE (canonicalised)."""
    import bc_ntt
    import torch

    if not os.path.exists(oracle.REF_LIB):
        pytest.skip("oracle/_ref/libref_ntt.so not built")
    ref = oracle.RefKernels()
    s = torch.cuda.current_stream().cuda_stream
    rng = np.random.default_rng(99)
    for log_n, cols, log_b in ((8, 3, 1), (14, 4, 2), (16, 8, 3), (20, 4, 1), (22, 2, 2)):
        n, B = 1 << log_n, 1 << log_b
        x = raw_u64(rng, cols * n)
        d_in = to_dev(x)
        d_ref = torch.zeros(B * cols * n, dtype=torch.int64, device="cuda")
        coef = torch.zeros(cols * n, dtype=torch.int64, device="cuda")
        ref.batch_ntt(d_in.data_ptr(), coef.data_ptr(), log_n, cols, n, n, True, True, 0, 0, s)
        for k in range(B):
            ref.batch_ntt(coef.data_ptr(), d_ref.data_ptr() + 8 * k * cols * n, log_n, cols, n, n, False, False,
                          log_b, k, s)
        d_new = torch.zeros_like(d_ref)
        bc_ntt.lde(d_in, d_new, log_n, cols, log_b)
        torch.cuda.synchronize()
        np.testing.assert_array_equal(to_host(d_new), oracle.canon(to_host(d_ref)), err_msg=f"log_n={log_n}")


def test_lde_benchmark_size_fused_equals_plain(gpu_ctx):
    """128 x 2^22, blowup 2: fused == plain on the device; two columns against the oracle."""
    import bc_ntt
    import torch

    log_n, cols, log_b = 22, 128, 1
    n, B = 1 << log_n, 2
    g = torch.Generator(device="cuda").manual_seed(3)
    x = torch.randint(-(2**63), 2**63 - 1, (cols * n,), device="cuda", dtype=torch.int64, generator=g)
    a = torch.empty(B * cols * n, dtype=torch.int64, device="cuda")
    bc_ntt.lde(x, a, log_n, cols, log_b, fused=True)
    b = torch.empty_like(a)
    bc_ntt.lde(x, b, log_n, cols, log_b, fused=False)
    torch.cuda.synchronize()
    assert torch.equal(a, b)
    del b
    for c in (0, 127):
        xc = to_host(x[c * n:(c + 1) * n])
        exp = oracle.lde(xc, log_n, 1, n, log_b, threads=2).reshape(B, n)
        for k in range(B):
            np.testing.assert_array_equal(to_host(a[(k * cols + c) * n:(k * cols + c + 1) * n]), exp[k])


@pytest.mark.parametrize("log_n,cols,log_b", [(16, 1029, 1), (20, 37, 1), (13, 4099, 1), (14, 2051, 2), (18, 301, 1),
                                              (21, 100, 1), (19, 203, 2)])
def test_lde_many_column_groups_fused_equals_plain(gpu_ctx, log_n, cols, log_b):
    """Many column groups per top-window CTA, ragged last group: two-tile pipelining in the short windows
    (the first five shapes), the next tile copied during the last coset's stores (the last two).  Fused ==
    plain on the device, first and last columns against the oracle."""
    import bc_ntt
    import torch

    n, B = 1 << log_n, 1 << log_b
    g = torch.Generator(device="cuda").manual_seed(log_n + cols)
    x = torch.randint(-(2**63), 2**63 - 1, (cols * n,), device="cuda", dtype=torch.int64, generator=g)
    a = torch.empty(B * cols * n, dtype=torch.int64, device="cuda")
    bc_ntt.lde(x, a, log_n, cols, log_b, fused=True)
    b = torch.empty_like(a)
    bc_ntt.lde(x, b, log_n, cols, log_b, fused=False)
    torch.cuda.synchronize()
    assert torch.equal(a, b)
    for c in (0, cols - 1):
        xc = to_host(x[c * n:(c + 1) * n])
        exp = oracle.lde(xc, log_n, 1, n, log_b, threads=2).reshape(B, n)
        for k in range(B):
            np.testing.assert_array_equal(to_host(a[(k * cols + c) * n:(k * cols + c + 1) * n]), exp[k])


@pytest.mark.parametrize("pinned", [False, True])
def test_lde_host_pipeline_matches_device(gpu_ctx, pinned):
    """bc_lde_host (host in, host out, chunked through a device workspace) == bc_lde_fused on the device."""
    import bc_ntt
    import torch

    rng = np.random.default_rng(31)
    for log_n, cols, log_b, chunk in ((16, 10, 1, 3), (12, 7, 3, 1), (20, 5, 2, 0)):
        n, B = 1 << log_n, 1 << log_b
        x = raw_u64(rng, cols * n)
        hx = torch.from_numpy(x.view(np.int64))
        hout = torch.zeros(B * cols * n, dtype=torch.int64)
        if pinned:
            hx, hout = hx.pin_memory(), hout.pin_memory()
        ws = torch.empty(3 * max(chunk, 2) * n * (1 + B), dtype=torch.int64, device="cuda")
        bc_ntt.lde_host(hx, hout, log_n, cols, log_b, ws, max_chunk_cols=chunk)
        # waiting on the caller's stream alone must be enough for the host output to be complete
        torch.cuda.current_stream().synchronize()
        ref = torch.empty(B * cols * n, dtype=torch.int64, device="cuda")
        bc_ntt.lde(to_dev(x), ref, log_n, cols, log_b)
        torch.cuda.synchronize()
        np.testing.assert_array_equal(hout.numpy().view(np.uint64), to_host(ref), err_msg=f"log_n={log_n}")
