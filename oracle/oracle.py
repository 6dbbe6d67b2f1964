"""ctypes wrapper of the CPU oracle (liboracle.so) and of the compiled reference kernels.

TEST INFRASTRUCTURE ONLY: imported by tests/, __graft_entry__.smoke() and the
cpu_baseline / reference legs of bench.py -- never by the product library.

* ``batch_ntt`` / ``lde``: CPU restatement (gl_oracle.c) of src/ntt.rs:179-369
  semantics, numpy uint64 arrays in and out.
* ``bit_reverse`` / ``powers_of`` / ``powers_by`` / ``omega_shift``: CPU
  restatements (gl_oracle.c) of the ops in src/ops_complex.rs;
  ``lagrange_coeffs`` / ``batch_eval`` / ``poly_eval``: barycentric evaluation
  (src/barycentric.rs) and direct polynomial evaluation.
* ``RefKernels``: the reference's own CUDA kernels (native/ntt.cu,
  native/context.cu, native/ops_complex.cu, native/barycentric.cu) built into
  oracle/_ref/libref_ntt.so by
  ``make -C oracle ref``, driven by ref_glue.cu's restatement of
  Context::create and batch_ntt_internal.
"""
from __future__ import annotations

import ctypes
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ORACLE_LIB = os.path.join(HERE, "liboracle.so")
REF_LIB = os.path.join(HERE, "_ref", "libref_ntt.so")
P = 0xFFFFFFFF00000001

_u32, _u64, _i32, _vp = ctypes.c_uint32, ctypes.c_uint64, ctypes.c_int, ctypes.c_void_p
_lib = None


def lib():
    global _lib
    if _lib is None:
        L = ctypes.CDLL(ORACLE_LIB)
        L.gl_oracle_batch_ntt.argtypes = [_vp, _vp, _u32, _u32, _u64, _u64, _i32, _i32, _u32, _u32, _i32]
        L.gl_oracle_batch_ntt.restype = _i32
        L.gl_oracle_lde.argtypes = [_vp, _vp, _u32, _u32, _u64, _u64, _u64, _u32, _i32]
        L.gl_oracle_lde.restype = _i32
        L.gl_oracle_dft_naive.argtypes = [_vp, _vp, _u32, _i32]
        L.gl_oracle_dft_naive.restype = None
        for f in ("gl_oracle_root_of_unity",):
            getattr(L, f).argtypes = [_u32]
            getattr(L, f).restype = _u64
        L.gl_oracle_coset.argtypes = [_u32, _u32, _u32]
        L.gl_oracle_coset.restype = _u64
        L.gl_oracle_mul.argtypes = [_u64, _u64]
        L.gl_oracle_mul.restype = _u64
        L.gl_oracle_pow.argtypes = [_u64, _u64]
        L.gl_oracle_pow.restype = _u64
        L.gl_oracle_bit_reverse.argtypes = [_vp, _u64, _vp, _u64, _u32, _u32]
        L.gl_oracle_bit_reverse.restype = None
        L.gl_oracle_powers_of.argtypes = [_u32, _u32, _i32, _i32, _i32, _vp, _u32]
        L.gl_oracle_powers_of.restype = None
        L.gl_oracle_powers_by.argtypes = [_u64, _u64, _i32, _u32, _i32, _vp, _u32]
        L.gl_oracle_powers_by.restype = None
        L.gl_oracle_omega_shift.argtypes = [_vp, _u32, _u32, _i32, _u32, _vp, _u32]
        L.gl_oracle_omega_shift.restype = None
        L.gl_oracle_lagrange_coeffs.argtypes = [_u64, _u64, _i32, _u64, _u32, _i32, _vp]
        L.gl_oracle_lagrange_coeffs.restype = None
        L.gl_oracle_batch_eval.argtypes = [_i32, _vp, _u32, _u32, _vp, _vp]
        L.gl_oracle_batch_eval.restype = None
        L.gl_oracle_poly_eval.argtypes = [_i32, _vp, _u32, _u32, _u64, _u64, _vp]
        L.gl_oracle_poly_eval.restype = None
        _lib = L
    return _lib


def _p(a: np.ndarray):
    assert a.dtype == np.uint64 and a.flags["C_CONTIGUOUS"]
    return a.ctypes.data_as(_vp)


def batch_ntt(inputs: np.ndarray, log_n: int, num_ntts: int, stride_in: int, stride_out: int,
              bitrev_inputs: bool, inverse: bool, log_ext: int = 0, coset_idx: int = 0,
              out: np.ndarray | None = None, threads: int = 1) -> np.ndarray:
    """CPU batched NTT with batch_ntt_internal's argument meaning."""
    if out is None:
        out = np.zeros(max(num_ntts * stride_out, 1), dtype=np.uint64)
    rc = lib().gl_oracle_batch_ntt(_p(inputs), _p(out), log_n, num_ntts, stride_in, stride_out,
                                   int(bitrev_inputs), int(inverse), log_ext, coset_idx, threads)
    if rc != 0:
        raise ValueError("oracle: invalid arguments")
    return out


def lde(evals_bitrev: np.ndarray, log_n: int, num_cols: int, stride_in: int, log_blowup: int,
        threads: int = 1) -> np.ndarray:
    """Coset LDE (bit-reversed evaluations in; 2^log_blowup coset blocks of num_cols x n out, bit-reversed)."""
    n = 1 << log_n
    out = np.zeros((1 << log_blowup) * num_cols * n, dtype=np.uint64)
    rc = lib().gl_oracle_lde(_p(evals_bitrev), _p(out), log_n, num_cols, stride_in, n, num_cols * n,
                             log_blowup, threads)
    if rc != 0:
        raise ValueError("oracle: invalid arguments")
    return out


def dft_naive(x: np.ndarray, log_n: int, inverse: bool) -> np.ndarray:
    y = np.zeros(1 << log_n, dtype=np.uint64)
    lib().gl_oracle_dft_naive(_p(np.ascontiguousarray(x, dtype=np.uint64)), _p(y), log_n, int(inverse))
    return y


def root_of_unity(log_size: int) -> int:
    return lib().gl_oracle_root_of_unity(log_size)


def canon(a: np.ndarray) -> np.ndarray:
    a = np.asarray(a, dtype=np.uint64)
    return np.where(a >= np.uint64(P), a - np.uint64(P), a)


def bitrev_permute(a: np.ndarray, log_n: int) -> np.ndarray:
    """Bit-reverse the last axis (length 2^log_n)."""
    idx = np.arange(1 << log_n, dtype=np.uint64)
    rev = np.zeros_like(idx)
    for b in range(log_n):
        rev |= ((idx >> np.uint64(b)) & np.uint64(1)) << np.uint64(log_n - 1 - b)
    return a[..., rev.astype(np.int64)]


def bit_reverse(src: np.ndarray, log_rows: int, cols: int, src_stride: int | None = None) -> np.ndarray:
    """dst[brev(i)] = src[i] per column (src/ops_complex.rs:306-318); dense output (stride 2^log_rows)."""
    rows = 1 << log_rows
    src = np.ascontiguousarray(src, dtype=np.uint64)
    dst = np.zeros(cols * rows, dtype=np.uint64)
    lib().gl_oracle_bit_reverse(_p(src), src_stride if src_stride is not None else rows, _p(dst), rows, log_rows,
                                cols)
    return dst


def powers_of(log_degree: int, offset: int, inverse: bool, bit_reverse: bool, of_g: bool, count: int) -> np.ndarray:
    """get_powers_of_w / get_powers_of_g (native/ops_complex.cu:9-33), canonical."""
    out = np.zeros(max(count, 1), dtype=np.uint64)
    lib().gl_oracle_powers_of(log_degree, offset, int(inverse), int(bit_reverse), int(of_g), _p(out), count)
    return out[:count]


def powers_by(base, offset: int, bit_reverse: bool, count: int) -> np.ndarray:
    """get_powers_by_val/ref (native/ops_complex.cu:35-74); base = int (base field) or (c0, c1) (extension,
    result laid out as all c0 then all c1)."""
    ext = isinstance(base, (tuple, list))
    c0, c1 = (base[0], base[1]) if ext else (base, 0)
    out = np.zeros(max((2 if ext else 1) * count, 1), dtype=np.uint64)
    lib().gl_oracle_powers_by(c0, c1, int(ext), offset, int(bit_reverse), _p(out), count)
    return out[:(2 if ext else 1) * count]


def omega_shift(src: np.ndarray, log_degree: int, offset: int, inverse: bool, shift: int) -> np.ndarray:
    """omega_shift (native/ops_complex.cu:76-87), canonical."""
    src = np.ascontiguousarray(src, dtype=np.uint64)
    out = np.zeros(max(len(src), 1), dtype=np.uint64)
    lib().gl_oracle_omega_shift(_p(src), log_degree, offset, int(inverse), shift, _p(out), len(src))
    return out[:len(src)]


EVAL_BASE_AT_BASE, EVAL_BASE_AT_EXT, EVAL_EXT_AT_EXT = 0, 1, 2


def lagrange_coeffs(x, coset: int, log_count: int, bit_reverse: bool) -> np.ndarray:
    """Barycentric coefficients L_i(x) on coset * <w_{2^log_count}> (src/barycentric.rs:83-126); x = int or
    (c0, c1); extension result = all c0 then all c1."""
    ext = isinstance(x, (tuple, list))
    x0, x1 = (x[0], x[1]) if ext else (x, 0)
    n = 1 << log_count
    out = np.zeros((2 if ext else 1) * n, dtype=np.uint64)
    lib().gl_oracle_lagrange_coeffs(x0, x1, int(ext), coset, log_count, int(bit_reverse), _p(out))
    return out


def batch_eval(kind: int, ys: np.ndarray, count: int, num_polys: int, coeffs: np.ndarray) -> np.ndarray:
    """sum_i y_{i,j} L_i per column (src/barycentric.rs:211-260); (c0, c1) pairs for the extension kinds."""
    ys = np.ascontiguousarray(ys, dtype=np.uint64)
    coeffs = np.ascontiguousarray(coeffs, dtype=np.uint64)
    out = np.zeros((1 if kind == EVAL_BASE_AT_BASE else 2) * max(num_polys, 1), dtype=np.uint64)
    lib().gl_oracle_batch_eval(kind, _p(ys), count, num_polys, _p(coeffs), _p(out))
    return out[:(1 if kind == EVAL_BASE_AT_BASE else 2) * num_polys]


def poly_eval(coeffs: np.ndarray, count: int, num_polys: int, x, ext_coeffs: bool = False) -> np.ndarray:
    """sum_i a_{i,j} x^i per column (Horner); (c0, c1) pairs per polynomial."""
    coeffs = np.ascontiguousarray(coeffs, dtype=np.uint64)
    x0, x1 = (x[0], x[1]) if isinstance(x, (tuple, list)) else (x, 0)
    out = np.zeros(2 * max(num_polys, 1), dtype=np.uint64)
    lib().gl_oracle_poly_eval(int(ext_coeffs), _p(coeffs), count, num_polys, x0, x1, _p(out))
    return out[:2 * num_polys]


class RefKernels:
    """The reference's own CUDA NTT kernels (needs a GPU and oracle/_ref/libref_ntt.so)."""

    def __init__(self):
        if not os.path.exists(REF_LIB):
            raise RuntimeError(f"{REF_LIB} missing: `make -C oracle ref` where the reference sources exist")
        L = ctypes.CDLL(REF_LIB)
        L.ref_context_create.argtypes = [_u32, _u32]
        L.ref_context_create.restype = _i32
        L.ref_context_destroy.argtypes = []
        L.ref_context_destroy.restype = _i32
        L.ref_batch_ntt.argtypes = [_vp, _vp, _u32, _u32, _u32, _u32, ctypes.c_bool, ctypes.c_bool, _u32, _u32,
                                    _vp]
        L.ref_batch_ntt.restype = _i32
        L.ref_bit_reverse.argtypes = [_vp, _u64, _vp, _u64, _u32, _u32, _vp]
        L.ref_bit_reverse.restype = _i32
        L.ref_get_powers_of.argtypes = [_u32, _u32, ctypes.c_bool, ctypes.c_bool, ctypes.c_bool, _vp, _u32, _vp]
        L.ref_get_powers_of.restype = _i32
        L.ref_get_powers_by_val.argtypes = [_u64, _u64, ctypes.c_bool, _u32, ctypes.c_bool, _vp, _u32, _vp]
        L.ref_get_powers_by_val.restype = _i32
        L.ref_omega_shift.argtypes = [_vp, _u32, _u32, ctypes.c_bool, _u32, _vp, _u32, _vp]
        L.ref_omega_shift.restype = _i32
        L.ref_barycentric_precompute.argtypes = [ctypes.c_bool, _vp, _vp, _u64, _vp, _u32, ctypes.c_bool, _vp]
        L.ref_barycentric_precompute.restype = _i32
        L.ref_batch_eval.argtypes = [_i32, _vp, _u32, _u32, _vp, _vp, _vp]
        L.ref_batch_eval.restype = _i32
        L.ref_batch_eval_partial.argtypes = [_i32, _vp, _u32, _u32, _vp, _vp, _vp]
        L.ref_batch_eval_partial.restype = _i32
        self.L = L
        rc = L.ref_context_create(12, 12)
        if rc != 0:
            raise RuntimeError(f"ref_context_create failed: {rc}")

    def batch_ntt(self, in_ptr: int, out_ptr: int, log_n: int, num_ntts: int, stride_in: int, stride_out: int,
                  bitrev_inputs: bool, inverse: bool, log_ext: int, coset_idx: int, stream: int):
        rc = self.L.ref_batch_ntt(in_ptr, out_ptr, log_n, num_ntts, stride_in, stride_out, bitrev_inputs, inverse,
                                  log_ext, coset_idx, stream)
        if rc != 0:
            raise RuntimeError(f"ref_batch_ntt failed: {rc}")

    def _ok(self, rc, what):
        if rc != 0:
            raise RuntimeError(f"{what} failed: {rc}")

    def bit_reverse(self, src_ptr: int, src_stride: int, dst_ptr: int, dst_stride: int, log_rows: int, cols: int,
                    stream: int):
        self._ok(self.L.ref_bit_reverse(src_ptr, src_stride, dst_ptr, dst_stride, log_rows, cols, stream),
                 "ref_bit_reverse")

    def get_powers_of(self, log_degree: int, offset: int, inverse: bool, bit_reverse: bool, of_g: bool,
                      result_ptr: int, count: int, stream: int):
        self._ok(self.L.ref_get_powers_of(log_degree, offset, inverse, bit_reverse, of_g, result_ptr, count, stream),
                 "ref_get_powers_of")

    def get_powers_by_val(self, base, offset: int, bit_reverse: bool, result_ptr: int, count: int, stream: int):
        ext = isinstance(base, (tuple, list))
        c0, c1 = (base[0], base[1]) if ext else (base, 0)
        self._ok(self.L.ref_get_powers_by_val(c0, c1, ext, offset, bit_reverse, result_ptr, count, stream),
                 "ref_get_powers_by_val")

    def omega_shift(self, src_ptr: int, log_degree: int, offset: int, inverse: bool, shift: int, dst_ptr: int,
                    count: int, stream: int):
        self._ok(self.L.ref_omega_shift(src_ptr, log_degree, offset, inverse, shift, dst_ptr, count, stream),
                 "ref_omega_shift")

    def barycentric_precompute(self, ext: bool, x_ptr: int, cf_ptr: int, coset: int, coeffs_ptr: int, count: int,
                               bit_reverse: bool, stream: int):
        self._ok(self.L.ref_barycentric_precompute(ext, x_ptr, cf_ptr, coset, coeffs_ptr, count, bit_reverse, stream),
                 "ref_barycentric_precompute")

    def batch_eval(self, kind: int, ys_ptr: int, count: int, num_polys: int, coeffs_ptr: int, stream: int) -> np.ndarray:
        out = np.zeros((1 if kind == 0 else 2) * max(num_polys, 1), dtype=np.uint64)
        self._ok(self.L.ref_batch_eval(kind, ys_ptr, count, num_polys, coeffs_ptr, _p(out), stream), "ref_batch_eval")
        return out[:(1 if kind == 0 else 2) * num_polys]

    def batch_eval_partial(self, kind: int, ys_ptr: int, count: int, num_polys: int, coeffs_ptr: int,
                           partial_ptr: int, stream: int):
        self._ok(self.L.ref_batch_eval_partial(kind, ys_ptr, count, num_polys, coeffs_ptr, partial_ptr, stream),
                 "ref_batch_eval_partial")

    def close(self):
        self.L.ref_context_destroy()
