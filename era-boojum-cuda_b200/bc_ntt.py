"""Python binding of libbc_ntt.so, mirroring the reference's Rust API.

The reference exposes ``boojum_cuda::ntt::{batch_ntt_internal,
batch_ntt_out_of_place, batch_ntt_in_place}`` (src/ntt.rs:179-369) and
``boojum_cuda::context::Context::{create, destroy}`` (src/context.rs:171-296).
This module exposes the same operations, with the same argument meaning, over
the C ABI declared in include/bc_ntt.h, and the ops of src/ops_complex.rs
(bit_reverse, get_powers_of_w/g, get_powers_by_val/ref, omega_shift) over
include/bc_ops.h, and barycentric evaluation (src/barycentric.rs) over
include/bc_barycentric.h.  Device buffers are torch CUDA tensors
of dtype int64 or uint64 (the words are reinterpreted, never converted);
streams default to torch's current stream.

Argument violations raise ``ValueError`` (the reference panics on its
asserts); CUDA failures raise ``RuntimeError``.  There is no CPU fallback:
loading fails loudly when the shared library is missing.
"""
from __future__ import annotations

import ctypes
import os

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "libbc_ntt.so")

P = 0xFFFFFFFF00000001
CUDA_ERROR_INVALID_VALUE = 1

_lib = None


def lib() -> ctypes.CDLL:
    """Load libbc_ntt.so (built in-tree by ``make -C era-boojum-cuda_b200``)."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise RuntimeError(f"{LIB_PATH} is missing: build it with `make -C {_HERE}`")
        L = ctypes.CDLL(LIB_PATH)
        _declare(L)
        _lib = L
    return _lib


_u32, _u64, _sz, _b, _vp = ctypes.c_uint32, ctypes.c_uint64, ctypes.c_size_t, ctypes.c_bool, ctypes.c_void_p

# name -> argument types; every entry point returns cudaError_t (int).
SIGNATURES = {
    "bc_ntt_context_create": [_u32, _u32],
    "bc_ntt_context_destroy": [],
    "bc_batch_ntt_internal": [_vp, _vp, _u32, _u32, _u64, _u64, _b, _b, _u32, _u32, _vp],
    "bc_batch_ntt_out_of_place": [_vp, _sz, _vp, _sz, _u32, _u32, _u64, _u64, _u64, _u64, _b, _b, _u32, _u32, _vp],
    "bc_batch_ntt_in_place": [_vp, _sz, _u32, _u32, _u64, _u64, _b, _b, _u32, _u32, _vp],
    "bc_batch_ntt_with_plan": [_vp, _vp, _u32, _u32, _u64, _u64, _b, _b, _u32, _u32, _vp, _vp, _u32, _vp],
    "bc_autotune": [_u32, _u32, _u32, _u32, _vp, _sz],
    "bc_plan_table_export": [_vp, _sz, _vp],
    "bc_plan_table_import": [ctypes.c_char_p],
    "bc_plan_table_clear": [],
    "bc_lde_plain": [_vp, _vp, _u32, _u32, _u64, _u64, _u64, _u32, _vp],
    "bc_lde_fused": [_vp, _vp, _u32, _u32, _u64, _u64, _u64, _u32, _vp],
    "bc_lde_fused_profiled": [_vp, _vp, _u32, _u32, _u64, _u64, _u64, _u32, _vp, _vp, _u32, _vp],
    "bc_lde_host": [_vp, _vp, _u32, _u32, _u64, _u64, _u64, _u32, _vp, _sz, _u32, _vp],
    "bc_lde_batch_plan_create": [_vp, _u32, _vp],
    "bc_lde_batch_plan_create_ex": [_vp, _u32, _u32, _vp],
    "bc_lde_batch_run": [_vp, _vp],
    "bc_lde_batch_status": [_vp, _vp, _vp],
    "bc_lde_batch_plan_set_wait_limit": [_vp, _u64],
    "bc_lde_batch_plan_info": [_vp, _vp, _vp, _vp],
    "bc_butterfly_peak_words": [_vp],
    "bc_butterfly_peak": [_vp, _sz, _u32, _vp, _vp],
    "bc_lde_batch_plan_destroy": [_vp],
    "bc_lde_batch_noalloc": [_vp, _u32, _vp, _vp],
    "bc_lde_server_create": [_vp, _vp],
    "bc_lde_server_submit": [_vp, _vp, _vp, _u32, _u32, _u32, _vp],
    "bc_lde_server_submit_device": [_vp, _vp, _vp, _u32, _u32, _u32, _vp],
    "bc_lde_server_set_device_batching": [_vp, _u64],
    "bc_lde_server_get_device_stats": [_vp, _vp, _vp, _vp],
    "bc_lde_server_poll": [_vp, _u64, _vp, _vp],
    "bc_lde_server_wait": [_vp, _u64, _u32, _vp],
    "bc_lde_server_cancel": [_vp, _u64],
    "bc_lde_server_release": [_vp, _u64],
    "bc_lde_server_get_stats": [_vp, _vp],
    "bc_lde_server_destroy": [_vp],
    "bc_bit_reverse": [_vp, _u64, _vp, _u64, _u32, _u32, _vp],
    "bc_bit_reverse_in_place": [_vp, _u64, _u32, _u32, _vp],
    "bc_get_powers_of_w": [_u32, _u32, _b, _b, _vp, _u32, _vp],
    "bc_get_powers_of_g": [_u32, _u32, _b, _b, _vp, _u32, _vp],
    "bc_get_powers_by_val_bf": [_u64, _u32, _b, _vp, _u32, _vp],
    "bc_get_powers_by_ref_bf": [_vp, _u32, _b, _vp, _u32, _vp],
    "bc_get_powers_by_val_ef": [_u64, _u64, _u32, _b, _vp, _u32, _vp],
    "bc_get_powers_by_ref_ef": [_vp, _u32, _b, _vp, _u32, _vp],
    "bc_omega_shift": [_vp, _u32, _u32, _b, _u32, _vp, _u32, _vp],
    "bc_omega_shift_in_place": [_vp, _u32, _u32, _b, _u32, _u32, _vp],
    "bc_precompute_lagrange_coeffs_at_base": [_vp, _vp, _u64, _vp, _u32, _b, _vp],
    "bc_precompute_lagrange_coeffs_at_ext": [_vp, _vp, _u64, _vp, _u32, _b, _vp],
    "bc_get_batch_eval_temp_storage_sizes": [ctypes.c_int, _u32, _u32, _vp, _vp],
    "bc_batch_eval": [ctypes.c_int, _vp, _u32, _u32, _vp, _vp, _sz, _vp, _sz, _vp, _vp],
}

CUDA_ERROR_NOT_READY = 600
CUDA_ERROR_TIMEOUT = 909


class ServerConfig(ctypes.Structure):
    _fields_ = [("memory_budget_bytes", _sz), ("slots", _u32), ("max_chunk_cols", _u32)]


class ServerStats(ctypes.Structure):
    _fields_ = [("completed", _u64), ("pending", _u64), ("running", _u64), ("p50_ms", ctypes.c_double),
                ("p99_ms", ctypes.c_double), ("max_ms", ctypes.c_double), ("span_s", ctypes.c_double),
                ("out_melem_per_s", ctypes.c_double), ("arena_largest_free", _sz)]


class LdeJob(ctypes.Structure):
    """bc_lde_job of include/bc_ntt.h."""
    _fields_ = [("evals_bitrev", _vp), ("out", _vp), ("stride_in", _u64), ("stride_out", _u64),
                ("coset_stride", _u64), ("log_n", _u32), ("num_cols", _u32), ("log_blowup", _u32),
                ("reserved", _u32)]


def _declare(L):
    for name, args in SIGNATURES.items():
        fn = getattr(L, name)
        fn.argtypes = args
        fn.restype = ctypes.c_int


def _check(rc: int, what: str):
    if rc == 0:
        return
    if rc == CUDA_ERROR_INVALID_VALUE:
        raise ValueError(f"{what}: invalid argument (cudaErrorInvalidValue)")
    raise RuntimeError(f"{what}: CUDA error {rc}")


def _stream(stream):
    if stream is None:
        import torch

        return torch.cuda.current_stream().cuda_stream
    if isinstance(stream, int):
        return stream
    return stream.cuda_stream


def _ptr(t, offset: int = 0):
    return t.data_ptr() + 8 * offset


def _len(t) -> int:
    return t.numel()


class Context:
    """Twiddle/power tables on the current device (src/context.rs:157-297)."""

    def __init__(self):
        self.live = False

    @classmethod
    def create(cls, powers_of_w_coarse_log_count: int = 12, powers_of_g_coarse_log_count: int = 12) -> "Context":
        _check(lib().bc_ntt_context_create(powers_of_w_coarse_log_count, powers_of_g_coarse_log_count),
               "Context.create")
        c = cls()
        c.live = True
        return c

    def destroy(self):
        if self.live:
            _check(lib().bc_ntt_context_destroy(), "Context.destroy")
            self.live = False


def batch_ntt_internal(inputs_ptr: int, outputs_ptr: int, log_n: int, num_ntts: int,
                       stride_between_input_arrays: int, stride_between_output_arrays: int,
                       bitrev_inputs: bool, inverse: bool, log_extension_degree: int, coset_index: int,
                       stream=None):
    """Raw-pointer entry point (src/ntt.rs:179-191)."""
    _check(lib().bc_batch_ntt_internal(inputs_ptr, outputs_ptr, log_n, num_ntts, stride_between_input_arrays,
                                       stride_between_output_arrays, bitrev_inputs, inverse,
                                       log_extension_degree, coset_index, _stream(stream)),
           "batch_ntt_internal")


def batch_ntt_out_of_place(inputs_matrix, outputs_matrix, log_n: int, num_ntts: int, inputs_offset: int,
                           outputs_offset: int, stride_between_input_arrays: int,
                           stride_between_output_arrays: int, bitrev_inputs: bool, inverse: bool,
                           log_extension_degree: int, coset_index: int, stream=None):
    """src/ntt.rs:294-335 over torch device tensors."""
    _check(lib().bc_batch_ntt_out_of_place(_ptr(inputs_matrix), _len(inputs_matrix), _ptr(outputs_matrix),
                                           _len(outputs_matrix), log_n, num_ntts, inputs_offset, outputs_offset,
                                           stride_between_input_arrays, stride_between_output_arrays,
                                           bitrev_inputs, inverse, log_extension_degree, coset_index,
                                           _stream(stream)),
           "batch_ntt_out_of_place")


def batch_ntt_in_place(inputs_matrix, log_n: int, num_ntts: int, inputs_offset: int,
                       stride_between_input_arrays: int, bitrev_inputs: bool, inverse: bool,
                       log_extension_degree: int, coset_index: int, stream=None):
    """src/ntt.rs:338-369 over a torch device tensor."""
    _check(lib().bc_batch_ntt_in_place(_ptr(inputs_matrix), _len(inputs_matrix), log_n, num_ntts, inputs_offset,
                                       stride_between_input_arrays, bitrev_inputs, inverse, log_extension_degree,
                                       coset_index, _stream(stream)),
           "batch_ntt_in_place")


def batch_ntt_with_plan(inputs, outputs, log_n: int, num_ntts: int, stride_in: int, stride_out: int,
                        bitrev_inputs: bool, inverse: bool, log_extension_degree: int, coset_index: int,
                        plan, stream=None):
    """Transform with an explicit pass plan: ``plan`` = [(bits, run), ...] from the top bits down."""
    bits = (ctypes.c_uint8 * len(plan))(*[k for k, _ in plan])
    runs = (ctypes.c_uint8 * len(plan))(*[c for _, c in plan])
    _check(lib().bc_batch_ntt_with_plan(_ptr(inputs), _ptr(outputs), log_n, num_ntts, stride_in, stride_out,
                                        bitrev_inputs, inverse, log_extension_degree, coset_index,
                                        ctypes.cast(bits, _vp), ctypes.cast(runs, _vp), len(plan),
                                        _stream(stream)),
           "batch_ntt_with_plan")


def lde(evals_bitrev, out, log_n: int, num_cols: int, log_blowup: int, stride_in: int | None = None,
        stride_out: int | None = None, coset_stride: int | None = None, fused: bool = True, stream=None):
    """Coset LDE of bit-reversed evaluations (torch device tensors); default layout coset-major."""
    n = 1 << log_n
    stride_in = n if stride_in is None else stride_in
    stride_out = n if stride_out is None else stride_out
    coset_stride = num_cols * stride_out if coset_stride is None else coset_stride
    fn = lib().bc_lde_fused if fused else lib().bc_lde_plain
    _check(fn(_ptr(evals_bitrev), _ptr(out), log_n, num_cols, stride_in, stride_out, coset_stride, log_blowup,
              _stream(stream)), "lde")


class LdeBatch:
    """A persistent-kernel batch plan over uneven LDE jobs (bc_lde_batch_*)."""

    def __init__(self, jobs, standalone_min_ctas: int = 0):
        """jobs: list of (evals tensor, out tensor, log_n, num_cols, log_blowup) with dense coset-major outputs,
        or LdeJob structures.  standalone_min_ctas > 0: jobs whose kernels are at least that wide run as their own
        kernels on a forked branch of the plan's graph (bc_lde_batch_plan_create_ex)."""
        arr = (LdeJob * max(1, len(jobs)))()
        for i, j in enumerate(jobs):
            if isinstance(j, LdeJob):
                arr[i] = j
            else:
                ev, out, log_n, cols, log_b = j
                n = 1 << log_n
                arr[i] = LdeJob(_ptr(ev), _ptr(out), n, n, cols * n, log_n, cols, log_b, 0)
        self._jobs = arr
        self.handle = ctypes.c_void_p()
        _check(lib().bc_lde_batch_plan_create_ex(ctypes.cast(arr, _vp), len(jobs), standalone_min_ctas,
                                                 ctypes.byref(self.handle)), "bc_lde_batch_plan_create_ex")

    def run(self, stream=None):
        _check(lib().bc_lde_batch_run(self.handle, _stream(stream)), "bc_lde_batch_run")

    def status(self, stream=None) -> int:
        st = ctypes.c_uint32(0)
        _check(lib().bc_lde_batch_status(self.handle, _stream(stream), ctypes.byref(st)), "bc_lde_batch_status")
        return st.value

    def set_wait_limit(self, cycles: int):
        """SM clock cycles one dependency wait of the persistent kernel may take (0: the default, about 4 s)."""
        _check(lib().bc_lde_batch_plan_set_wait_limit(self.handle, cycles), "bc_lde_batch_plan_set_wait_limit")

    def info(self):
        r, i, g = ctypes.c_uint32(), ctypes.c_uint32(), ctypes.c_uint32()
        _check(lib().bc_lde_batch_plan_info(self.handle, ctypes.byref(r), ctypes.byref(i), ctypes.byref(g)),
               "bc_lde_batch_plan_info")
        return {"records": r.value, "items": i.value, "grid": g.value}

    def close(self):
        if self.handle:
            _check(lib().bc_lde_batch_plan_destroy(self.handle), "bc_lde_batch_plan_destroy")
            self.handle = ctypes.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def lde_host(host_evals, host_out, log_n: int, num_cols: int, log_blowup: int, workspace, max_chunk_cols: int = 0,
             stream=None):
    """LDE from host tensors (pinned for overlap) to host tensors through a device workspace tensor."""
    n = 1 << log_n
    _check(lib().bc_lde_host(_ptr(host_evals), _ptr(host_out), log_n, num_cols, n, n, num_cols * n, log_blowup,
                             _ptr(workspace), workspace.numel() * workspace.element_size(), max_chunk_cols,
                             _stream(stream)), "lde_host")


class LdeServer:
    """Continuous-batching LDE server (bc_lde_server_*) on the current device."""

    PENDING, RUNNING, DONE, CANCELLED, FAILED = range(5)

    def __init__(self, memory_budget_bytes: int, slots: int = 4, max_chunk_cols: int = 0):
        cfg = ServerConfig(memory_budget_bytes, slots, max_chunk_cols)
        self.handle = ctypes.c_void_p()
        _check(lib().bc_lde_server_create(ctypes.byref(cfg), ctypes.byref(self.handle)), "bc_lde_server_create")
        self._keep = {}

    def submit(self, host_evals, host_out, log_n: int, num_cols: int, log_blowup: int) -> int:
        rid = ctypes.c_uint64()
        _check(lib().bc_lde_server_submit(self.handle, _ptr(host_evals), _ptr(host_out), log_n, num_cols, log_blowup,
                                          ctypes.byref(rid)), "bc_lde_server_submit")
        self._keep[rid.value] = (host_evals, host_out)
        return rid.value

    def submit_device(self, dev_evals, dev_out, log_n: int, num_cols: int, log_blowup: int) -> int:
        """A request on device tensors (dense layouts); small pending ones are coalesced into one batch launch."""
        rid = ctypes.c_uint64()
        _check(lib().bc_lde_server_submit_device(self.handle, _ptr(dev_evals), _ptr(dev_out), log_n, num_cols,
                                                 log_blowup, ctypes.byref(rid)), "bc_lde_server_submit_device")
        self._keep[rid.value] = (dev_evals, dev_out)
        return rid.value

    def set_device_batching(self, max_batch_elems: int):
        """Output elements up to which pending device requests are coalesced (0: none)."""
        _check(lib().bc_lde_server_set_device_batching(self.handle, max_batch_elems), "set_device_batching")

    def device_stats(self):
        b, br, sr = ctypes.c_uint64(), ctypes.c_uint64(), ctypes.c_uint64()
        _check(lib().bc_lde_server_get_device_stats(self.handle, ctypes.byref(b), ctypes.byref(br), ctypes.byref(sr)),
               "bc_lde_server_get_device_stats")
        return {"batches": b.value, "batched_requests": br.value, "single_requests": sr.value}

    def poll(self, rid: int):
        st, lat = ctypes.c_int(), ctypes.c_double()
        _check(lib().bc_lde_server_poll(self.handle, rid, ctypes.byref(st), ctypes.byref(lat)), "poll")
        return st.value, lat.value

    def wait(self, rid: int, timeout_ms: int = 60000) -> float:
        """Latency in ms; raises TimeoutError / RuntimeError (cancelled or failed)."""
        lat = ctypes.c_double()
        rc = lib().bc_lde_server_wait(self.handle, rid, timeout_ms, ctypes.byref(lat))
        if rc == CUDA_ERROR_TIMEOUT:
            raise TimeoutError(f"request {rid} not finished after {timeout_ms} ms")
        if rc == CUDA_ERROR_NOT_READY:
            raise RuntimeError(f"request {rid} was cancelled")
        _check(rc, "bc_lde_server_wait")
        return lat.value

    def cancel(self, rid: int) -> bool:
        rc = lib().bc_lde_server_cancel(self.handle, rid)
        if rc == CUDA_ERROR_NOT_READY:
            return False
        _check(rc, "bc_lde_server_cancel")
        return True

    def release(self, rid: int) -> bool:
        """Forgets a finished (done, cancelled or failed) request and drops the host buffers kept for it;
        False while it is pending or running."""
        rc = lib().bc_lde_server_release(self.handle, rid)
        if rc == CUDA_ERROR_NOT_READY:
            return False
        _check(rc, "bc_lde_server_release")
        self._keep.pop(rid, None)
        return True

    def stats(self) -> dict:
        st = ServerStats()
        _check(lib().bc_lde_server_get_stats(self.handle, ctypes.byref(st)), "bc_lde_server_get_stats")
        return {f: getattr(st, f) for f, _ in ServerStats._fields_}

    def close(self):
        if self.handle:
            _check(lib().bc_lde_server_destroy(self.handle), "bc_lde_server_destroy")
            self.handle = ctypes.c_void_p()
            self._keep.clear()


def autotune(log_n: int, log_blowup: int, num_cols: int, reps: int = 3) -> str:
    """Times every candidate plan for (log_n, log_blowup) on the current device, then the launch knobs of the
    best window split, and keeps the fastest; returns one report line per timed candidate."""
    buf = ctypes.create_string_buffer(16384)
    _check(lib().bc_autotune(log_n, log_blowup, num_cols, reps, buf, len(buf)), "bc_autotune")
    return buf.value.decode()


def plan_table_export() -> str:
    need = ctypes.c_size_t(0)
    _check(lib().bc_plan_table_export(None, 0, ctypes.byref(need)), "bc_plan_table_export")
    buf = ctypes.create_string_buffer(max(1, need.value))
    _check(lib().bc_plan_table_export(buf, len(buf), None), "bc_plan_table_export")
    return buf.value.decode()


def plan_table_import(text: str):
    _check(lib().bc_plan_table_import(text.encode()), "bc_plan_table_import")


def plan_table_clear():
    _check(lib().bc_plan_table_clear(), "bc_plan_table_clear")


PLANS_PATH = os.path.join(_HERE, "plans_b200.txt")


def load_tuned_plans(path: str = PLANS_PATH) -> bool:
    """Loads a plan table written by tune_plans.py (the current device must have a context)."""
    if not os.path.exists(path):
        return False
    text = "".join(line for line in open(path) if line.strip() and not line.startswith("#"))
    plan_table_import(text)
    return True


# ---------------------------------------------------------------- ops (src/ops_complex.rs, include/bc_ops.h)
def _u32_count(n: int, what: str) -> int:
    if n > 0xFFFFFFFF:
        raise ValueError(f"{what}: more than 2^32 - 1 elements")
    return n


def bit_reverse(src, dst, log_rows: int, cols: int, src_stride: int | None = None, dst_stride: int | None = None,
                stream=None):
    """bit_reverse (src/ops_complex.rs:306-318): dst[brev(i)] = src[i] in each column of 2^log_rows rows."""
    rows = 1 << log_rows
    ss = rows if src_stride is None else src_stride
    ds = rows if dst_stride is None else dst_stride
    if cols and (_len(src) < (cols - 1) * ss + rows or _len(dst) < (cols - 1) * ds + rows):
        raise ValueError("bit_reverse: matrix does not fit its buffer")
    _check(lib().bc_bit_reverse(_ptr(src), ss, _ptr(dst), ds, log_rows, cols, _stream(stream)), "bit_reverse")


def bit_reverse_in_place(values, log_rows: int, cols: int, stride: int | None = None, stream=None):
    """bit_reverse_in_place (src/ops_complex.rs:320-329)."""
    rows = 1 << log_rows
    st = rows if stride is None else stride
    if cols and _len(values) < (cols - 1) * st + rows:
        raise ValueError("bit_reverse_in_place: matrix does not fit its buffer")
    _check(lib().bc_bit_reverse_in_place(_ptr(values), st, log_rows, cols, _stream(stream)), "bit_reverse_in_place")


def get_powers_of_w(log_degree: int, offset: int, inverse: bool, bit_reverse: bool, result, stream=None):
    """get_powers_of_w (src/ops_complex.rs:40-85): len(result) powers of w_{2^log_degree}."""
    n = _u32_count(_len(result), "get_powers_of_w")
    _check(lib().bc_get_powers_of_w(log_degree, offset, inverse, bit_reverse, _ptr(result), n, _stream(stream)),
           "get_powers_of_w")


def get_powers_of_g(log_degree: int, offset: int, inverse: bool, bit_reverse: bool, result, stream=None):
    """get_powers_of_g (src/ops_complex.rs:40-86): len(result) powers of 7^(2^(24 - log_degree))."""
    n = _u32_count(_len(result), "get_powers_of_g")
    _check(lib().bc_get_powers_of_g(log_degree, offset, inverse, bit_reverse, _ptr(result), n, _stream(stream)),
           "get_powers_of_g")


def get_powers_by_val(base, offset: int, bit_reverse: bool, result, stream=None):
    """get_powers_by_val (src/ops_complex.rs:117-131).  base: int (base field; len(result) powers) or
    (c0, c1) (extension; result holds 2 * count words, all c0 then all c1)."""
    if isinstance(base, (tuple, list)):
        n = _u32_count(_len(result) // 2, "get_powers_by_val")
        _check(lib().bc_get_powers_by_val_ef(base[0], base[1], offset, bit_reverse, _ptr(result), n,
                                             _stream(stream)), "get_powers_by_val")
    else:
        n = _u32_count(_len(result), "get_powers_by_val")
        _check(lib().bc_get_powers_by_val_bf(base, offset, bit_reverse, _ptr(result), n, _stream(stream)),
               "get_powers_by_val")


def get_powers_by_ref(base, offset: int, bit_reverse: bool, result, ext: bool = False, stream=None):
    """get_powers_by_ref (src/ops_complex.rs:176-190): base is a device tensor holding the base (1 word, or
    2 words for the extension)."""
    if ext:
        if _len(base) < 2:
            raise ValueError("get_powers_by_ref: an extension base takes 2 words")
        n = _u32_count(_len(result) // 2, "get_powers_by_ref")
        _check(lib().bc_get_powers_by_ref_ef(_ptr(base), offset, bit_reverse, _ptr(result), n, _stream(stream)),
               "get_powers_by_ref")
    else:
        n = _u32_count(_len(result), "get_powers_by_ref")
        _check(lib().bc_get_powers_by_ref_bf(_ptr(base), offset, bit_reverse, _ptr(result), n, _stream(stream)),
               "get_powers_by_ref")


def omega_shift(src, log_degree: int, offset: int, inverse: bool, shift: int, dst, stream=None):
    """omega_shift (src/ops_complex.rs:226-242): dst[i] = src[i] * w^(shift * (i + offset)), w = w_{2^log_degree}."""
    if _len(src) != _len(dst):
        raise ValueError("omega_shift: src and dst lengths differ")
    n = _u32_count(_len(dst), "omega_shift")
    _check(lib().bc_omega_shift(_ptr(src), log_degree, offset, inverse, shift, _ptr(dst), n, _stream(stream)),
           "omega_shift")


def omega_shift_in_place(values, log_degree: int, offset: int, inverse: bool, shift: int, stream=None):
    """omega_shift_in_place (src/ops_complex.rs:244-258)."""
    n = _u32_count(_len(values), "omega_shift_in_place")
    _check(lib().bc_omega_shift_in_place(_ptr(values), log_degree, offset, inverse, shift, n, _stream(stream)),
           "omega_shift_in_place")


# ---------------------------------------------------------------- barycentric (src/barycentric.rs, include/bc_barycentric.h)
EVAL_BASE_AT_BASE, EVAL_BASE_AT_EXT, EVAL_EXT_AT_EXT = 0, 1, 2


def precompute_lagrange_coeffs(x, common_factor_storage, coset: int, lagrange_coeffs, bit_reverse: bool,
                               ext: bool = False, stream=None):
    """precompute_lagrange_coeffs (src/barycentric.rs:83-126): x and common_factor_storage are device tensors
    of 1 word (base field) or 2 words (extension, ext=True); lagrange_coeffs holds count (2 * count) words."""
    w = 2 if ext else 1
    if _len(x) < w or _len(common_factor_storage) < w:
        raise ValueError("precompute_lagrange_coeffs: x / storage too short")
    count = _len(lagrange_coeffs) // w
    fn = lib().bc_precompute_lagrange_coeffs_at_ext if ext else lib().bc_precompute_lagrange_coeffs_at_base
    _check(fn(_ptr(x), _ptr(common_factor_storage), coset, _ptr(lagrange_coeffs), count, bit_reverse,
              _stream(stream)), "precompute_lagrange_coeffs")


def get_batch_eval_temp_storage_sizes(kind: int, count: int, num_polys: int):
    """get_batch_eval_temp_storage_sizes (src/barycentric.rs:193-209): (u64 words, bytes) of scratch."""
    words, nbytes = ctypes.c_size_t(0), ctypes.c_size_t(0)
    _check(lib().bc_get_batch_eval_temp_storage_sizes(kind, count, num_polys, ctypes.byref(words),
                                                      ctypes.byref(nbytes)), "get_batch_eval_temp_storage_sizes")
    return words.value, nbytes.value


def batch_eval(kind: int, batch_ys, count: int, num_polys: int, lagrange_coeffs, temp_partial_reduce,
               temp_final_reduce, evals, stream=None):
    """batch_eval (src/barycentric.rs:211-260): evals[j] = sum_i ys[i, j] L_i for num_polys columns of count
    rows; extension kinds write (c0, c1) pairs.  temp_final_reduce may be None (0 bytes needed)."""
    xw = 1 if kind == EVAL_BASE_AT_BASE else 2
    yw = 2 if kind == EVAL_EXT_AT_EXT else 1
    if _len(batch_ys) < yw * num_polys * count or _len(lagrange_coeffs) < xw * count or _len(evals) < xw * num_polys:
        raise ValueError("batch_eval: buffers too short")
    fin_ptr = _ptr(temp_final_reduce) if temp_final_reduce is not None else None
    fin_len = temp_final_reduce.numel() * temp_final_reduce.element_size() if temp_final_reduce is not None else 0
    _check(lib().bc_batch_eval(kind, _ptr(batch_ys), count, num_polys, _ptr(lagrange_coeffs),
                               _ptr(temp_partial_reduce), _len(temp_partial_reduce), fin_ptr, fin_len, _ptr(evals),
                               _stream(stream)), "batch_eval")
