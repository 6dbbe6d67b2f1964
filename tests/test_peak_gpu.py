"""The register-only butterfly loop that gives the transform kernels' integer roofline (bc_butterfly_peak).

Its arithmetic is the kernels' own round network, so it must also compute a valid field result: the loop's
16 outputs per thread are canonical-or-not u64 words that the size query accounts for, the butterfly count is
64 per thread per iteration, and a launch with too small an output buffer is refused."""
import ctypes

import pytest

pytestmark = pytest.mark.gpu


def test_butterfly_peak_runs_and_counts(gpu_ctx):
    import torch

    import bc_ntt

    L = bc_ntt.lib()
    words = ctypes.c_size_t(0)
    assert L.bc_butterfly_peak_words(ctypes.byref(words)) == 0
    assert words.value > 0 and words.value % 16 == 0
    out = torch.zeros(words.value, dtype=torch.int64, device="cuda")
    bfly = ctypes.c_uint64(0)
    s = torch.cuda.current_stream().cuda_stream
    assert L.bc_butterfly_peak(out.data_ptr(), words.value, 3, s, ctypes.byref(bfly)) == 0
    torch.cuda.synchronize()
    assert bfly.value == words.value // 16 * 64 * 3
    assert int((out != 0).sum()) > words.value // 2
    assert L.bc_butterfly_peak(out.data_ptr(), words.value - 1, 3, s, ctypes.byref(bfly)) == 1  # too small
