"""CPU checks of bench.py's host-side helpers: the committed ncu record it scales into `roofline.traffic` and
`roofline.limiter`, the L2 note of `config`, and the percentile used for p50/p99."""
import os
import sys

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)

import bench  # noqa: E402


def test_measured_traffic_scales_with_columns():
    byts8, alu, fma = bench.measured_traffic(22, 1, 8)
    assert byts8 is not None and alu is not None and fma is not None
    byts128, _, _ = bench.measured_traffic(22, 1, 128)
    assert byts128 == round(byts8 * 16)
    # one launch at 8 columns moves about the algorithmic bytes (8 n cols (1 + B)), not several times them
    algorithmic = 8 * (1 << 22) * 8 * 3
    assert 0.8 * algorithmic < byts8 < 1.2 * algorithmic
    assert 0 < alu <= 100 and 0 < fma <= 100


def test_measured_traffic_absent_record():
    assert bench.measured_traffic(19, 3, 8) == (None, None, None)


def test_l2_note_follows_the_workload():
    saved = bench.LOG_N, bench.COLS, bench.LOG_BLOWUP
    try:
        bench.LOG_N, bench.COLS, bench.LOG_BLOWUP = 22, 128, 1
        assert bench.l2_note() == "inputs 4 GiB and outputs 8 GiB, larger than L2; no flush"
        bench.LOG_N, bench.COLS, bench.LOG_BLOWUP = 14, 4, 2
        assert "fit in L2" in bench.l2_note()
    finally:
        bench.LOG_N, bench.COLS, bench.LOG_BLOWUP = saved


def test_percentile():
    xs = list(range(101))
    assert bench.pct(xs, 50) == 50
    assert bench.pct(xs, 99) == 99
    assert bench.pct([3.0], 99) == 3.0


def test_uniform_words_in_field_and_seeded():
    import numpy as np

    a = bench.uniform_words(200_000, 5, device="cpu").numpy().view(np.uint64)
    b = bench.uniform_words(200_000, 5, device="cpu").numpy().view(np.uint64)
    assert np.array_equal(a, b)
    assert (a < bench.P).all()
    # both halves spread over their whole range (no fold onto small values)
    hi, lo = a >> np.uint64(32), a & np.uint64(0xFFFFFFFF)
    assert hi.max() > 0xFFF00000 and lo.max() > 0xFFF00000 and hi.min() < 0x100000
    assert abs(float(hi.mean()) / 2**32 - 0.5) < 0.01
