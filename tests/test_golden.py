"""The CPU oracle against the reference's own kernels, without a GPU: every golden case (tests/golden/cases.py)
recomputed by the oracle must have the digest that the reference's CUDA kernels produced for it
(tests/golden/reference_hashes.json, written by tests/golden/make_reference_hashes.py on a B200)."""
import json
import os
import sys

import pytest

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(HERE, "golden"))

import cases  # noqa: E402

HASHES = os.path.join(HERE, "golden", "reference_hashes.json")


def _golden():
    with open(HASHES) as f:
        return json.load(f)["digests"]


def test_golden_covers_every_case():
    assert set(_golden()) == {c["name"] for c in cases.cases()}


@pytest.mark.parametrize("kind", ["ntt", "lde", "bitrev", "powers", "powby", "oshift", "lagr", "beval"])
def test_oracle_matches_reference_digests(kind):
    golden = _golden()
    bad = [c["name"] for c in cases.cases() if c["kind"] == kind and cases.digest(cases.oracle_output(c)) !=
           golden[c["name"]]]
    assert not bad, f"oracle differs from the reference's kernels on {bad}"


def test_splitmix64_known_answer():
    """The input generator itself: SplitMix64 from seed 0 starts 0xE220A8397B1DCDAF, 0x6E789E6AA1B965F4."""
    x = cases.splitmix64(0, 2)
    assert [int(v) for v in x] == [0xE220A8397B1DCDAF, 0x6E789E6AA1B965F4]
