#!/usr/bin/env python3
"""Runs every golden case (cases.py) through the reference's own CUDA kernels and writes their digests.

    python tests/golden/make_reference_hashes.py [--out tests/golden/reference_hashes.json]

Needs a GPU and oracle/_ref/libref_ntt.so (`make -C oracle ref`: the
reference's native/ntt.cu, context.cu, ops_complex.cu and barycentric.cu
compiled for sm_100a with oracle/ref_glue.cu).  The reference's outputs are
reduced to [0, p) before hashing (its kernels may leave values in [p, 2^64)).
"""
from __future__ import annotations

import argparse
import json
import os
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, HERE)
sys.path.insert(0, os.path.join(ROOT, "oracle"))

import numpy as np  # noqa: E402

import cases  # noqa: E402


def main():
    import torch

    import oracle

    ap = argparse.ArgumentParser()
    ap.add_argument("--out", default=os.path.join(HERE, "reference_hashes.json"))
    args = ap.parse_args()
    torch.cuda.set_device(0)
    ref = oracle.RefKernels()
    s = torch.cuda.current_stream().cuda_stream

    def dev(a: np.ndarray):
        return torch.from_numpy(np.ascontiguousarray(a).view(np.int64)).cuda()

    def zeros(n: int):
        return torch.zeros(max(n, 1), dtype=torch.int64, device="cuda")

    def host(t) -> np.ndarray:
        torch.cuda.synchronize()
        return t.cpu().numpy().view(np.uint64)

    digests = {}
    for c in cases.cases():
        k, name = c["kind"], c["name"]
        if k == "ntt":
            n = 1 << c["log_n"]
            x = dev(cases.words(name, c["cols"] * n))
            y = zeros(c["cols"] * n)
            ref.batch_ntt(x.data_ptr(), y.data_ptr(), c["log_n"], c["cols"], n, n, c["brev"], c["inv"], c["e"], c["k"],
                          s)
            got = host(y)[: c["cols"] * n]
        elif k == "lde":
            n, B = 1 << c["log_n"], 1 << c["log_b"]
            x = dev(cases.words(name, c["cols"] * n))
            coef, y = zeros(c["cols"] * n), zeros(B * c["cols"] * n)
            ref.batch_ntt(x.data_ptr(), coef.data_ptr(), c["log_n"], c["cols"], n, n, True, True, 0, 0, s)
            for j in range(B):
                ref.batch_ntt(coef.data_ptr(), y.data_ptr() + 8 * j * c["cols"] * n, c["log_n"], c["cols"], n, n,
                              False, False, c["log_b"], j, s)
            got = host(y)[: B * c["cols"] * n]
        elif k == "bitrev":
            rows = 1 << c["log_rows"]
            x = dev(cases.words(name, c["cols"] * rows))
            y = zeros(c["cols"] * rows)
            ref.bit_reverse(x.data_ptr(), rows, y.data_ptr(), rows, c["log_rows"], c["cols"], s)
            got = host(y)[: c["cols"] * rows]
        elif k == "powers":
            y = zeros(c["count"])
            ref.get_powers_of(c["log_degree"], c["offset"], c["inv"], c["brev"], c["of_g"], y.data_ptr(), c["count"], s)
            got = host(y)[: c["count"]]
        elif k == "powby":
            w = 2 if c["ext"] else 1
            y = zeros(w * c["count"])
            ref.get_powers_by_val(cases.powby_base(c), c["offset"], c["brev"], y.data_ptr(), c["count"], s)
            got = host(y)[: w * c["count"]]
        elif k == "oshift":
            x = dev(cases.words(name, c["count"]))
            y = zeros(c["count"])
            ref.omega_shift(x.data_ptr(), c["log_degree"], c["offset"], c["inv"], c["shift"], y.data_ptr(),
                            c["count"], s)
            got = host(y)[: c["count"]]
        elif k == "lagr":
            w = 2 if c["ext"] else 1
            pt = cases.lagr_point(c)
            x = dev(np.array(pt if c["ext"] else [pt], dtype=np.uint64))
            cf, y = zeros(w), zeros(w << c["log_count"])
            ref.barycentric_precompute(c["ext"], x.data_ptr(), cf.data_ptr(), 7, y.data_ptr(), 1 << c["log_count"],
                                       c["brev"], s)
            got = host(y)[: w << c["log_count"]]
        elif k == "beval":
            ys, coeffs = cases.beval_inputs(c)
            dys, dcf = dev(ys), dev(coeffs)
            got = ref.batch_eval(c["eval_kind"], dys.data_ptr(), 1 << c["log_count"], c["num_polys"], dcf.data_ptr(), s)
        else:
            raise ValueError(k)
        digests[name] = cases.digest(got)
    ref.close()
    with open(args.out, "w") as f:
        json.dump({"generator": "tests/golden/make_reference_hashes.py (reference kernels via oracle/_ref)",
                   "device": torch.cuda.get_device_name(0), "digests": digests}, f, indent=1, sort_keys=True)
    print(f"wrote {len(digests)} digests to {args.out}")


if __name__ == "__main__":
    main()
