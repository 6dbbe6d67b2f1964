"""Golden cases: the reference's own kernels' outputs, pinned as SHA-256 digests.

The reference ships no golden vectors for this path (its tests compare against
boojum's CPU code, which is not vendored).  These cases are run once through
the reference's CUDA kernels compiled from its sources (oracle/_ref, driven by
oracle/ref_glue.cu) by make_reference_hashes.py on a GPU; the digests of their
canonical outputs are committed in reference_hashes.json, and
tests/test_golden.py recomputes every case with the CPU oracle and compares
digests -- so the oracle is pinned to the reference without a GPU.

Inputs come from SplitMix64 (seeded per case by the case's name), independent
of numpy's generators.  A digest is SHA-256 of the canonical ([0, p)) outputs
as little-endian u64 words.

Cases (reference entry point -> oracle function):
  ntt_*     batch_ntt_internal (src/ntt.rs:179-290): every (bitrev_inputs,
            inverse) pair, plain and coset (log_extension_degree, coset_index)
            = (1, 1) and (3, 5); log_n 1..15 (the one-stage kernels) and 16, 17
            (the multi-stage kernels); raw u64 inputs, non-canonical included.
  lde_*     the composition the reference's callers run (benches/ntt.rs:110-116).
  bitrev_*  bit_reverse (src/ops_complex.rs:271-329).
  powers_*  get_powers_of_w / _g (src/ops_complex.rs:40-86).
  powby_*   get_powers_by_val (src/ops_complex.rs:117-160).
  oshift_*  omega_shift (src/ops_complex.rs:207-236).
  lagr_*    precompute_lagrange_coeffs (src/barycentric.rs:83-148).
  beval_*   batch_eval (src/barycentric.rs:183-281).
"""
from __future__ import annotations

import hashlib
import zlib

import numpy as np

P = 0xFFFFFFFF00000001


def splitmix64(seed: int, n: int) -> np.ndarray:
    """n SplitMix64 outputs for `seed` (state seed + i * golden gamma, i = 1..n)."""
    with np.errstate(over="ignore"):
        z = np.uint64(seed & 0xFFFFFFFFFFFFFFFF) + np.arange(1, n + 1, dtype=np.uint64) * np.uint64(
            0x9E3779B97F4A7C15)
        z = (z ^ (z >> np.uint64(30))) * np.uint64(0xBF58476D1CE4E5B9)
        z = (z ^ (z >> np.uint64(27))) * np.uint64(0x94D049BB133111EB)
        return z ^ (z >> np.uint64(31))


def words(name: str, n: int, canonical: bool = False) -> np.ndarray:
    """The case's input words: raw u64, or reduced below p."""
    x = splitmix64(zlib.crc32(name.encode()), n)
    return x % np.uint64(P) if canonical else x


def digest(a: np.ndarray) -> str:
    c = np.asarray(a, dtype=np.uint64)
    c = np.where(c >= np.uint64(P), c - np.uint64(P), c)
    return hashlib.sha256(np.ascontiguousarray(c, dtype="<u8").tobytes()).hexdigest()


def cases() -> list[dict]:
    out = []
    for log_n in (1, 2, 3, 4, 6, 9, 12, 15, 16, 17):
        for brev in (False, True):
            for inv in (False, True):
                for e, k in ((0, 0), (1, 1), (3, 5)):
                    out.append(dict(kind="ntt", name=f"ntt_n{log_n}_b{int(brev)}_i{int(inv)}_e{e}_k{k}", log_n=log_n,
                                    cols=2, brev=brev, inv=inv, e=e, k=k))
    for log_n, cols, log_b in ((5, 3, 1), (12, 3, 2), (16, 2, 1)):
        out.append(dict(kind="lde", name=f"lde_n{log_n}_c{cols}_b{log_b}", log_n=log_n, cols=cols, log_b=log_b))
    for log_rows in (0, 1, 5, 10, 12, 14):
        out.append(dict(kind="bitrev", name=f"bitrev_r{log_rows}", log_rows=log_rows, cols=3))
    for log_degree, offset, count in ((12, 77, 4096 + 13), (24, 2**32 - 300, 1000), (20, 5, 3)):
        for of_g in (False, True):
            for inv in (False, True):
                for brev in (False, True):
                    out.append(dict(kind="powers", name=f"powers_d{log_degree}_o{offset}_g{int(of_g)}_i{int(inv)}"
                                    f"_b{int(brev)}", log_degree=log_degree, offset=offset, count=count, of_g=of_g,
                                    inv=inv, brev=brev))
    for ext in (False, True):
        for offset, count, brev in ((0, 5000, False), (17, 4099, True)):
            out.append(dict(kind="powby", name=f"powby_x{int(ext)}_o{offset}_b{int(brev)}", ext=ext, offset=offset,
                            count=count, brev=brev))
    for log_degree, offset, shift, count in ((24, 3, 2**31 + 7, 5000), (10, 2**32 - 1000, 3, 4097)):
        for inv in (False, True):
            out.append(dict(kind="oshift", name=f"oshift_d{log_degree}_o{offset}_i{int(inv)}", log_degree=log_degree,
                            offset=offset, shift=shift, count=count, inv=inv))
    for ext in (False, True):
        for log_count in (0, 5, 12):
            for brev in (False, True):
                out.append(dict(kind="lagr", name=f"lagr_x{int(ext)}_n{log_count}_b{int(brev)}", ext=ext,
                                log_count=log_count, brev=brev))
    for kind in (0, 1, 2):
        out.append(dict(kind="beval", name=f"beval_k{kind}", eval_kind=kind, log_count=10, num_polys=3))
    return out


def powby_base(c: dict):
    b = words(c["name"] + "/base", 2)
    return (int(b[0]), int(b[1])) if c["ext"] else int(b[0])


def lagr_point(c: dict):
    x = words(c["name"] + "/x", 2, canonical=True)
    return (int(x[0]), int(x[1])) if c["ext"] else int(x[0])


def beval_inputs(c: dict):
    count, polys, kind = 1 << c["log_count"], c["num_polys"], c["eval_kind"]
    ys = words(c["name"] + "/ys", (2 if kind == 2 else 1) * polys * count, canonical=True)
    coeffs = words(c["name"] + "/coeffs", (1 if kind == 0 else 2) * count, canonical=True)
    return ys, coeffs


def oracle_output(c: dict) -> np.ndarray:
    """The case computed by the CPU oracle (oracle/oracle.py)."""
    import oracle

    k = c["kind"]
    if k == "ntt":
        n = 1 << c["log_n"]
        x = words(c["name"], c["cols"] * n)
        return oracle.batch_ntt(x, c["log_n"], c["cols"], n, n, c["brev"], c["inv"], c["e"], c["k"], threads=4)
    if k == "lde":
        n = 1 << c["log_n"]
        x = words(c["name"], c["cols"] * n)
        return oracle.lde(x, c["log_n"], c["cols"], n, c["log_b"], threads=4)
    if k == "bitrev":
        x = words(c["name"], c["cols"] << c["log_rows"])
        return oracle.bit_reverse(x, c["log_rows"], c["cols"])
    if k == "powers":
        return oracle.powers_of(c["log_degree"], c["offset"], c["inv"], c["brev"], c["of_g"], c["count"])
    if k == "powby":
        return oracle.powers_by(powby_base(c), c["offset"], c["brev"], c["count"])
    if k == "oshift":
        x = words(c["name"], c["count"])
        return oracle.omega_shift(x, c["log_degree"], c["offset"], c["inv"], c["shift"])
    if k == "lagr":
        return oracle.lagrange_coeffs(lagr_point(c), 7, c["log_count"], c["brev"])
    if k == "beval":
        ys, coeffs = beval_inputs(c)
        return oracle.batch_eval(c["eval_kind"], ys, 1 << c["log_count"], c["num_polys"], coeffs)
    raise ValueError(k)
