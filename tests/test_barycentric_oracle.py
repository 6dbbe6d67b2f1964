"""CPU checks of the oracle's barycentric evaluation (src/barycentric.rs).

The reference's tests (src/barycentric.rs:307-683) evaluate random polynomials
at a random point two ways: Horner on the coefficients, and barycentric
evaluation of the polynomial's values on the coset 7 * H (computed with
batch_ntt_in_place, natural -> bit-reversed, log_extension_degree 1, coset 0)
with bit-reversed Lagrange coefficients.  The same identity pins the oracle
here, with the oracle's own NTT; plus the coefficient formula checked in pure
Python and the reference's zero convention for a point inside the domain.
"""
import numpy as np
import pytest

import oracle
from conftest import P, uniform


def _coset_values(a: np.ndarray, log_n: int, cols: int) -> np.ndarray:
    n = 1 << log_n
    return oracle.batch_ntt(a, log_n, cols, n, n, False, False, 1, 0) if log_n else a.copy()


@pytest.mark.parametrize("log_n", [0, 1, 2, 5, 9])
def test_barycentric_equals_horner(log_n):
    rng = np.random.default_rng(10 + log_n)
    n, cols = 1 << log_n, 3
    a = uniform(rng, cols * n)
    ys = _coset_values(a, log_n, cols)
    x = int(uniform(rng, 1)[0])
    got = oracle.batch_eval(oracle.EVAL_BASE_AT_BASE, ys, n, cols, oracle.lagrange_coeffs(x, 7, log_n, True))
    exp = oracle.poly_eval(a, n, cols, x)
    assert [int(v) for v in got] == [int(v) for v in exp[0::2]]
    xe = tuple(int(v) for v in uniform(rng, 2))
    le = oracle.lagrange_coeffs(xe, 7, log_n, True)
    got = oracle.batch_eval(oracle.EVAL_BASE_AT_EXT, ys, n, cols, le)
    np.testing.assert_array_equal(got, oracle.poly_eval(a, n, cols, xe))
    # extension values: each coordinate column transformed on its own (the NTT is F_p-linear)
    ae = uniform(rng, 2 * cols * n)
    yse = _coset_values(ae, log_n, 2 * cols)
    got = oracle.batch_eval(oracle.EVAL_EXT_AT_EXT, yse, n, cols, le)
    np.testing.assert_array_equal(got, oracle.poly_eval(ae, n, cols, xe, ext_coeffs=True))


def test_coefficient_formula():
    """L_i = c (x^N - c^N) / (N c^N) * w^i / (x - c w^i), natural order, pure Python."""
    log_n, c = 4, 7
    n = 1 << log_n
    x = 123456789
    w = oracle.root_of_unity(log_n)
    cf = c * (pow(x, n, P) - pow(c, n, P)) * pow(n * pow(c, n, P), P - 2, P) % P
    got = oracle.lagrange_coeffs(x, c, log_n, False)
    for i in range(n):
        wi = pow(w, i, P)
        assert int(got[i]) == cf * wi * pow((x - c * wi) % P, P - 2, P) % P


def test_point_in_domain_gives_zeros():
    """x = c w^5: the reference's batch inverse of a zero is zero and cf = 0, so every coefficient is 0."""
    log_n = 4
    x = 7 * pow(oracle.root_of_unity(log_n), 5, P) % P
    assert not oracle.lagrange_coeffs(x, 7, log_n, False).any()
    assert not oracle.lagrange_coeffs((x, 0), 7, log_n, True).any()
