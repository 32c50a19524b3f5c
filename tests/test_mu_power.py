"""mu = T**0.666 (ModAssign.f90:20, Tvec**0.666D0) as the FP64 kernels form it.

The kernels evaluate the power from tables (a table-driven reduction with a binomial
series, axj_pow.cuh); axj_mu_of_T runs the same operations on the host. The oracle
computes C's pow(T, 0.666), as the reference's T**0.666D0 does. The table-driven
power stays within 1 ulp of pow for T in [2^-16, 2^16) and equals it at almost every
point; outside that range and for zero, negative or non-finite T it takes
exp2(0.666 log2 T), with pow's special values.
"""
import math

import numpy as np
import pytest

import axisymmetricjet_b200 as axj


@pytest.fixture(scope="module")
def mu_of_t():
    lib = axj.load_library()
    return lib.axj_mu_of_T


def _ulps(a, b):
    return np.abs(np.asarray(a).view(np.int64) - np.asarray(b).view(np.int64))


@pytest.mark.parametrize("lo,hi", [(0.3, 3.0), (2.0 ** -16, 2.0 ** 16 * (1 - 1e-12)), (0.999, 1.001)])
def test_within_one_ulp_of_pow(mu_of_t, lo, hi):
    rng = np.random.default_rng(20)
    T = np.exp(rng.uniform(math.log(lo), math.log(hi), 40000))
    got = np.array([mu_of_t(float(t)) for t in T])
    ref = np.array([math.pow(float(t), 0.666) for t in T])
    d = _ulps(got, ref)
    assert d.max() <= 1
    assert (d > 0).mean() < 0.01


def test_table_edges_and_interval_boundaries(mu_of_t):
    # every mantissa interval and exponent of the tables, at both ends of each interval
    vals = []
    for e in range(-16, 16):
        for j in range(128):
            m0 = 1.0 + j / 128.0
            vals += [math.ldexp(m0, e), math.ldexp(np.nextafter(m0 + 1.0 / 128.0, 0.0), e)]
    got = np.array([mu_of_t(v) for v in vals])
    ref = np.array([math.pow(v, 0.666) for v in vals])
    assert _ulps(got, ref).max() <= 1


def test_special_values(mu_of_t):
    assert mu_of_t(0.0) == 0.0
    assert mu_of_t(1.0) == 1.0
    assert math.isnan(mu_of_t(-1.0))
    assert math.isnan(mu_of_t(float("nan")))
    assert mu_of_t(float("inf")) == float("inf")
    # outside the tables' exponents: the exp2 / log2 form (its error grows with |log2 T|)
    for t in (1e-6, 3e5, 1e-310):
        assert abs(mu_of_t(t) / math.pow(t, 0.666) - 1.0) < 1e-13
