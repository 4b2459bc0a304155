"""CPU tests of the optiBasis error-functional oracle (oracle/ikerror.py)
against the values and basis gradients of the reference's own Python
(optiBasis/IkError.py HermiteLossFunc(_Bound0), fixtures made by
tests/golden/make_ikerror_golden.py), plus finite differences and the
factorised-vs-direct sum."""
import json
import os

import numpy as np
import pytest

from oracle.ikerror import IkErrorOracle, bspline_initial_basis

GOLDEN = os.path.join(os.path.dirname(__file__), "golden", "ikerror_cases.json")


def cases():
    with open(GOLDEN) as f:
        return json.load(f)["cases"]


def make(c):
    return IkErrorOracle(c["CC"], c["nbin"], c["beta"], c["KK"], c["L"], c["q2"], c["natoms"], c["l_cut"],
                         c["bound0"])


@pytest.fixture(scope="module", params=[c["name"] for c in cases()])
def case(request):
    c = next(c for c in cases() if c["name"] == request.param)
    return c, make(c)


def test_initial_basis_matches_reference(case):
    c, _ = case
    vv = bspline_initial_basis(c["CC"], c["nbin"], c["order"], c["bound0"])
    assert np.abs(vv - np.array(c["evals"][0]["vv"])).max() < 1e-13


def test_hat_matches_reference(case):
    c, o = case
    hat = o.phi(0, c["evals"][1]["vv"])
    assert np.abs(hat - np.array(c["hat_axis0_last"])).max() < 1e-15


def test_value_and_gradient_match_reference(case):
    c, o = case
    for e in c["evals"]:
        assert abs(o.value(e["vv"]) - e["value"]) < 1e-12 * e["value"]
        d, dr = o.deriv(e["vv"]), np.array(e["deriv"])
        assert np.abs(d - dr).max() < 1e-11 * np.abs(dr).max()


def test_gradient_against_central_differences(case):
    c, o = case
    vv = np.array(c["evals"][0]["vv"])
    g = o.deriv(vv)
    # five-point stencil, truncation O(h^4): the functional is strongly curved
    # through the 1/phi(m)^2 factors (a plain central difference at h = 1e-6
    # is only good to ~3e-6 here; the stencil at 1e-6 to ~1e-10)
    h = 1e-6
    for b in range(0, len(vv), max(1, len(vv) // 5)):
        e = np.zeros_like(vv)
        e[b] = h
        fd = (-o.value(vv + 2 * e) + 8 * o.value(vv + e) - 8 * o.value(vv - e) + o.value(vv - 2 * e)) / (12 * h)
        assert abs(fd - g[b]) < 1e-8 * np.abs(g).max(), (b, fd, g[b])


def test_factorised_sum_equals_triple_sum():
    c = next(c for c in cases() if c["name"] == "aniso")
    o = make(c)
    vv = c["evals"][1]["vv"]
    assert abs(o.sum_o1_direct(vv) / o.sum_o1(vv) - 1) < 1e-13
