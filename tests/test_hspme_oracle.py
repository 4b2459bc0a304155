"""CPU tests of the Hermite-basis SPME oracle (oracle/hspme.py): with the
basis of the order-4 cardinal B-spline it is the reference SPME (the oracle's
spme_rec, pinned to RE/src/EleRecBSpline.cpp built here, in
tests/test_spme_oracle.py); its adjoint gradients of the energy and of the
force-error functional equal central differences."""
import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, os.path.join(ROOT, "md.error_b200"))


@pytest.fixture(scope="module")
def case():
    from oracle.hspme import HermiteSPME
    rng = np.random.default_rng(1)
    n, L = 24, 5.0
    r = rng.uniform(0, L, (n, 3))
    q = rng.uniform(-1, 1, n)
    hs = HermiteSPME((8, 8, 8), (L, L, L), 1.3, 2.0, 4)
    return hs, q, r, rng


def bspline4(CC, nbin):
    from mdforce.optibasis import bspline_initial_basis  # host code only
    return bspline_initial_basis(CC, nbin, 4)


def test_bspline_basis_is_reference_spme(orc):
    from oracle.hspme import HermiteSPME
    rng = np.random.default_rng(0)
    n, L = 40, 6.0
    r = rng.uniform(0, L, (n, 3))
    q = np.where(np.arange(n) % 2 == 0, 1.0, -1.0)
    hs = HermiteSPME((16, 16, 16), (L, L, L), 1.2, 2.0, 16)
    E, F, _ = hs.forward(bspline4(2.0, 16), q, r)
    Eo, Fo = orc.spme_rec(r, q, np.array([L, L, L]), (16, 16, 16), 4, 1.2, 0)
    assert abs(E - Eo) < 1e-13 * abs(Eo)
    # the Nyquist planes of the ik derivative: zeroed here, FFTW's c2r convention there
    assert np.linalg.norm(F - Fo) < 1e-6 * np.linalg.norm(Fo)


def test_energy_adjoint_vs_central_differences(case):
    hs, q, r, rng = case
    c = bspline4(2.0, 4) + rng.normal(0, 0.1, 8)
    E, F, dq, dr, dc = hs.energy_grad(c, q, r)
    h = 1e-6
    fd = np.array([(hs.forward(c + h * e, q, r)[0] - hs.forward(c - h * e, q, r)[0]) / (2 * h)
                   for e in np.eye(hs.ncoef)])
    assert np.linalg.norm(dc - fd) < 1e-8 * np.linalg.norm(fd)
    for i, d in ((3, 1), (17, 2)):
        rp, rm = r.copy(), r.copy()
        rp[i, d] += h
        rm[i, d] -= h
        assert abs((hs.forward(c, q, rp)[0] - hs.forward(c, q, rm)[0]) / (2 * h) - dr[i, d]) < 1e-7 * abs(dr).max()
        qp, qm = q.copy(), q.copy()
        qp[i] += h
        qm[i] -= h
        assert abs((hs.forward(c, qp, r)[0] - hs.forward(c, qm, r)[0]) / (2 * h) - dq[i]) < 1e-7 * abs(dq).max()


def test_force_error_adjoint_vs_central_differences(case):
    hs, q, r, rng = case
    c = bspline4(2.0, 4) + rng.normal(0, 0.1, 8)
    fref = rng.normal(0, 1, r.shape)
    L, dq, dr, dc = hs.force_error_grad(c, q, r, fref)

    def loss(cc, qq, rr):
        _, F, _ = hs.forward(cc, qq, rr)
        return ((F - fref) ** 2).sum() / rr.shape[0]

    h = 1e-6
    fd = np.array([(loss(c + h * e, q, r) - loss(c - h * e, q, r)) / (2 * h) for e in np.eye(hs.ncoef)])
    assert np.linalg.norm(dc - fd) < 1e-7 * np.linalg.norm(fd)
    for i, d in ((3, 1), (17, 2)):
        rp, rm = r.copy(), r.copy()
        rp[i, d] += h
        rm[i, d] -= h
        assert abs((loss(c, q, rp) - loss(c, q, rm)) / (2 * h) - dr[i, d]) < 1e-6 * abs(dr).max()
        qp, qm = q.copy(), q.copy()
        qp[i] += h
        qm[i] -= h
        assert abs((loss(c, qp, r) - loss(c, qm, r)) / (2 * h) - dq[i]) < 1e-6 * abs(dq).max()
