"""CPU tests of the electrostatics oracle: B-spline basics, and ik / analytic
SPME, exact Ewald and real-space Ewald against the reference's own
ElectrostaticInteraction built from its sources (oracle/_ref/libref_spme.so),
on the same seeded inputs."""
import numpy as np
import pytest


def test_bspline_partition_of_unity_and_derivative(orc):
    for n in (2, 4, 6, 8):
        for f in (0.0, 0.13, 0.5, 0.91):
            w, dw = orc.bspline_weights(n, f)
            assert abs(w.sum() - 1.0) < 1e-14
            assert abs(dw.sum()) < 1e-13
            # derivative against a central difference of M_n (off the knots, where
            # M_2' jumps)
            h = 1e-6
            for j in range(n if f > 0 else 0):
                x = f + j
                fd = (orc.bspline(n, x + h) - orc.bspline(n, x - h)) / (2 * h) if 0 < x - h and x + h < n else None
                if fd is not None:
                    assert abs(dw[j] - fd) < 1e-6


def test_bspline_order4_closed_form(orc):
    # M_4 on [0,1): x^3/6
    for x in (0.1, 0.5, 0.9):
        assert abs(orc.bspline(4, x) - x ** 3 / 6) < 1e-15


@pytest.fixture(scope="module")
def charges():
    rng = np.random.default_rng(0)
    n, L = 200, 8.0
    pos = rng.uniform(0, L, (n, 3))
    q = np.where(np.arange(n) < n // 2, 1.0, -1.0)
    return pos, q, np.array([L, L, L])


@pytest.mark.parametrize("K,order,method", [((16, 16, 16), 6, 0), ((16, 16, 15), 4, 0), ((15, 15, 15), 6, 0),
                                            ((16, 12, 20), 6, 1), ((16, 16, 16), 8, 0)])
def test_spme_oracle_matches_reference_build(orc, charges, K, order, method):
    if not orc.ref_available("libref_spme.so"):
        pytest.skip("reference SPME not built (needs the reference tree at build time)")
    pos, q, box = charges
    ref = orc.ref_spme(pos, q, box, 1.5, K, 3.5, method, order)
    E, F = orc.spme_rec(pos, q, box, K, order, 1.5, method)
    Ed, Fd = orc.ewald_dir(pos, q, box, 1.5, 3.5)
    Es = orc.ewald_self(q, 1.5)
    tol = 1e-9 if order == 8 else 1e-11  # the reference evaluates M_8 from polynomial tables
    assert np.abs(F - ref["rec"]).max() < tol * np.abs(F).max() * 10
    assert np.abs(Fd - ref["dir"]).max() < 1e-12
    assert abs(E + Ed + Es - ref["energy"]) < tol * abs(ref["energy"]) * 10


def test_exact_ewald_oracle_matches_reference_build(orc, charges):
    if not orc.ref_available("libref_spme.so"):
        pytest.skip("reference SPME not built")
    pos, q, box = charges
    ref = orc.ref_spme(pos, q, box, 1.5, (10, 10, 10), 3.5, 2, 6)
    E, F = orc.ewald_rec_exact(pos, q, box, (10, 10, 10), 1.5)
    Ed, _ = orc.ewald_dir(pos, q, box, 1.5, 3.5)
    assert np.abs(F - ref["rec"]).max() < 1e-12
    assert abs(E + Ed + orc.ewald_self(q, 1.5) - ref["energy"]) < 1e-11 * abs(ref["energy"])


def test_spme_converges_to_exact_ewald(orc, charges):
    pos, q, box = charges
    Ee, Fe = orc.ewald_rec_exact(pos, q, box, (24, 24, 24), 1.5)
    errs = []
    for K in (16, 32):
        E, F = orc.spme_rec(pos, q, box, (K, K, K), 6, 1.5, 0)
        errs.append(np.sqrt(((F - Fe) ** 2).sum(1).mean()))
    assert errs[1] < errs[0] / 20


@pytest.mark.parametrize("K,order", [((16, 16, 16), 6), ((16, 12, 20), 4)])
def test_error_estimates_match_reference_build(orc, charges, K, order):
    if not orc.ref_available("libref_spme.so"):
        pytest.skip("reference SPME not built")
    pos, q, box = charges
    ref = orc.ref_spme(pos, q, box, 1.5, K, 3.5, 0, order)
    c2 = float((q * q).sum())
    d, r = orc.error_estimate_pme(box, K, 1.5, 3.5, c2, len(q))
    e = orc.error_estimate_spme_ik(box, K, order, 1.5, c2, len(q))
    assert abs(d - ref["err_dir"]) <= 1e-14 * ref["err_dir"]
    assert abs(r - ref["err_rec"]) <= 1e-13 * ref["err_rec"]
    assert abs(e - ref["err_interp"]) <= 1e-13 * ref["err_interp"]


@pytest.mark.parametrize("K,box,beta,order", [((8, 8, 16), (3.0, 3.0, 6.0), 2.5, 4),
                                              ((10, 12, 9), (3.1, 3.5, 2.9), 3.0, 6)])
def test_errmap_oracle_matches_reference_build(orc, K, box, beta, order):
    if not orc.ref_available("libref_errmap.so"):
        pytest.skip("reference error map not built")
    rng = np.random.default_rng(2)
    rho1 = rng.normal(0, 5, K)
    rho2 = np.abs(rng.normal(30, 5, K))
    a1, a2 = orc.spme_ik_errmap(K, box, beta, order, rho1, rho2, 1.0)
    b1, b2 = orc.ref_spme_ik_errmap(K, box, beta, order, rho1, rho2, 1.0)
    assert np.abs(a1 - b1).max() < 1e-12 * np.abs(b1).max()
    assert np.abs(a2 - b2).max() < 1e-12 * np.abs(b2).max()


def test_dft3d_matches_numpy(orc):
    rng = np.random.default_rng(3)
    a = rng.normal(size=(4, 6, 5)) + 1j * rng.normal(size=(4, 6, 5))
    assert np.abs(orc.dft3d(a, -1) - np.fft.fftn(a)).max() < 1e-12
    assert np.abs(orc.dft3d(a, +1) - np.fft.ifftn(a) * a.size).max() < 1e-12


@pytest.mark.parametrize("K,order", [((16, 16, 16), 6), ((16, 12, 15), 4), ((8, 16, 32), 8)])
def test_selfcorr_oracle_matches_reference_build(orc, charges, K, order):
    if not orc.ref_available("libref_spme.so"):
        pytest.skip("reference SPME not built")
    pos, q, box = charges
    box = np.array([box[0], box[1], box[2] * 1.125])
    a = orc.spme_selfcorr(pos, q, box, K, order, 1.5)
    b = orc.ref_selfcorr(pos, q, box, 1.5, K, order)
    assert np.abs(a - b).max() < 1e-12 * np.abs(b).max()


@pytest.mark.parametrize("K,box,beta,rc", [((8, 8, 24), (6.0, 6.0, 18.0), 2.5, 1.35),
                                           ((5, 6, 15), (5.0, 6.0, 15.0), 3.0, 1.2)])
def test_dir_errmap_oracle_matches_reference_build(orc, K, box, beta, rc):
    """ErrorEstimate_dir restated (oracle_errmap.c) against the reference's own
    analyze/src/ErrorEstimate_dir.cpp built in oracle/_ref."""
    if not orc.ref_available("libref_errdir.so"):
        pytest.skip("reference ErrorEstimate_dir not built (needs the reference tree at build time)")
    rng = np.random.default_rng(1)
    z = (np.arange(K[2]) + 0.5) * box[2] / K[2]
    rho2 = np.ascontiguousarray(np.broadcast_to(np.where(np.abs(z - box[2] / 2) < 4, 30.0, 1.0), K), np.float64)
    rho2 = rho2 * (1 + 0.1 * rng.random(K))
    rho1 = np.ascontiguousarray(rho2 * 0.1 * (rng.random(K) - 0.5))
    a1, a2 = orc.dir_errmap(K, box, beta, rc, rho1, rho2, 1.0)
    b1, b2 = orc.ref_dir_errmap(K, box, beta, rc, rho1, rho2, 1.0)
    assert np.abs(a1 - b1).max() < 1e-12 * np.abs(b1).max()
    assert np.abs(a2[..., 0] - b2[..., 0]).max() < 1e-12 * np.abs(b2[..., 0]).max()


@pytest.mark.parametrize("K,box,beta,order", [((8, 8, 16), (3.0, 3.0, 6.0), 2.5, 4),
                                              ((7, 6, 5), (5.0, 4.0, 3.5), 1.8, 5),
                                              ((10, 12, 9), (3.1, 3.5, 2.9), 3.0, 6)])
def test_ana_errmap_oracle_matches_reference_build(orc, K, box, beta, order):
    """ErrorEstimate_SPME_Ana restated (oracle_errmap.c) against the reference's own
    analyze/src/ErrorEstimate_SPME_Ana.cpp built in oracle/_ref: error1, error2, the
    self error and FConvRho1; even and odd grids, even and odd orders."""
    if not orc.ref_available("libref_errana.so"):
        pytest.skip("reference ErrorEstimate_SPME_Ana not built (needs the reference tree at build time)")
    rng = np.random.default_rng(4)
    rho1 = rng.normal(0, 5, K)
    rho2 = np.abs(rng.normal(30, 5, K))
    a1, a2, aself, afc = orc.spme_ana_errmap(K, box, beta, order, rho1, rho2, 1.3, with_fconv=True)
    b1, b2, bself, bfc = orc.ref_spme_ana_errmap(K, box, beta, order, rho1, rho2, 1.3, with_fconv=True)
    # real parts are the estimate; the imaginary parts are transform rounding and
    # are compared on the scale of the real parts
    for a, b in ((a1, b1), (a2, b2)):
        scale = np.abs(b[..., 0]).max()
        assert np.abs(a[..., 0] - b[..., 0]).max() < 1e-12 * scale
        assert np.abs(a[..., 1] - b[..., 1]).max() < 1e-12 * scale
    assert abs(aself - bself) <= 1e-12 * abs(bself)
    assert np.abs(afc - bfc).max() < 1e-12 * np.abs(bfc).max()
