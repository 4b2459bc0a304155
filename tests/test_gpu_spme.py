"""GPU tests of the electrostatics path through the C ABI: SPME charge mesh,
ik and analytic reciprocal forces/energies, real-space Ewald, self energy and
the FP64 exact Ewald sum, each against the CPU oracle (pinned to the
reference's own EleRecBSpline / EleRecFBSpline / EleRecES / EleDir built from
its sources, tests/test_spme_oracle.py), plus the charged-fluid benchmark
system (20736 charges, 64^3, order 6, beta 0.95) against an FP64 Ewald
reference."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

TOL = {0: 2e-5, 1: 1e-10}  # relative RMS force error, mixed / FP64


def rel_rms(a, b):
    return float(np.sqrt(((a - b) ** 2).sum() / (b ** 2).sum()))


@pytest.fixture(scope="module")
def small():
    rng = np.random.default_rng(0)
    n, L = 300, 9.0
    pos = rng.uniform(0, L, (n, 3))
    q = np.where(np.arange(n) < n // 2, 1.0, -1.0)
    rng.shuffle(q)
    return pos, q, np.array([L, L, L])


def make(mdf, pos, q, box, prec):
    sys = mdf.MDSystem(pos, box, charge=q, precision=prec)
    return sys


@pytest.mark.parametrize("prec", [0, 1])
def test_spread_mesh(mdf, orc, small, prec):
    pos, q, box = small
    sys = make(mdf, pos, q, box, prec)
    sp = mdf.SPME(sys, (16, 16, 32), 6, 1.3)
    sys.clear_stats()
    sp.apply()
    Q = sp.mesh()
    Qo = orc.spme_spread(pos, q, box, (16, 16, 32), 6)
    assert np.abs(Q - Qo).max() < (1e-5 if prec == 0 else 1e-12)


@pytest.mark.parametrize("method", ["ik", "analytic"])
@pytest.mark.parametrize("prec", [0, 1])
def test_reciprocal_forces_and_energy(mdf, orc, small, prec, method):
    pos, q, box = small
    K, order, beta = (16, 16, 32), 6, 1.3
    sys = make(mdf, pos, q, box, prec)
    sp = mdf.SPME(sys, K, order, beta, method)
    eng = mdf.InteractionEngine(sys)
    eng.clearInteraction()
    sys.clear_stats()
    sp.apply()
    F = sys.forces()
    E = sys.stats()[mdf.STAT_ELEC_REC]
    Eo, Fo = orc.spme_rec(pos, q, box, K, order, beta, 0 if method == "ik" else 1)
    assert rel_rms(F, Fo) < TOL[prec]
    assert abs(E - Eo) < 1e-6 * abs(Eo) + (1e-12 if prec else 1e-6)


def test_reciprocal_matches_reference_build(mdf, orc, small):
    if not orc.ref_available("libref_spme.so"):
        pytest.skip("reference SPME not built")
    pos, q, box = small
    sys = make(mdf, pos, q, box, 1)
    for method, m in (("ik", 0), ("analytic", 1)):
        sp = mdf.SPME(sys, (16, 16, 16), 6, 1.5, method)
        eng = mdf.InteractionEngine(sys)
        eng.clearInteraction()
        sys.clear_stats()
        sp.apply()
        ref = orc.ref_spme(sys.positions(), q, box, 1.5, (16, 16, 16), 4.0, m, 6)
        assert rel_rms(sys.forces(), ref["rec"]) < 1e-10


@pytest.mark.parametrize("prec", [0, 1])
def test_real_space_and_self(mdf, orc, small, prec):
    pos, q, box = small
    beta, rc = 1.3, 4.0
    sys = make(mdf, pos, q, box, prec)
    sys.set_rcut(np.full(len(q), rc, np.float32))
    eng = mdf.InteractionEngine(sys)
    eng.registNonBondedInteraction(0.0, 1.0, 0.0)  # LJ off (eps = 0)
    mdf.registCoulomb(eng, beta)
    cl = mdf.CellList(sys, rc + 0.3)
    cl.rebuild()
    nl = mdf.NeighborList(sys, rc + 0.3, 0.3, expansion=3.0)
    nl.fit(sys, cl)
    eng.clearInteraction()
    sys.clear_stats()
    eng.applyNonBondedInteraction(sys, nl, with_stats=True)
    F = sys.forces()
    E = sys.stats()[mdf.STAT_ELEC_DIR]
    gp = sys.positions()
    Eo, Fo = orc.ewald_dir(gp, q, box, beta, rc)
    assert rel_rms(F, Fo) < TOL[prec]
    assert abs(E - Eo) < (1e-5 if prec == 0 else 1e-10) * abs(Eo)
    es = mdf.ewald_self_energy(sys, beta)
    assert abs(es - orc.ewald_self(q, beta)) < 1e-10 * abs(es)


def test_exact_ewald_fp64(mdf, orc, small):
    pos, q, box = small
    sys = make(mdf, pos, q, box, 1)
    eng = mdf.InteractionEngine(sys)
    eng.clearInteraction()
    E = mdf.ewald_exact(sys, (10, 10, 10), 1.3)
    Eo, Fo = orc.ewald_rec_exact(sys.positions(), q, box, (10, 10, 10), 1.3)
    assert abs(E - Eo) < 1e-11 * abs(Eo)
    assert rel_rms(sys.forces(), Fo) < 1e-11


@pytest.mark.slow
def test_charged_fluid_against_fp64_ewald(mdf):
    """20736 +-1 charges, 30^3 box, mesh 64^3, order 6, beta 0.95, real-space
    rc 3.0, ik: the mixed path against FP64 real space (rc = 14.9, all pairs)
    plus the exact reciprocal sum (|m| <= 39, truncation < 1e-12)."""
    s = mdf.systems.charged_fluid()
    beta, K, order = 0.95, (64, 64, 64), 6
    out = {}
    for prec, rc, spme in ((0, 3.0, True), (1, 14.9, False)):
        sys = mdf.MDSystem(s.pos, s.box, charge=s.charge, precision=prec)
        sys.set_rcut(np.full(s.n, rc, np.float32))
        eng = mdf.InteractionEngine(sys)
        eng.registNonBondedInteraction(0.0, 1.0, 0.0)
        mdf.registCoulomb(eng, beta)
        cl = mdf.CellList(sys, 3.3)
        cl.rebuild()
        nl = mdf.NeighborList(sys, rc + 0.3, 0.3, expansion=1.2)
        nl.fit(sys, cl)
        eng.clearInteraction()
        sys.clear_stats()
        eng.applyNonBondedInteraction(sys, nl, with_stats=True)
        if spme:
            mdf.SPME(sys, K, order, beta, "ik").apply()
            e_rec = sys.stats()[mdf.STAT_ELEC_REC]
        else:
            e_rec = mdf.ewald_exact(sys, (78, 78, 78), beta)
        st = sys.stats()
        out[prec] = (sys.forces(), st[mdf.STAT_ELEC_DIR] + e_rec + mdf.ewald_self_energy(sys, beta))
    F, E = out[0]
    Fo, Eo = out[1]
    err = float(np.sqrt(((F - Fo) ** 2).sum(1).mean()))
    # real-space truncation at 3.0 plus SPME interpolation: a-priori ~1e-3 for
    # these parameters (errorEstimatePME / rec_BSpline::errorEstimate)
    assert err < 5e-3, err
    assert abs(E - Eo) / abs(Eo) < 1e-3


@pytest.mark.parametrize("prec", [0, 1])
def test_error_estimates_on_device(mdf, orc, small, prec):
    pos, q, box = small
    sys = make(mdf, pos, q, box, prec)
    c2 = float((q * q).sum())
    for K, order in (((16, 16, 32), 6), ((32, 32, 32), 4)):
        d, r = mdf.errorEstimatePME(sys, K, 1.3, 4.0)
        do, ro = orc.error_estimate_pme(box, K, 1.3, 4.0, c2, len(q))
        assert abs(d - do) < 1e-12 * do and abs(r - ro) < 1e-10 * ro
        e = mdf.errorEstimateInterpolRec(sys, K, order, 1.3)
        eo = orc.error_estimate_spme_ik(box, K, order, 1.3, c2, len(q))
        assert abs(e - eo) < 1e-10 * eo
    beta = mdf.choose_beta(sys, 4.0, 1e-4)
    d, _ = mdf.errorEstimatePME(sys, (16, 16, 16), beta, 4.0)
    assert abs(d - 1e-4) < 1e-9


@pytest.mark.parametrize("K,box,beta,order", [((8, 8, 16), (3.0, 3.0, 6.0), 2.5, 4),
                                              ((10, 12, 9), (3.1, 3.5, 2.9), 3.0, 6)])
def test_error_map_matches_oracle(mdf, orc, K, box, beta, order):
    rng = np.random.default_rng(2)
    rho1 = rng.normal(0, 5, K)
    rho2 = np.abs(rng.normal(30, 5, K))
    em = mdf.ErrorEstimate_SPME_Ik(K, box, beta, order)
    em.set_profile(rho1, rho2)
    e1, e2 = em.calError(1.0)
    o1, o2 = orc.spme_ik_errmap(K, box, beta, order, rho1, rho2, 1.0)
    assert np.abs(e1 - o1).max() < 1e-11 * np.abs(o1).max()
    assert np.abs(e2 - o2).max() < 1e-11 * np.abs(o2).max()


@pytest.mark.parametrize("K,box,beta,rc", [((8, 8, 24), (6.0, 6.0, 18.0), 2.5, 1.35),
                                           ((6, 5, 16), (5.0, 4.5, 14.0), 3.0, 1.2)])
def test_dir_error_map_matches_oracle(mdf, orc, K, box, beta, rc):
    """Real-space map (ErrorEstimate_dir) against the oracle, which matches the
    reference's own build to 1e-12; even and odd grid sizes."""
    rng = np.random.default_rng(3)
    rho1 = rng.normal(0, 5, K)
    rho2 = np.abs(rng.normal(30, 5, K))
    em = mdf.ErrorEstimate_dir(K, box, beta, rc)
    em.set_profile(rho1, rho2)
    e1, e2 = em.calError(1.0)
    o1, o2 = orc.dir_errmap(K, box, beta, rc, rho1, rho2, 1.0)
    assert np.abs(e1[..., 0] - o1[..., 0]).max() < 1e-10 * np.abs(o1[..., 0]).max()
    assert np.abs(e2[..., 0] - o2[..., 0]).max() < 1e-10 * np.abs(o2[..., 0]).max()
    assert np.all(np.isfinite(em.rms()))


def test_dir_error_map_rejects_unconverged_quadrature(mdf):
    """erfc(beta rcut) = 4e-4: the reference's 1e-20 quadrature would not finish;
    the map reports that instead of running on."""
    with pytest.raises(mdf.MDException):
        mdf.ErrorEstimate_dir((4, 4, 8), (6.0, 6.0, 18.0), 2.5, 1.0)


@pytest.mark.parametrize("K,box,beta,order", [((8, 8, 16), (3.0, 3.0, 6.0), 2.5, 4),
                                              ((7, 6, 5), (5.0, 4.0, 3.5), 1.8, 5),
                                              ((10, 12, 9), (3.1, 3.5, 2.9), 3.0, 6)])
def test_ana_error_map_matches_oracle(mdf, orc, K, box, beta, order):
    """Analytic-differentiation map (ErrorEstimate_SPME_Ana) against the oracle,
    which matches the reference's own build to 1e-12: error1, error2, the self
    error and FConvRho1 of every alias index; even and odd grids and orders."""
    rng = np.random.default_rng(4)
    rho1 = rng.normal(0, 5, K)
    rho2 = np.abs(rng.normal(30, 5, K))
    em = mdf.ErrorEstimate_SPME_Ana(K, box, beta, order)
    em.set_profile(rho1, rho2)
    e1, e2 = em.calError(1.3)
    o1, o2, oself, ofc = orc.spme_ana_errmap(K, box, beta, order, rho1, rho2, 1.3, with_fconv=True)
    for a, b in ((e1, o1), (e2, o2)):
        scale = np.abs(b[..., 0]).max()
        assert np.abs(a[..., 0] - b[..., 0]).max() < 1e-11 * scale
        assert np.abs(a[..., 1] - b[..., 1]).max() < 1e-9 * scale
    assert abs(em.self_error() - oself) <= 1e-11 * abs(oself)
    for slot, k in enumerate((-2, -1, 1, 2)):
        fc = em.fconv(k)
        assert np.abs(fc - ofc[slot]).max() < 1e-11 * np.abs(ofc[slot]).max()
    rms = em.rms(1.3)
    assert np.allclose(rms, np.sqrt(o1[..., 0] + o2[..., 0] + oself * 1.3 ** 4), rtol=1e-10, atol=0)


def test_ana_error_map_print_error_and_arguments(mdf, orc, tmp_path):
    K, box = (8, 8, 16), (3.0, 3.0, 6.0)
    rng = np.random.default_rng(5)
    rho1 = rng.normal(0, 5, K)
    rho2 = np.abs(rng.normal(30, 5, K))
    em = mdf.ErrorEstimate_SPME_Ana(K, box, 2.5, 4)
    em.set_profile(rho1, rho2)
    path = tmp_path / "error.out"
    em.print_error(str(path))
    rows = np.loadtxt(path)
    assert rows.shape == (K[0], 9)
    o1, o2, oself, _ = orc.spme_ana_errmap(K, box, 2.5, 4, rho1, rho2, 1.0)
    assert np.allclose(rows[:, 0], (np.arange(K[0]) + 0.5) * box[0] / K[0], atol=1e-6)
    assert np.allclose(rows[:, 1], np.sqrt(o1[:, 0, 0, 0] + o2[:, 0, 0, 0] + oself), rtol=1e-5)
    assert np.allclose(rows[:, 6], oself, rtol=1e-5)
    for k in (0, 3, -3):
        with pytest.raises(mdf.MDException):
            em.fconv(k)
    # the other maps have no self term and no FConvRho1
    import ctypes as C
    ik = mdf.ErrorEstimate_SPME_Ik(K, box, 2.5, 4)
    v = C.c_double(-1.0)
    assert mdf.lib.md_errmap_self_error(ik.h, C.byref(v)) == 0 and v.value == 0.0
    out = np.zeros((3,) + K + (2,))
    assert mdf.lib.md_errmap_ana_fconv(ik.h, 1, out.ctypes.data_as(C.POINTER(C.c_double))) == 11


def test_error_map_of_a_charged_slab(mdf, orc):
    """Deposited profile of a charged slab (analyze/app/error.spme.ik.cpp on a
    configuration): the profile and the error map against the oracle."""
    s = mdf.systems.charged_slab(n=8192, box=(20.0, 20.0, 80.0), half=12.0)
    K = (16, 16, 64)
    sys = mdf.MDSystem(s.pos, s.box, charge=s.charge, precision=1)
    em = mdf.ErrorEstimate_SPME_Ik(K, s.box, 1.0, 6)
    em.deposit(sys)
    rho1, rho2 = em.profile()
    h = s.box / np.array(K)
    idx = np.floor(np.mod(s.pos, s.box) / h).astype(int)
    idx = np.minimum(idx, np.array(K) - 1)
    c1 = np.zeros(K)
    c2 = np.zeros(K)
    np.add.at(c1, tuple(idx.T), np.sign(s.charge))
    np.add.at(c2, tuple(idx.T), 1.0)
    dv = np.prod(h)
    assert np.allclose(rho1, c1 / dv, rtol=0, atol=1e-12)
    assert np.allclose(rho2, c2 / dv, rtol=0, atol=1e-12)
    e1, e2 = em.calError(1.0)
    o1, o2 = orc.spme_ik_errmap(K, s.box, 1.0, 6, rho1, rho2, 1.0)
    # real parts are the estimate; the imaginary parts are transform rounding
    # (~1e-13) and are compared on the scale of the real parts
    for a, b in ((e1, o1), (e2, o2)):
        scale = np.abs(b[..., 0]).max()
        assert np.abs(a[..., 0] - b[..., 0]).max() < 1e-11 * scale
        assert np.abs(a[..., 1] - b[..., 1]).max() < 1e-9 * scale
    rms = em.rms(1.0)
    assert np.all(np.isfinite(rms)) and rms.max() > 0


@pytest.mark.parametrize("prec", [0, 1])
def test_self_correction(mdf, orc, small, prec):
    pos, q, box = small
    for K, order in (((16, 16, 32), 6), ((32, 16, 16), 4)):
        sys = make(mdf, pos, q, box, prec)
        sp = mdf.SPME(sys, K, order, 1.3, "analytic")
        eng = mdf.InteractionEngine(sys)
        eng.clearInteraction()
        sp.self_correction()
        Fo = orc.spme_selfcorr(sys.positions(), q, box, K, order, 1.3)
        assert np.abs(sys.forces() - Fo).max() < (1e-6 if prec == 0 else 1e-13) * np.abs(Fo).max()


def test_mean_force_field_matches_the_error1_components(mdf, orc):
    """print_meanf: the signed mean force error field; its squares summed over
    the three components are error1's real part."""
    K, box = (8, 8, 16), (3.0, 3.0, 6.0)
    rng = np.random.default_rng(6)
    rho1 = rng.normal(0, 5, K)
    rho2 = np.abs(rng.normal(30, 5, K))
    for em in (mdf.ErrorEstimate_SPME_Ik(K, box, 2.5, 4), mdf.ErrorEstimate_SPME_Ana(K, box, 2.5, 4)):
        em.set_profile(rho1, rho2)
        mf = em.mean_force(1.3)
        e1, _ = em.calError(1.3)
        assert mf.shape == (3,) + K
        assert np.allclose((mf ** 2).sum(axis=0), e1[..., 0], rtol=1e-12, atol=1e-14 * np.abs(e1[..., 0]).max())


def test_choose_spme_params_meets_target(mdf):
    """md_choose_spme_params on a charged liquid-vapour slab (4000 +-1 charges,
    16 x 16 x 48, liquid rho 0.8 for |z - 24| < 7.5, vapour elsewhere): both
    largest per-bin estimates within target / sqrt(2); each mesh axis needed
    (halving it breaks the reciprocal budget, by the ik map); and the FP64
    forces with the chosen beta and K (real space at rc 3 + ik SPME, order 6)
    within the target RMS of the converged Ewald sum (real space at rc 7.9,
    exact reciprocal sum to 1e-12)."""
    box = np.array([16.0, 16.0, 48.0])
    n = 4000
    thick, n_in = mdf.systems.slab_counts(n, box, 2, 0.8, 0.02)
    pos = mdf.systems.slab(n, n_in, box, 2, 24.0, 0.5 * thick, 0.8, 5)
    q = mdf.systems.charges(n, 6)
    target, rc, order = 2e-3, 3.0, 6
    sys = mdf.MDSystem(pos, box, charge=q, precision=1)
    beta, K, e_dir, e_rec = mdf.choose_spme_params(sys, rc, order, target, kmax=256)
    tb = target / np.sqrt(2)
    assert e_dir <= tb * (1 + 1e-9) and e_rec <= tb
    assert all(k & (k - 1) == 0 for k in K)
    for d in range(3):
        if K[d] // 2 <= order:
            continue
        Kh = list(K)
        Kh[d] //= 2
        em = mdf.ErrorEstimate_SPME_Ik(Kh, box, beta, order)
        em.deposit(sys)
        assert np.nanmax(em.rms(1.0)) > tb, (K, d)
    out = {}
    for which, rcut in (("chosen", rc), ("reference", 7.9)):
        s = mdf.MDSystem(pos, box, charge=q, precision=1)
        s.set_rcut(np.full(n, rcut, np.float32))
        eng = mdf.InteractionEngine(s)
        eng.registNonBondedInteraction(0.0, 1.0, 0.0)
        mdf.registCoulomb(eng, beta)
        cl = mdf.CellList(s, 3.3)
        cl.rebuild()
        nl = mdf.NeighborList(s, rcut + 0.3, 0.3, expansion=1.5)
        nl.fit(s, cl)
        eng.clearInteraction()
        eng.applyNonBondedInteraction(s, nl)
        if which == "chosen":
            mdf.SPME(s, K, order, beta, "ik").apply()
        else:
            mmax = [2 * int(np.ceil(1.67 * beta * L)) + 1 for L in box]
            mdf.ewald_exact(s, mmax, beta)
        out[which] = s.forces()
    err = float(np.sqrt(((out["chosen"] - out["reference"]) ** 2).sum(1).mean()))
    assert err < target, (err, beta, K, e_dir, e_rec)
